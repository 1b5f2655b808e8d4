"""GPU parity of the B200 provider, called through its C ABI (via the plan API).

* the reference's own known-answer cases (tests/sycl_tests.cpp:318-399 and
  tests/host_tests.cpp:133-165, as golden fixtures) with the reference's bound
  |a - e| <= tol * (1 + |e|);
* parity with the oracle (CPU restatement of the portable provider) and with an
  FP64 FFT on the same seeded inputs at sizes the oracle finishes in seconds;
  tolerance: rel-L2 <= 1e-5 * log2(N) (float) / 1e-12 * log2(N) (double) against
  FP64, and against the oracle max(that, 2 * oracle's own FP64 error) because the
  reference forms its Bluestein chirp angle in float (7e-3 rel-L2 at N=65537);
* the full benchmark sizes through size-independent properties: forward/backward
  round trip, linearity, Parseval, and FP64 checks of sampled lines.
"""
import json
import math
import os

import numpy as np
import pytest

from conftest import fp64_fft, gaussian_complex, norm_scale, rel_l2, uniform_complex

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


@pytest.fixture(scope="module")
def sf():
    import syclfft_b200
    return syclfft_b200


def spec_tol(n, dbl):
    return (1e-12 if dbl else 1e-5) * max(1.0, math.log2(max(n, 2)))


def run(sf, torch, x, shape, batch, d, norm=0, dbl=False, in_place=False):
    opts = sf.plan_options(placement=sf.placement.in_place if in_place else sf.placement.out_of_place,
                           normalization=sf.normalization(norm))
    p = sf.plan_many_dft("double" if dbl else "float", shape, batch, d, opts)
    xt = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    if in_place:
        p.execute(xt).synchronize()
        out = xt
    else:
        out = torch.empty_like(xt)
        p.execute(xt, out).synchronize()
    return out.cpu().numpy(), p


def golden_cases():
    return json.load(open(os.path.join(GOLDEN, "golden.json")))["cases"]


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c["name"])
def test_reference_known_answers(sf, torch, case):
    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    x, y = g[case["name"] + "__x"], g[case["name"] + "__y"]
    dt = np.complex128 if case["double"] else np.complex64
    out, p = run(sf, torch, x.astype(dt), case["shape"], case["batch"], case["direction"],
                 ["none", "forward", "backward", "orthogonal"].index(case["norm"]), case["double"],
                 case["placement"] == "in_place")
    assert np.all(np.abs(out - y) <= case["tol"] * (1 + np.abs(y))), case["source"]
    assert p.selected_provider() == sf.provider.b200


def test_round_trip_13_chained(sf, torch):
    # sycl_tests.cpp:372-399: forward then backward (backward normalization), chained by an event
    x = np.load(os.path.join(GOLDEN, "golden.npz"))["roundtrip13__x"].astype(np.complex64)
    fwd = sf.plan_dft_1d("float", 13, sf.direction.forward)
    bwd = sf.plan_dft_1d("float", 13, sf.direction.backward,
                         sf.plan_options(normalization=sf.normalization.backward))
    xt = torch.from_numpy(x).cuda()
    spec = torch.empty_like(xt)
    back = torch.empty_like(xt)
    done = fwd.execute(xt, spec)
    bwd.execute(spec, back, dependencies=[done]).synchronize()
    assert np.max(np.abs(back.cpu().numpy() - x)) < 2e-3


def test_repeated_and_concurrent_plans(sf, torch):
    # sycl_tests.cpp:231-256 (repeat on one plan) and 410-435 (two plans)
    a = torch.zeros(8, dtype=torch.complex64, device="cuda"); a[0] = 1
    b = torch.zeros(8, dtype=torch.complex64, device="cuda"); b[1] = 1
    p1 = sf.plan_dft_1d("float", 8, sf.direction.forward)
    p2 = sf.plan_dft_1d("float", 8, sf.direction.forward)
    oa, ob, oa2 = torch.empty_like(a), torch.empty_like(b), torch.empty_like(a)
    s2 = torch.cuda.Stream()
    e1 = p1.execute(a, oa)
    e2 = p2.execute(b, ob, stream=s2)
    e3 = p1.execute(a, oa2)
    for e in (e1, e2, e3):
        e.synchronize()
    assert torch.allclose(oa, torch.ones_like(oa), atol=1e-5)
    assert torch.equal(oa, oa2)
    assert abs(ob[0].real.item() - 1.0) < 1e-5


def test_event_span_dependency(sf, torch):
    # sycl_tests.cpp:483-506: two producers on another stream, FFT waits on both events
    x = torch.empty(8, dtype=torch.complex64, device="cuda")
    out = torch.empty_like(x)
    prod = torch.cuda.Stream()
    with torch.cuda.stream(prod):
        x[:4] = torch.tensor([1, 0, 0, 0], dtype=torch.complex64, device="cuda")
        e1 = torch.cuda.Event(); e1.record(prod)
        x[4:] = 0
        e2 = torch.cuda.Event(); e2.record(prod)
    p = sf.plan_dft_1d("float", 8, sf.direction.forward)
    p.execute(x, out, dependencies=[e1, e2]).synchronize()
    assert torch.allclose(out, torch.ones_like(out), atol=1e-5)


PARITY = [
    # (shape, batch, double, gaussian)
    ([1024], 16, False, False),
    ([4096], 64, False, False),
    ([13440], 8, False, False),
    ([16384], 4, False, False),
    ([65536], 4, True, False),
    ([32768], 4, False, False),
    ([8192], 8, True, False),
    ([1009], 16, False, True),
    ([1009], 16, True, True),
    ([4099], 4, False, True),
    ([4099], 4, True, True),
    ([65537], 2, False, True),
    ([65537], 2, True, True),
    ([64, 64, 64], 1, False, False),
    ([256, 256], 1, True, False),
    ([2048, 32], 1, True, False),
    ([11, 3], 1, False, False),
    ([40000, 3], 1, False, False),
    ([257, 5], 2, True, True),
    ([6], 5, False, False),
    ([35], 3, True, False),
    ([1], 7, False, False),
]


@pytest.mark.parametrize("shape,batch,dbl,gauss", PARITY, ids=lambda v: str(v))
def test_parity_vs_oracle_and_fp64(sf, torch, oracle_mod, shape, batch, dbl, gauss):
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    gen = gaussian_complex if gauss else uniform_complex
    x = gen(n * batch, 1000 + n, dt)
    for d, norm in ((-1, 1), (1, 3)):
        out, _ = run(sf, torch, x, shape, batch, d, norm, dbl)
        ref64 = fp64_fft(x, shape, batch, d, norm_scale(norm, d, n))
        ora = oracle_mod.OraclePlan(shape, batch, d, norm, dbl).execute(x)
        e64 = rel_l2(out, ref64)
        e_or = rel_l2(out, ora)
        e_or64 = rel_l2(ora, ref64)
        tol = spec_tol(n, dbl)
        assert e64 <= tol, f"vs FP64 {e64:.3e} > {tol:.3e}"
        assert e_or <= max(tol, 2 * e_or64), f"vs oracle {e_or:.3e} (oracle vs FP64 {e_or64:.3e})"


def test_config1_exact_case_vs_oracle(sf, torch, oracle_mod):
    """The CPU-baseline workload exactly: complex<float> N=1024, batch 1, forward, out of place,
    normalization none, re/im ~ U[-1, 1) from a seed; against the oracle and FP64."""
    n = 1024
    x = uniform_complex(n, 1, np.complex64)
    out, p = run(sf, torch, x, [n], 1, -1, 0, False, in_place=False)
    assert p.batch_count() == 1
    ref64 = fp64_fft(x, [n], 1, -1)
    ora = oracle_mod.OraclePlan([n], 1, -1, 0, False).execute(x)
    tol = spec_tol(n, False)
    assert rel_l2(out, ref64) <= tol
    assert rel_l2(out, ora) <= max(tol, 2 * rel_l2(ora, ref64))
    # the reference's element-wise bound (sycl_tests.cpp:242, float 4e-4) holds as well
    assert np.all(np.abs(out - ora) <= 4e-4 * (1 + np.abs(ora)))


LEAN = [
    # (length, batch, double, stage radices the planner gives the first pass)
    ([810], 33, False, [2, 15, 3, 3, 3]),
    ([3000], 9, False, [8, 15, 5, 5]),
    ([105], 40, False, [15, 7]),
    ([45], 100, False, [15, 3]),
    ([2187], 4, False, [3, 3, 3, 3, 3, 3, 3]),
    ([6125], 3, False, [5, 5, 5, 7, 7]),
    ([840], 17, True, [8, 3, 5, 7]),
    ([1125], 5, True, [3, 3, 5, 5, 5]),
    ([30000], 3, False, [2, 15, 5]),
    ([680400], 2, False, [2, 15, 3, 3, 3]),
    ([784000], 1, True, [5, 5, 5, 7]),
]


@pytest.mark.parametrize("shape,batch,dbl,radices", LEAN, ids=lambda v: str(v))
def test_runtime_length_lean_kernel(sf, torch, shape, batch, dbl, radices):
    """7-smooth lengths without a size-specialised kernel run on the lean runtime-length kernel
    (whole lines, or the column and row passes of a four-step), whose stages form each
    butterfly's twiddles from one base twiddle and, at 16 values a thread, run a (3, 5) pair of
    stages as one radix-15 stage: both directions and two normalizations against an FP64 FFT."""
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 4242 + n, dt)
    for d, norm in ((-1, 0), (1, 3)):
        out, p = run(sf, torch, x, shape, batch, d, norm, dbl)
        passes = p.describe()["passes"]
        assert all(ps["lean"] for ps in passes), passes
        assert passes[0]["radices"] == radices
        assert rel_l2(out, fp64_fft(x, shape, batch, d, norm_scale(norm, d, n))) <= spec_tol(n, dbl)


GENERIC = [([4096], 16, False), ([13440], 2, False), ([256, 64], 2, True), ([64, 48, 40], 1, False),
           ([2048], 8, True), ([128, 256], 2, False), ([65536], 4, True)]


@pytest.mark.parametrize("cluster", ["8", "16", "off"])
@pytest.mark.parametrize("shape,batch,dbl", [([65536], 6, True), ([65536], 3, False), ([131072], 2, False),
                                             ([32768], 5, True), ([32768], 4, False)], ids=lambda v: str(v))
def test_long_line_paths(sf, torch, shape, batch, dbl, cluster, monkeypatch):
    """Long lines on the cluster kernel (cluster sizes 8 and 16) and on the two-pass four-step."""
    monkeypatch.setenv("SYCLFFT_B200_CLUSTER", cluster)
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 5 + n, dt)
    for d, norm in ((-1, 3), (1, 1)):
        out, p = run(sf, torch, x, shape, batch, d, norm, dbl)
        kinds = [ps["kind"] for ps in p.describe()["passes"]]
        assert kinds == (["fourstep_cols", "fourstep_rows"] if cluster == "off" else ["cluster"]), kinds
        assert rel_l2(out, fp64_fft(x, shape, batch, d, norm_scale(norm, d, n))) <= spec_tol(n, dbl)
    xt = torch.from_numpy(x).cuda()
    keep = xt.clone()
    ip = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction.forward,
                          sf.plan_options(placement=sf.placement.in_place))
    ip.execute(xt).synchronize()
    assert rel_l2(xt.cpu().numpy(), fp64_fft(keep.cpu().numpy(), shape, batch, -1)) <= spec_tol(n, dbl)


@pytest.mark.parametrize("shape,batch,dbl", GENERIC, ids=lambda v: str(v))
def test_generic_kernel_path(sf, torch, oracle_mod, shape, batch, dbl, monkeypatch):
    """The runtime-parameterised kernel (the fallback for sizes without a specialised
    kernel) on sizes that normally take the specialised one."""
    monkeypatch.setenv("SYCLFFT_B200_KERNELS", "generic")
    monkeypatch.setenv("SYCLFFT_B200_CLUSTER", "off")
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 77 + n, dt)
    out, p = run(sf, torch, x, shape, batch, 1, 2, dbl)
    assert all(ps["fixed_id"] == -1 for ps in p.describe()["passes"])
    assert rel_l2(out, fp64_fft(x, shape, batch, 1, 1.0 / n)) <= spec_tol(n, dbl)


@pytest.mark.parametrize("piped", ["1", "0"])
@pytest.mark.parametrize("shape,batch,dbl", [([13440], 300, False), ([8192], 200, False), ([13440], 3, False)],
                         ids=lambda v: str(v))
def test_pipelined_kernel(sf, torch, shape, batch, dbl, piped, monkeypatch):
    """Persistent copy-engine-pipelined kernel (many lines per CTA) vs the plain kernel, both
    directions, in place and out of place, with unaligned buffers falling back to the plain kernel."""
    monkeypatch.setenv("SYCLFFT_B200_PIPED", piped)
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 31 + n, dt)
    for d, norm in ((-1, 3), (1, 1)):
        out, p = run(sf, torch, x, shape, batch, d, norm, dbl)
        ids = [ps["piped_id"] for ps in p.describe()["passes"]]
        assert (ids[0] >= 0) == (piped == "1"), ids
        assert rel_l2(out, fp64_fft(x, shape, batch, d, norm_scale(norm, d, n))) <= spec_tol(n, dbl)
    out, _ = run(sf, torch, x, shape, batch, -1, 0, dbl, in_place=True)
    assert rel_l2(out, fp64_fft(x, shape, batch, -1)) <= spec_tol(n, dbl)
    # 8-byte-aligned (not 16) buffers: the provider must take the plain kernel
    xt = torch.from_numpy(np.concatenate([np.zeros(1, dt), x])).cuda()
    yt = torch.empty_like(xt)
    p = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction.forward)
    from syclfft_b200 import _provider
    import ctypes
    err = ctypes.create_string_buffer(1024)
    es = xt.element_size()
    rc = p._api.execute(p._handle, xt.data_ptr() + es, yt.data_ptr() + es, torch.cuda.current_stream().cuda_stream,
                        err, 1024)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    assert rel_l2(yt[1:].cpu().numpy(), fp64_fft(x, shape, batch, -1)) <= spec_tol(n, dbl)
    assert p._lib.syclfft_b200_plan_status(p._handle) == 0


def test_in_place_multi_axis(sf, torch):
    x = uniform_complex(2 * 12 * 40 * 9, 3)
    out, _ = run(sf, torch, x.copy(), [12, 40, 9], 2, -1, 0, False, in_place=True)
    assert rel_l2(out, fp64_fft(x, [12, 40, 9], 2, -1)) < spec_tol(12 * 40 * 9, False)


def test_out_of_place_keeps_input(sf, torch):
    for shape, dbl in (([4096], False), ([65536], True), ([65537], False), ([64, 64, 64], False)):
        n = int(np.prod(shape))
        x = torch.randn(2 * n, dtype=torch.complex128 if dbl else torch.complex64, device="cuda")
        keep = x.clone()
        p = sf.plan_many_dft("double" if dbl else "float", shape, 2, sf.direction.forward)
        out = torch.empty_like(x)
        p.execute(x, out).synchronize()
        assert torch.equal(x, keep)


# Full benchmark sizes, checked through size-independent properties.
FULL = [([4096], 16384, False), ([13440], 4096, False), ([65536], 512, True)]


@pytest.mark.parametrize("shape,batch,dbl", FULL, ids=lambda v: str(v))
def test_full_size_properties(sf, torch, shape, batch, dbl):
    n = int(np.prod(shape))
    cdt = torch.complex128 if dbl else torch.complex64
    g = torch.Generator(device="cuda").manual_seed(n)
    x = (torch.rand(batch * n, device="cuda", generator=g, dtype=torch.float64 if dbl else torch.float32) * 2 - 1)
    x = torch.complex(x, torch.roll(x, 1)).to(cdt)
    orig = x.clone()
    opts = sf.plan_options(placement=sf.placement.in_place, normalization=sf.normalization.orthogonal)
    kind = "double" if dbl else "float"
    fwd = sf.plan_many_dft(kind, shape, batch, sf.direction.forward, opts)
    bwd = sf.plan_many_dft(kind, shape, batch, sf.direction.backward, opts)
    fwd.execute(x).synchronize()
    # Parseval with orthogonal normalization
    e_in = torch.linalg.vector_norm(orig.to(torch.complex128)).item()
    e_out = torch.linalg.vector_norm(x.to(torch.complex128)).item()
    assert abs(e_out - e_in) / e_in < spec_tol(n, dbl)
    # sampled lines against FP64
    rows = np.random.default_rng(0).choice(batch, 8, replace=False)
    xs = orig.view(batch, n)[rows].cpu().numpy()
    ys = x.view(batch, n)[rows].cpu().numpy()
    assert rel_l2(ys, np.fft.fft(xs.astype(np.complex128), axis=1) / math.sqrt(n)) < spec_tol(n, dbl)
    # round trip
    bwd.execute(x).synchronize()
    assert rel_l2(x.cpu().numpy(), orig.cpu().numpy()) < 2 * spec_tol(n, dbl)
    # linearity: F(a + 2b) = F(a) + 2 F(b)
    a, b = orig[: n * 64].clone(), torch.roll(orig[: n * 64], 7).clone()
    f64 = sf.plan_many_dft(kind, shape, 64, sf.direction.forward, opts)
    lhs = a + 2 * b
    f64.execute(lhs); f64.execute(a); f64.execute(b)
    torch.cuda.synchronize()
    assert rel_l2((a + 2 * b).cpu().numpy(), lhs.cpu().numpy()) < 2 * spec_tol(n, dbl)


def test_bluestein_full_config_vs_fp64(sf, torch):
    # config 3: N in {1009, 4099, 65537} x batch 256, out-of-place, forward normalization, N(0,1)
    for n in (1009, 4099, 65537):
        for dbl in (False, True):
            dt = np.complex128 if dbl else np.complex64
            x = gaussian_complex(256 * n, n, dt)
            out, _ = run(sf, torch, x, [n], 256, -1, 1, dbl)
            ref = fp64_fft(x, [n], 256, -1, 1.0 / n)
            assert rel_l2(out, ref) < spec_tol(n, dbl)


def test_multidim_full_configs(sf, torch):
    # config 4: 3D c64 256^3 in place fwd+bwd (backward norm); 2D c128 2048^2 out of place
    rng = np.random.default_rng(4)
    x = uniform_complex(256 ** 3, 11)
    idx = np.indices((256, 256, 256)).reshape(3, -1).T
    for _ in range(8):
        k = rng.integers(0, 256, 3)
        x += (rng.uniform(0.5, 2) * np.exp(2j * np.pi * (idx @ k) / 256 + 1j * rng.uniform(0, 2 * np.pi))).astype(np.complex64)
    orig = x.copy()
    opts = sf.plan_options(placement=sf.placement.in_place, normalization=sf.normalization.backward)
    f = sf.plan_dft_3d("float", 256, 256, 256, sf.direction.forward, opts)
    b = sf.plan_dft_3d("float", 256, 256, 256, sf.direction.backward, opts)
    xt = torch.from_numpy(x).cuda()
    f.execute(xt).synchronize()
    assert rel_l2(xt.cpu().numpy(), fp64_fft(orig, [256, 256, 256], 1, -1)) < spec_tol(256 ** 3, False)
    b.execute(xt).synchronize()
    assert rel_l2(xt.cpu().numpy(), orig) < 2 * spec_tol(256 ** 3, False)
    y = uniform_complex(2048 * 2048, 12, np.complex128)
    out, _ = run(sf, torch, y, [2048, 2048], 1, -1, 0, True)
    assert rel_l2(out, fp64_fft(y, [2048, 2048], 1, -1)) < spec_tol(2048 * 2048, True)


@pytest.mark.parametrize("shape,batch,dbl", [([65536], 6, True), ([65536], 5, False), ([16384], 7, True),
                                             ([131072], 2, False)], ids=str)
def test_tma_staged_column_pass(shape, batch, dbl, monkeypatch):
    """Four-step plans with the column pass on the TMA-staged kernel (tensor-map box loads into
    shared memory, opt-in), forward and backward, against FP64."""
    import torch
    import syclfft_b200 as sf
    monkeypatch.setenv("SYCLFFT_B200_TMA", "1")
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 31 + n, dt)
    for d in (sf.direction.forward, sf.direction.backward):
        p = sf.plan_many_dft("double" if dbl else "float", shape, batch, d)
        assert any(ps.get("tma") for ps in p.describe()["passes"]), p.describe()
        xi = torch.from_numpy(x).cuda()
        out = torch.empty_like(xi)
        p.execute(xi, out).synchronize()
        ref = fp64_fft(x, shape, batch, int(d))
        tol = (1e-12 if dbl else 1e-5) * math.log2(n)
        assert rel_l2(out.cpu().numpy(), ref) <= tol


@pytest.mark.parametrize("in_place", [False, True])
def test_pipelined_cluster_kernel(sf, torch, in_place, monkeypatch):
    """complex<double> 65536-point lines in one pass on 16-CTA clusters (opt-in
    SYCLFFT_B200_CLUSTER=pipe): both directions and a normalization against FP64, more lines than
    resident clusters so every cluster walks several lines."""
    monkeypatch.setenv("SYCLFFT_B200_CLUSTER", "pipe")
    n, batch = 65536, 37
    x = uniform_complex(n * batch, 65, np.complex128)
    for d, norm in ((-1, 0), (1, 3)):
        out, p = run(sf, torch, x, [n], batch, d, norm, True, in_place)
        passes = p.describe()["passes"]
        assert len(passes) == 1 and passes[0]["cluster_pipe"] == 1, passes
        ref = fp64_fft(x, [n], batch, d, norm_scale(norm, d, n))
        assert rel_l2(out, ref) <= spec_tol(n, True)


@pytest.mark.parametrize("shape,batch,dbl", [([65536], 8, False), ([65536], 6, True), ([65521], 6, False),
                                             ([65521], 5, True), ([4099], 6, True), ([24, 65536], 1, False),
                                             ([13440], 7, False)],
                         ids=lambda v: str(v))
def test_fused_multipass_matches_separate_passes(sf, torch, monkeypatch, shape, batch, dbl):
    """The fused launches (four-step columns + rows, Bluestein forward columns + rows + inverse
    columns, with the intermediate in an L2-resident ring) against the same plan's separate
    passes (SYCLFFT_B200_FUSED4=0) and FP64, both directions through execute_ex, with every
    normalization."""
    import ctypes
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 31 + n, dt)
    xi = torch.from_numpy(x).cuda()
    outs = {}
    # 13440 fits one block: its fused four-step (112 x 120) is the opt-in alternative to the
    # single pass (SYCLFFT_B200_FUSED4_SINGLE=1)
    monkeypatch.setenv("SYCLFFT_B200_FUSED4_SINGLE", "1")
    for fused in ("1", "0"):  # opt-in fused launches, then the default separate passes
        monkeypatch.setenv("SYCLFFT_B200_FUSED4", fused)
        p = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction.forward)
        desc = p.describe()
        assert bool(desc.get("fused_fourstep") or desc.get("fused_bluestein")) == (fused == "1"), desc
        for d, nm in ((-1, 0), (1, 2), (-1, 3)):
            out = torch.empty_like(xi)
            rc = p._lib.syclfft_b200_execute_ex(p._handle, xi.data_ptr(), out.data_ptr(), 0, d, nm,
                                                torch.cuda.current_stream().cuda_stream, p._err, 1024)
            assert rc == 0, p._err.value
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert rel_l2(got, fp64_fft(x, shape, batch, d, norm_scale(nm, d, n))) <= spec_tol(n, dbl), (fused, d, nm)
            outs[(fused, d, nm)] = got
    for d, nm in ((-1, 0), (1, 2), (-1, 3)):
        assert rel_l2(outs[("1", d, nm)], outs[("0", d, nm)]) <= spec_tol(n, dbl)


@pytest.mark.parametrize("shape,batch,dbl", [([257], 64, False), ([641], 9, True), ([12289], 8, False),
                                             ([12289], 5, True), ([65537], 6, False), ([65537], 5, True),
                                             ([5, 257], 3, False)],
                         ids=lambda v: str(v))
def test_rader_lengths(sf, torch, monkeypatch, shape, batch, dbl):
    """Prime lengths whose L - 1 the catalog covers run Rader's algorithm (gather by generator
    powers, length-(L-1) convolution with the x[0] term, scatter): against FP64 and against
    the same plan on Bluestein's convolution (SYCLFFT_B200_RADER=0), in both directions and
    with every normalization through execute_ex's overrides, in place, and on a sub-batch."""
    import ctypes
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 17 + n, dt)
    xi = torch.from_numpy(x).cuda()
    outs = {}
    for rader in ("1", "0"):
        monkeypatch.setenv("SYCLFFT_B200_RADER", rader)
        p = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction.forward)
        kinds = [q["kind"] for q in p.describe()["passes"]]
        assert any(k.startswith("rader") for k in kinds) == (rader == "1"), kinds
        for d, nm in ((-1, 0), (1, 2), (-1, 3), (1, 1)):
            out = torch.empty_like(xi)
            rc = p._lib.syclfft_b200_execute_ex(p._handle, xi.data_ptr(), out.data_ptr(), 0, d, nm,
                                                torch.cuda.current_stream().cuda_stream, p._err, 1024)
            assert rc == 0, p._err.value
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert rel_l2(got, fp64_fft(x, shape, batch, d, norm_scale(nm, d, n))) <= spec_tol(n, dbl), (rader, d, nm)
            outs[(rader, d, nm)] = got
    for d, nm in ((-1, 0), (1, 2), (-1, 3), (1, 1)):
        assert rel_l2(outs[("1", d, nm)], outs[("0", d, nm)]) <= 2 * spec_tol(n, dbl)
    monkeypatch.delenv("SYCLFFT_B200_RADER")
    # in place, backward plan, orthogonal normalization
    got, p = run(sf, torch, x, shape, batch, sf.direction.backward, norm=3, dbl=dbl, in_place=True)
    assert any(q["kind"].startswith("rader") for q in p.describe()["passes"])
    assert rel_l2(got, fp64_fft(x, shape, batch, 1, norm_scale(3, 1, n))) <= spec_tol(n, dbl)
    # the first b lines of a plan made for the whole batch
    p = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction.forward)
    b = max(1, batch // 2)
    out = torch.zeros_like(xi)
    rc = p._lib.syclfft_b200_execute_ex(p._handle, xi.data_ptr(), out.data_ptr(), b, -1, 1,
                                        torch.cuda.current_stream().cuda_stream, p._err, 1024)
    assert rc == 0, p._err.value
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert rel_l2(got[:n * b], fp64_fft(x[:n * b], shape, b, -1, norm_scale(1, -1, n))) <= spec_tol(n, dbl)
    assert not np.any(got[n * b:])  # lines past the sub-batch untouched
