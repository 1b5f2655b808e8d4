"""GPU parity of the real transforms (syclfft_b200_create_real): R2C against numpy.fft.rfft
and C2R against numpy.fft.irfft in FP64, with the complex tolerance of the same length
(rel-L2 <= 1e-5 * log2(N) float, 1e-12 * log2(N) double); normalizations, round trips,
partial batches, capture into a CUDA graph and the split-precision inner plan."""
import math

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


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


def tol(n, dbl):
    return (1e-12 if dbl else 1e-5) * max(1.0, math.log2(max(n, 2)))


def scale_of(norm, direction, n):
    if norm == 3:
        return 1 / math.sqrt(n)
    if (norm == 1 and direction == -1) or (norm == 2 and direction == 1):
        return 1 / n
    return 1.0


def real_lines(n, batch, seed, dbl):
    rng = np.random.default_rng(seed)
    return rng.uniform(-1, 1, (batch, n)).astype(np.float64 if dbl else np.float32)


def spectra(n, batch, seed, dbl):
    rng = np.random.default_rng(seed)
    s = rng.uniform(-1, 1, (batch, n // 2 + 1)) + 1j * rng.uniform(-1, 1, (batch, n // 2 + 1))
    return s.astype(np.complex128 if dbl else np.complex64)


SIZES = [2, 8, 30, 256, 512, 1000, 2018, 2048, 4096, 8192, 13440, 26880, 131072]


@pytest.mark.parametrize("dbl", [False, True])
@pytest.mark.parametrize("n", SIZES)
def test_r2c_matches_rfft(torch, sf, n, dbl):
    batch = 3
    x = real_lines(n, batch, n, dbl)
    p = sf.plan_dft_r2c_1d("double" if dbl else "float", n, batch)
    d = p.describe()
    assert d["real"] == "r2c" and d["n"] == n
    xt = torch.from_numpy(x).cuda()
    out = torch.empty(batch * (n // 2 + 1), dtype=p.dtype, device="cuda")
    p.execute(xt, out).synchronize()
    ref = np.fft.rfft(x.astype(np.float64), axis=1).reshape(-1)
    assert rel_l2(out.cpu().numpy(), ref) <= tol(n, dbl)


@pytest.mark.parametrize("dbl", [False, True])
@pytest.mark.parametrize("n", SIZES)
def test_c2r_matches_irfft(torch, sf, n, dbl):
    batch = 3
    s = spectra(n, batch, n + 7, dbl)
    p = sf.plan_dft_c2r_1d("double" if dbl else "float", n, batch)
    st = torch.from_numpy(s).cuda()
    out = torch.empty(batch * n, dtype=p.real_dtype, device="cuda")
    p.execute(st, out).synchronize()
    ref = (np.fft.irfft(s.astype(np.complex128), n, axis=1) * n).reshape(-1)
    # the spectrum's energy is spread over n outputs: compare relative to the reference
    assert rel_l2(out.cpu().numpy(), ref) <= tol(n, dbl)


@pytest.mark.parametrize("norm", [0, 1, 2, 3])
def test_normalizations(torch, sf, norm):
    n, batch = 4096, 2
    opts = sf.plan_options(normalization=sf.normalization(norm))
    x = real_lines(n, batch, 11, True)
    f = sf.plan_dft_r2c_1d("double", n, batch, opts)
    b = sf.plan_dft_c2r_1d("double", n, batch, opts)
    xt = torch.from_numpy(x).cuda()
    spec = torch.empty(batch * (n // 2 + 1), dtype=torch.complex128, device="cuda")
    back = torch.empty(batch * n, dtype=torch.float64, device="cuda")
    f.execute(xt, spec).synchronize()
    ref = np.fft.rfft(x, axis=1).reshape(-1) * scale_of(norm, -1, n)
    assert rel_l2(spec.cpu().numpy(), ref) <= tol(n, True)
    b.execute(spec, back).synchronize()
    want = x.reshape(-1) * n * scale_of(norm, -1, n) * scale_of(norm, 1, n)
    assert rel_l2(back.cpu().numpy(), want) <= tol(n, True)


@pytest.mark.parametrize("n", [1024, 13440, 65536])
def test_round_trip_float(torch, sf, n):
    batch = 16
    opts = sf.plan_options(normalization=sf.normalization.backward)
    x = real_lines(n, batch, 5, False)
    f = sf.plan_dft_r2c_1d("float", n, batch, opts)
    b = sf.plan_dft_c2r_1d("float", n, batch, opts)
    xt = torch.from_numpy(x).cuda()
    spec = torch.empty(batch * (n // 2 + 1), dtype=torch.complex64, device="cuda")
    back = torch.empty(batch * n, dtype=torch.float32, device="cuda")
    f.execute(xt, spec)
    b.execute(spec, back).synchronize()
    assert rel_l2(back.cpu().numpy(), x.reshape(-1)) <= 2 * tol(n, False)


def test_partial_batch_leaves_other_lines(torch, sf):
    import ctypes
    from syclfft_b200 import _provider
    n, batch, run = 512, 8, 3
    p = sf.plan_dft_r2c_1d("float", n, batch)
    x = real_lines(n, batch, 3, False)
    xt = torch.from_numpy(x).cuda()
    out = torch.full((batch * (n // 2 + 1),), 7 + 7j, dtype=torch.complex64, device="cuda")
    err = ctypes.create_string_buffer(_provider.ERR_CAP)
    s = torch.cuda.current_stream()
    rc = p._lib.syclfft_b200_execute_batch(p._handle, xt.data_ptr(), out.data_ptr(), run, s.cuda_stream, err,
                                           _provider.ERR_CAP)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(batch, -1)
    ref = np.fft.rfft(x[:run].astype(np.float64), axis=1)
    assert rel_l2(got[:run], ref) <= tol(n, False)
    assert np.all(got[run:] == np.complex64(7 + 7j))


def test_errors(torch, sf):
    p = sf.plan_dft_r2c_1d("float", 64, 2)
    x = torch.zeros(128, dtype=torch.float32, device="cuda")
    with pytest.raises(sf.SyclfftError) as e:
        p.execute(x, torch.zeros(66, dtype=torch.complex128, device="cuda"))
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        p.execute(x, torch.zeros(10, dtype=torch.complex64, device="cuda"))
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        p.execute(x)
    assert e.value.code == sf.error_code.invalid_argument
    with pytest.raises(sf.SyclfftError) as e:
        sf.plan_dft_c2r_1d("float", 64, 1, sf.plan_options(placement=sf.placement.in_place))
    assert e.value.code == sf.error_code.invalid_argument


def test_graph_capture_replays_the_transform(torch, sf):
    n, batch = 13440, 4
    p = sf.plan_dft_r2c_1d("float", n, batch)
    x = real_lines(n, batch, 9, False)
    xt = torch.from_numpy(x).cuda()
    out = torch.empty(batch * (n // 2 + 1), dtype=torch.complex64, device="cuda")
    p.execute(xt, out).synchronize()
    eager = out.clone()
    out.zero_()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            p.execute(xt, out, stream=s)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out, eager)


def test_split_precision_inner_plan(torch, sf):
    n, batch = 512, 64
    opts = sf.plan_options(split_precision=True)
    p = sf.plan_dft_r2c_1d("float", n, batch, opts)
    passes = p.describe()["inner"]["passes"]
    assert any(q.get("tc_id", -1) >= 0 for q in passes)
    x = real_lines(n, batch, 17, False)
    xt = torch.from_numpy(x).cuda()
    out = torch.empty(batch * (n // 2 + 1), dtype=torch.complex64, device="cuda")
    p.execute(xt, out).synchronize()
    ref = np.fft.rfft(x.astype(np.float64), axis=1).reshape(-1)
    assert rel_l2(out.cpu().numpy(), ref) <= tol(n, False)


# half lengths with a fused one-pass kernel: 256..4096 (float), 256..2048 (double)
FUSED = [(512, False), (2048, False), (8192, False), (512, True), (4096, True)]


@pytest.mark.parametrize("n,dbl", FUSED)
def test_fused_matches_two_pass(torch, sf, n, dbl, monkeypatch):
    """The one-pass real kernels (pre-/post-process inside the size-specialised FFT) against the
    two-pass form (complex FFT of length n/2, then the separate pass) and FP64, both kinds,
    with a normalization and a partial batch of lines."""
    batch = 37
    scalar = "double" if dbl else "float"
    opts = sf.plan_options(normalization=sf.normalization.orthogonal)
    x = real_lines(n, batch, 3 + n, dbl)
    s = spectra(n, batch, 5 + n, dbl)
    outs = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("SYCLFFT_B200_REAL_FUSED", mode)
        f = sf.plan_dft_r2c_1d(scalar, n, batch, opts)
        b = sf.plan_dft_c2r_1d(scalar, n, batch, opts)
        assert f.describe()["fused"] == int(mode) and b.describe()["fused"] == int(mode)
        if mode == "1":
            assert f.launches() == 1 and b.launches() == 1
        spec = torch.empty(batch * (n // 2 + 1), dtype=f.dtype, device="cuda")
        back = torch.empty(batch * n, dtype=b.real_dtype, device="cuda")
        f.execute(torch.from_numpy(x).cuda(), spec)
        b.execute(torch.from_numpy(s).cuda(), back).synchronize()
        outs[mode] = (spec.cpu().numpy(), back.cpu().numpy())
    scale = 1 / math.sqrt(n)
    ref_f = np.fft.rfft(x.astype(np.float64), axis=1).reshape(-1) * scale
    ref_b = (np.fft.irfft(s.astype(np.complex128), n, axis=1) * n).reshape(-1) * scale
    for mode in ("1", "0"):
        assert rel_l2(outs[mode][0], ref_f) <= tol(n, dbl)
        assert rel_l2(outs[mode][1], ref_b) <= tol(n, dbl)
    assert rel_l2(outs["1"][0], outs["0"][0]) <= tol(n, dbl)


def test_misaligned_real_buffers_are_rejected(torch, sf):
    n, batch = 1024, 2
    p = sf.plan_dft_r2c_1d("float", n, batch)
    x = torch.zeros(n * batch + 1, dtype=torch.float32, device="cuda")
    out = torch.zeros(batch * (n // 2 + 1), dtype=torch.complex64, device="cuda")
    with pytest.raises(sf.SyclfftError) as e:
        p.execute(x.data_ptr() + 4, out)   # a real array starting at an odd float
    assert e.value.code == sf.error_code.execution_failed
    assert "aligned" in str(e.value)


MULTI = [([8, 64], 3, False, 0), ([16, 12, 10], 2, True, 3), ([32, 8192], 2, False, 1),
         ([64, 512], 4, True, 2), ([5, 6, 4], 1, False, 0), ([30, 1000], 3, False, 3)]


@pytest.mark.parametrize("shape,batch,dbl,norm", MULTI, ids=str)
def test_multidimensional_real_transforms(torch, sf, shape, batch, dbl, norm):
    """rfftn / irfftn over 2D and 3D shapes (last axis fused or two-pass, outer axes on the
    strided complex kernels) against numpy in FP64, then the C2R of the R2C result."""
    total = math.prod(shape)
    axes = tuple(range(1, len(shape) + 1))
    spec_shape = shape[:-1] + [shape[-1] // 2 + 1]
    scalar = "double" if dbl else "float"
    opts = sf.plan_options(normalization=sf.normalization(norm))
    f = sf.plan_dft_r2c(scalar, shape, batch, opts)
    b = sf.plan_dft_c2r(scalar, shape, batch, opts)
    d = f.describe()
    assert d["shape"] == shape and "outer" in d
    rng = np.random.default_rng(total + batch)
    x = rng.uniform(-1, 1, [batch] + shape).astype(np.float64 if dbl else np.float32)
    xt = torch.from_numpy(x).cuda()
    spec = torch.empty(batch * math.prod(spec_shape), dtype=f.dtype, device="cuda")
    back = torch.empty_like(xt)
    b.execute(spec, back, dependencies=[f.execute(xt, spec)]).synchronize()
    sf_ = scale_of(norm, -1, total)
    sb_ = scale_of(norm, 1, total)
    ref = np.fft.rfftn(x.astype(np.float64), axes=axes) * sf_
    tol_ = (1e-12 if dbl else 1e-5) * max(1.0, math.log2(total))
    assert rel_l2(spec.cpu().numpy(), ref.reshape(-1)) <= tol_
    want = x.astype(np.float64) * total * sf_ * sb_
    assert rel_l2(back.cpu().numpy(), want.reshape(-1)) <= 2 * tol_
    # C2R of an arbitrary spectrum (imaginary parts at bins 0 and n/2 ignored) against irfftn
    s = (rng.uniform(-1, 1, [batch] + spec_shape) + 1j * rng.uniform(-1, 1, [batch] + spec_shape))
    s = s.astype(np.complex128 if dbl else np.complex64)
    out = torch.empty_like(xt)
    b.execute(torch.from_numpy(s).cuda(), out).synchronize()
    ref_b = np.fft.irfftn(s.astype(np.complex128), s=shape, axes=axes) * total * sb_
    assert rel_l2(out.cpu().numpy(), ref_b.reshape(-1)) <= tol_
