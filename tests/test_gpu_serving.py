"""Serving-path features on the GPU: grouped launches (many requests of a length family in
one launch), plans that run a smaller batch than planned, device-generated Bluestein
tables, and the continuous-batching loop, whose results must be the same for a request
served alone and in the mix."""
import ctypes
import math

import numpy as np
import pytest

from conftest import fp64_fft, norm_scale, rel_l2, uniform_complex

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def spec_tol(n, dbl):
    return (1e-12 if dbl else 1e-5) * max(1.0, math.log2(max(n, 2)))


def test_grouped_launch_matches_fp64(torch):
    from syclfft_b200 import _provider
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    rng = np.random.default_rng(3)
    for n, dbl in ((4096, False), (256, True), (13440, False), (64, False)):
        assert lib.syclfft_b200_group_supports(2 if dbl else 1, n) == 1
        g = lib.syclfft_b200_group_create(2 if dbl else 1, n, -1, err, 1024)
        assert g, err.value
        dt = np.complex128 if dbl else np.complex64
        reqs = []
        for i in range(7):
            b = int(rng.integers(1, 40))
            d = int(rng.choice([-1, 1]))
            nm = int(rng.integers(0, 4))
            x = uniform_complex(n * b, 100 * i + n, dt)
            xi = torch.from_numpy(x).cuda()
            xo = xi if i % 3 == 0 else torch.empty_like(xi)  # some in place
            reqs.append((x, xi, xo, b, d, nm))
        items = (_provider.GroupItemV1 * len(reqs))()
        for k, (x, xi, xo, b, d, nm) in enumerate(reqs):
            items[k].in_, items[k].out, items[k].batch = xi.data_ptr(), xo.data_ptr(), b
            items[k].direction, items[k].normalization = d, nm
        rc = lib.syclfft_b200_group_execute(g, items, len(reqs), torch.cuda.current_stream().cuda_stream, err, 1024)
        assert rc == 0, err.value
        torch.cuda.synchronize()
        for x, xi, xo, b, d, nm in reqs:
            ref = fp64_fft(x, [n], b, d, norm_scale(nm, d, n))
            assert rel_l2(xo.cpu().numpy(), ref) <= spec_tol(n, dbl)
        lib.syclfft_b200_group_destroy(g)
    assert lib.syclfft_b200_group_supports(1, 1009) == 0


def test_family_launch_matches_fp64(torch):
    """Requests of every length of a radix family (powers of two up to 4096 float / 2048
    double), with their own batches, directions and normalizations, some in place, in one
    launch; again from a captured CUDA graph with new inputs."""
    from syclfft_b200 import _provider
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    rng = np.random.default_rng(8)
    for dbl, top in ((False, 4096), (True, 2048)):
        sc = 2 if dbl else 1
        assert lib.syclfft_b200_family_supports(sc, 64) and lib.syclfft_b200_family_supports(sc, top)
        assert not lib.syclfft_b200_family_supports(sc, 2 * top) and not lib.syclfft_b200_family_supports(sc, 96)
        fam = lib.syclfft_b200_family_create(sc, -1, err, 1024)
        assert fam, err.value
        dt = np.complex128 if dbl else np.complex64
        reqs = []
        n = 64
        while n <= top:
            for _ in range(2):
                b = int(rng.integers(1, 70))
                d = int(rng.choice([-1, 1]))
                nm = int(rng.integers(0, 4))
                xi = torch.from_numpy(uniform_complex(n * b, n + b, dt)).cuda()
                xo = xi if len(reqs) % 3 == 0 else torch.empty_like(xi)
                reqs.append((n, xi, xo, b, d, nm))
            n *= 2
        items = (_provider.FamilyItemV1 * len(reqs))()
        for k, (n, xi, xo, b, d, nm) in enumerate(reqs):
            items[k].in_, items[k].out, items[k].n, items[k].batch = xi.data_ptr(), xo.data_ptr(), n, b
            items[k].direction, items[k].normalization = d, nm
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        inputs = [xi.clone() for _, xi, _, _, _, _ in reqs]
        assert lib.syclfft_b200_family_execute(fam, items, len(reqs), s.cuda_stream, err, 1024) == 0, err.value
        torch.cuda.synchronize()
        for (n, xi, xo, b, d, nm), x in zip(reqs, inputs):
            ref = fp64_fft(x.cpu().numpy(), [n], b, d, norm_scale(nm, d, n))
            assert rel_l2(xo.cpu().numpy(), ref) <= spec_tol(n, dbl), (n, b, d, nm)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s):
            assert lib.syclfft_b200_family_execute(fam, items, len(reqs), s.cuda_stream, err, 1024) == 0
        fresh = [x.clone().normal_() for x in inputs]
        for (n, xi, xo, b, d, nm), x in zip(reqs, fresh):
            xi.copy_(x)
        graph.replay()
        torch.cuda.synchronize()
        for (n, xi, xo, b, d, nm), x in zip(reqs, fresh):
            ref = fp64_fft(x.cpu().numpy(), [n], b, d, norm_scale(nm, d, n))
            assert rel_l2(xo.cpu().numpy(), ref) <= spec_tol(n, dbl), (n, b, d, nm)
        del graph
        lib.syclfft_b200_family_destroy(fam)


@pytest.mark.parametrize("shape,dbl", [([4096], False), ([65536], True), ([65537], False), ([1009], True),
                                       ([13440], False), ([24, 40], False), ([30000], True)], ids=str)
def test_execute_smaller_batch(torch, shape, dbl):
    """A plan for up to 8 transforms runs the first 3 (same tables and scratch)."""
    from syclfft_b200 import _provider
    api = _provider.provider()
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    cfg = _provider.make_config(shape, 8, 1, double=dbl, normalization=2)
    h = api.create(ctypes.byref(cfg), err, 1024)
    assert h, err.value
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(3 * n, 7 + n, dt)
    xi = torch.from_numpy(x).cuda()
    out = torch.zeros(8 * n, dtype=xi.dtype, device="cuda")
    rc = lib.syclfft_b200_execute_batch(h, xi.data_ptr(), out.data_ptr(), 3, torch.cuda.current_stream().cuda_stream,
                                        err, 1024)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert rel_l2(got[: 3 * n], fp64_fft(x, shape, 3, 1, 1.0 / n)) <= spec_tol(n, dbl)
    assert not np.any(got[3 * n:])  # nothing written past the requested batch
    assert lib.syclfft_b200_execute_batch(h, xi.data_ptr(), out.data_ptr(), 9, None, err, 1024) != 0
    api.destroy(h)


def test_device_bluestein_tables_accuracy(torch):
    """Chirp spectra made on the device (FP64 FFT) keep Bluestein at FP64 accuracy."""
    import syclfft_b200 as sf
    for n in (257, 4099, 30011, 65537):
        x = uniform_complex(2 * n, n, np.complex128)
        p = sf.plan_many_dft("double", [n], 2, sf.direction.forward)
        xt = torch.from_numpy(x).cuda()
        out = torch.empty_like(xt)
        p.execute(xt, out).synchronize()
        assert rel_l2(out.cpu().numpy(), fp64_fft(x, [n], 2, -1)) <= spec_tol(n, True)


def test_serving_alone_vs_mix(torch):
    """Each request's result is the same served alone (plain, one at a time) and in the mix
    (continuous batching, grouped launches, several streams)."""
    from syclfft_b200 import serving
    reqs = serving.make_request_stream(count=160, rate=20000.0, seed=11, max_batch=16)
    reqs = [r for r in reqs if r.lengths[0] <= 1 << 16]
    srv = serving.Server(budget_bytes=2e9, streams=3)
    try:
        mixed = srv.run(reqs, mode="served", keep_results=True)
        results = {r.rid: r.result for r in reqs}
        alone = srv.run(reqs, mode="plain", keep_results=True)
        for r in reqs:
            a, b = results[r.rid].numpy(), r.result.numpy()
            assert rel_l2(a, b) <= spec_tol(r.lengths[0], r.double), r
        # and against FP64 for a few
        for r in reqs[:12]:
            x = serving.synthetic_input(r).cpu().numpy()
            n = r.lengths[0]
            ref = fp64_fft(x, [n], r.batch, r.direction, norm_scale(r.normalization, r.direction, n))
            assert rel_l2(results[r.rid].numpy(), ref) <= spec_tol(n, r.double)
        for st in (mixed, alone):
            assert st["requests"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0
        assert mixed["groups"] + mixed["families"] >= 1
    finally:
        srv.close()


def test_serving_alone_vs_mix_full_stream_shape(torch):
    """The serving configuration's request mix at its real shape: lengths up to 2^20 (powers of
    two, 7-smooth, primes up to 65537), batches up to 512, 20% complex<double>, random
    direction and normalization, Poisson arrivals at 50k/s; an admission budget small enough
    that requests wait for memory, and a plan budget small enough that resident plans are
    evicted. Every result must be the same served alone and in the mix: the L2 norm of each
    output and 2048 sampled elements (fixed positions per request) within the float/double
    tolerance, and a handful of outputs against an FP64 FFT in full. (Plans are evicted by their
    real device bytes; an 8 MB plan budget keeps only a few dozen resident.)"""
    from syclfft_b200 import serving
    reqs = serving.make_request_stream(count=600, rate=50000.0, seed=23)
    assert max(r.lengths[0] for r in reqs) > 1 << 17 and max(r.batch for r in reqs) > 256
    assert any(r.double for r in reqs) and any(r.lengths[0] > 60000 and not serving._smooth7(r.lengths[0])
                                               for r in reqs)
    largest = max(2 * r.elements * (16 if r.double else 8) for r in reqs)
    full = {r.rid for r in sorted(reqs, key=lambda r: r.elements)[::60]}  # ten, small to large

    def keep(r):
        out = r.out.view(-1)
        g = torch.Generator(device=out.device).manual_seed(r.rid)
        idx = torch.randint(0, out.numel(), (2048,), device=out.device, generator=g)
        norm = float(torch.linalg.vector_norm(out.to(torch.complex128)))
        return norm, out[idx].cpu(), (out.cpu() if r.rid in full else None)

    srv = serving.Server(budget_bytes=max(1.05 * largest, 6e9), streams=4, plan_budget_bytes=8e6)
    try:
        mixed = srv.run(reqs, mode="served", keep_results=keep)
        results = {r.rid: r.result for r in reqs}
        alone = srv.run(reqs, mode="plain", keep_results=keep)
    finally:
        srv.close()
    assert mixed["max_waiting"] > 0, mixed      # admission had to wait for memory
    assert mixed["plan_evictions"] > 0, mixed   # resident plans were evicted
    for r in reqs:
        n = r.lengths[0]
        tol = spec_tol(n, r.double)
        (na, sa, fa), (nb, sb, fb) = results[r.rid], r.result
        assert abs(na - nb) <= tol * max(nb, 1e-30), (r, na, nb)
        assert rel_l2(sa.numpy(), sb.numpy()) <= tol, r
    for r in reqs:
        if r.rid not in full:
            continue
        x = serving.synthetic_input(r).cpu().numpy()
        n = r.lengths[0]
        ref = fp64_fft(x, [n], r.batch, r.direction, norm_scale(r.normalization, r.direction, n))
        assert rel_l2(results[r.rid][2].numpy(), ref) <= spec_tol(n, r.double), r
    for st in (mixed, alone):
        assert st["requests"] == len(reqs) and st["p99_ms"] >= st["p50_ms"] > 0


def test_cuda_graph_capture_and_replay(torch):
    """Plan executes and grouped launches are capturable in a CUDA graph; replays with new
    input data give the same results as direct execution."""
    import syclfft_b200 as sf
    from syclfft_b200 import _provider
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    opts = sf.plan_options(placement=sf.placement.in_place, normalization=sf.normalization.orthogonal)
    plans = [sf.plan_many_dft("float", [4096], 64, sf.direction.forward, opts),
             sf.plan_many_dft("double", [65536], 4, sf.direction.backward, opts),
             sf.plan_many_dft("float", [1009], 16, sf.direction.forward, opts)]
    bufs = [torch.randn(4096 * 64, dtype=torch.complex64, device="cuda"),
            torch.randn(65536 * 4, dtype=torch.complex128, device="cuda"),
            torch.randn(1009 * 16, dtype=torch.complex64, device="cuda")]
    g = lib.syclfft_b200_group_create(1, 256, -1, err, 1024)
    ga = torch.randn(256 * 8, dtype=torch.complex64, device="cuda")
    gb = torch.randn(256 * 3, dtype=torch.complex64, device="cuda")
    items = (_provider.GroupItemV1 * 2)()
    items[0].in_, items[0].out, items[0].batch, items[0].direction, items[0].normalization = ga.data_ptr(), ga.data_ptr(), 8, -1, 0
    items[1].in_, items[1].out, items[1].batch, items[1].direction, items[1].normalization = gb.data_ptr(), gb.data_ptr(), 3, 1, 2
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())

    def step():
        for p, b in zip(plans, bufs):
            p.execute(b, stream=s)
        assert lib.syclfft_b200_group_execute(g, items, 2, s.cuda_stream, err, 1024) == 0, err.value

    with torch.cuda.stream(s):
        step()  # warm-up outside capture (kernel attributes, tables)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=s):
        step()
    for trial in range(2):
        inputs = [b.clone().normal_() for b in bufs] + [ga.clone().normal_(), gb.clone().normal_()]
        for dst, src in zip(bufs + [ga, gb], inputs):
            dst.copy_(src)
        graph.replay()
        torch.cuda.synchronize()
        for (p, b, x) in zip(plans, bufs, inputs):
            n = int(np.prod(p.shape()))
            d = int(p.direction())
            ref = fp64_fft(x.cpu().numpy(), p.shape(), p.batch_count(), d, 1 / math.sqrt(n))
            assert rel_l2(b.cpu().numpy(), ref) <= spec_tol(n, b.dtype == torch.complex128)
        assert rel_l2(ga.cpu().numpy(), fp64_fft(inputs[3].cpu().numpy(), [256], 8, -1)) <= spec_tol(256, False)
        assert rel_l2(gb.cpu().numpy(), fp64_fft(inputs[4].cpu().numpy(), [256], 3, 1, 1 / 256)) <= spec_tol(256, False)
    del graph
    lib.syclfft_b200_group_destroy(g)


@pytest.mark.parametrize("shape,dbl", [([4096], False), ([13440], False), ([65536], True), ([1009], False),
                                       ([1009], True), ([4099], True), ([65537], False), ([30011], True),
                                       ([24, 1009], False), ([60, 40], True)], ids=str)
def test_execute_ex_direction_override(torch, shape, dbl):
    """A forward plan run as a backward transform (and the reverse) through execute_ex, with
    every normalization: Bluestein plans conjugate outside their chirp products."""
    from syclfft_b200 import _provider
    lib = _provider.load()
    api = _provider.provider(lib)
    err = ctypes.create_string_buffer(1024)
    n = int(np.prod(shape))
    batch = 3
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 5 + n, dt)
    xi = torch.from_numpy(x).cuda()
    s = torch.cuda.current_stream().cuda_stream
    for plan_dir in (-1, 1):
        cfg = _provider.make_config(shape, batch, plan_dir, double=dbl, normalization=0)
        h = api.create(ctypes.byref(cfg), err, 1024)
        assert h, err.value
        for d, nm in ((-plan_dir, 0), (-plan_dir, 3), (plan_dir, 1)):
            out = torch.empty_like(xi)
            assert lib.syclfft_b200_execute_ex(h, xi.data_ptr(), out.data_ptr(), batch, d, nm, s, err, 1024) == 0, \
                err.value
            torch.cuda.synchronize()
            ref = fp64_fft(x, shape, batch, d, norm_scale(nm, d, n))
            assert rel_l2(out.cpu().numpy(), ref) <= spec_tol(n, dbl), (plan_dir, d, nm)
        api.destroy(h)


def test_serving_helpers_fill_and_execute_many(torch):
    """syclfft_b200_fill_uniform: value i depends on (seed, i) only -- the same whether a buffer
    is filled alone or among 300 others (two launches of up to 256 items), in [-1, 1), mean
    about 0; syclfft_b200_execute_many gives what one execute_ex per item gives."""
    from syclfft_b200 import _provider, serving
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    reqs = [serving.Request(i, (int(n),), 3, bool(i % 3 == 0), -1, 0, 1000 + i, 0.0)
            for i, n in enumerate(np.random.default_rng(2).choice([64, 100, 1024, 3000, 65536], 300))]
    bufs = [torch.empty(2 * r.elements, dtype=torch.float64 if r.double else torch.float32, device="cuda")
            for r in reqs]
    for r, b in zip(reqs, bufs):
        r.in_ptr = b.data_ptr()
    serving.fill_inputs(reqs, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    for r, b in list(zip(reqs, bufs))[::37]:
        alone = serving.synthetic_input(r).view(torch.float64 if r.double else torch.float32)
        torch.cuda.synchronize()
        assert torch.equal(alone, b)
        assert float(b.min()) >= -1.0 and float(b.max()) < 1.0
    allv = torch.cat([b.double() for b in bufs])
    assert abs(float(allv.mean())) < 5e-3 and abs(float(allv.var()) - 1 / 3) < 5e-3
    # execute_many vs execute_ex, mixed plans, directions and normalizations
    plans = {}
    items = (_provider.ExecItemV1 * 12)()
    outs_many, outs_one = [], []
    for i, r in enumerate(reqs[:12]):
        key = (r.lengths[0], r.double)
        if key not in plans:
            cfg = _provider.make_config([r.lengths[0]], 8, -1, r.double, False, 0, False, 0)
            plans[key] = lib.syclfft_b200_create_ex(ctypes.byref(cfg), 0, err, 1024)
            assert plans[key], err.value
        o1, o2 = torch.empty_like(bufs[i]), torch.empty_like(bufs[i])
        outs_many.append(o1)
        outs_one.append(o2)
        d, nm = (-1, 1) if i % 2 else (1, 3)
        items[i].plan, items[i].in_, items[i].out = plans[key], bufs[i].data_ptr(), o1.data_ptr()
        items[i].batch, items[i].direction, items[i].normalization = r.batch, d, nm
        assert lib.syclfft_b200_execute_ex(plans[key], bufs[i].data_ptr(), o2.data_ptr(), r.batch, d, nm,
                                           torch.cuda.current_stream().cuda_stream, err, 1024) == 0, err.value
    assert lib.syclfft_b200_execute_many(items, 12, torch.cuda.current_stream().cuda_stream, err, 1024) == 0, err.value
    torch.cuda.synchronize()
    for a, b in zip(outs_many, outs_one):
        assert torch.equal(a, b)
    items[3].direction = 5
    assert lib.syclfft_b200_execute_many(items, 12, torch.cuda.current_stream().cuda_stream, err, 1024) != 0
    assert b"execute item 3" in err.value and b"direction" in err.value
    torch.cuda.synchronize()
    for h in plans.values():
        _provider.provider(lib).destroy(h)


def test_release_stream_scratch_and_execute_again(torch):
    """A stream-scratch plan's arena released between executes (as Server.close does before its
    streams go) is allocated again by the next execute on that stream: same results."""
    from syclfft_b200 import _provider
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    cfg = _provider.make_config([65536], 8, -1, False, False, 0, False, 0)
    h = lib.syclfft_b200_create_ex(ctypes.byref(cfg), _provider.CREATE_STREAM_SCRATCH, err, 1024)
    assert h, err.value
    s = torch.cuda.Stream()
    x = torch.randn(65536 * 8, dtype=torch.complex64, device="cuda")
    outs = []
    for _ in range(2):
        y = torch.empty_like(x)
        assert lib.syclfft_b200_execute_ex(h, x.data_ptr(), y.data_ptr(), 0, -1, 0, s.cuda_stream, err, 1024) == 0, err.value
        lib.syclfft_b200_release_stream_scratch(s.cuda_stream, torch.cuda.current_device())
        outs.append(y)
    lib.syclfft_b200_release_stream_scratch(s.cuda_stream, torch.cuda.current_device())  # nothing held: no-op
    torch.cuda.synchronize()
    assert torch.equal(outs[0], outs[1])
    ref = torch.fft.fft(x.view(8, 65536).to(torch.complex128), dim=1).reshape(-1)
    assert float((outs[0] - ref).abs().norm() / ref.abs().norm()) < 1e-5 * 16
    _provider.provider(lib).destroy(h)
