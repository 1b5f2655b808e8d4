"""Split-precision tensor-core path (complex<float>, SYCLFFT_B200_CREATE_SPLIT_BF16 /
plan_options.split_precision): BF16 hi/lo radix-16 matrix products with FP32 accumulation.

Every case reports its relative L2 and max error against an FP64 FFT beside the error of
the pure-FP32 path on the same input, and holds the tensor-core result to the float
tolerance (1e-5 relative L2 scaled by log2 N) and to 2e-5 unscaled.
"""
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


def max_err(a, ref):
    return float(np.abs(a - ref).max() / np.abs(ref).max())


def run(torch, shape, batch, d, x, split, norm=0, in_place=False):
    import syclfft_b200 as sf
    opts = sf.plan_options(placement=sf.placement.in_place if in_place else sf.placement.out_of_place,
                           normalization=sf.normalization(norm), split_precision=split)
    p = sf.plan_many_dft("float", shape, batch, sf.direction(d), opts)
    xi = torch.from_numpy(x).cuda()
    if in_place:
        p.execute(xi).synchronize()
        out = xi
    else:
        out = torch.empty_like(xi)
        p.execute(xi, out).synchronize()
    desc = p.describe()
    return out.cpu().numpy(), desc


def tc_passes(desc):
    return [ps for ps in desc["passes"] if ps.get("tc_id", -1) >= 0]


CASES = [
    ([256], 4096, -1, 0, False),
    ([256], 3000, 1, 3, True),       # ragged last tile (3000 lines, 16 per CTA)
    ([4096], 256, -1, 1, False),
    ([4096], 129, 1, 3, True),
    ([256, 256], 4, -1, 0, False),   # contiguous axis, then a strided axis (adjacent columns)
    ([16, 256], 8, 1, 2, False),     # only the last axis has a tensor-core kernel
    ([256, 48], 8, -1, 0, True),     # strided 256-point axis with 48 columns (3 column tiles)
]


@pytest.mark.parametrize("shape,batch,d,norm,in_place", CASES, ids=str)
def test_split_precision_vs_fp64(torch, shape, batch, d, norm, in_place):
    n = int(np.prod(shape))
    x = uniform_complex(n * batch, 11 + n + batch, np.complex64)
    got, desc = run(torch, shape, batch, d, x.copy(), True, norm, in_place)
    assert tc_passes(desc), desc
    fp32, desc32 = run(torch, shape, batch, d, x.copy(), False, norm, in_place)
    assert not tc_passes(desc32)
    ref = fp64_fft(x, shape, batch, d, norm_scale(norm, d, n))
    e_tc, e_32 = rel_l2(got, ref), rel_l2(fp32, ref)
    print(f"\n{shape} x{batch} dir {d}: split-BF16 rel-L2 {e_tc:.3e} max {max_err(got, ref):.3e} | "
          f"FP32 rel-L2 {e_32:.3e} max {max_err(fp32, ref):.3e}")
    assert e_tc <= 1e-5 * max(1.0, math.log2(n))
    assert e_tc <= 2e-5


def test_split_precision_3d_config(torch):
    """3D 256^3 in place, forward then backward with backward normalization, input uniform
    plus eight plane waves; every axis runs on the tensor cores."""
    import syclfft_b200 as sf
    shape = [256, 256, 256]
    n = 256 ** 3
    rng = np.random.default_rng(404)
    x = uniform_complex(n, 404, np.complex64).reshape(shape)
    grid = np.indices(shape, dtype=np.float64)
    for _ in range(8):
        k = rng.integers(-128, 128, 3)
        amp, ph = rng.uniform(0.5, 2.0), rng.uniform(0, 2 * np.pi)
        x += (amp * np.exp(1j * (2 * np.pi * np.tensordot(k, grid, axes=1) / 256 + ph))).astype(np.complex64)
    x = x.reshape(-1).astype(np.complex64)
    del grid
    ref = np.fft.fftn(x.reshape(shape).astype(np.complex128)).reshape(-1)
    res = {}
    for split in (True, False):
        opts = sf.plan_options(placement=sf.placement.in_place, normalization=sf.normalization.backward,
                               split_precision=split)
        fwd = sf.plan_many_dft("float", shape, 1, sf.direction.forward, opts)
        bwd = sf.plan_many_dft("float", shape, 1, sf.direction.backward, opts)
        assert (len(tc_passes(fwd.describe())) == 3) == split
        buf = torch.from_numpy(x.copy()).cuda()
        fwd.execute(buf).synchronize()
        spec = buf.cpu().numpy()
        bwd.execute(buf).synchronize()
        back = buf.cpu().numpy()
        res[split] = (rel_l2(spec, ref), max_err(spec, ref), rel_l2(back, x), max_err(back, x))
    for split, (e, m, rt, rtm) in res.items():
        print(f"\n256^3 {'split-BF16' if split else 'FP32'}: forward rel-L2 {e:.3e} max {m:.3e}; "
              f"round trip rel-L2 {rt:.3e} max {rtm:.3e}")
    e, _, rt, _ = res[True]
    assert e <= 2e-5 and rt <= 4e-5


def test_split_precision_other_lengths_and_double(torch):
    """Lengths without a tensor-core kernel, and double plans, keep their FP32/FP64 passes."""
    for shape, dbl in (([1000], False), ([13440], False), ([65536], False), ([256], True), ([4096, 4096], False)):
        import syclfft_b200 as sf
        opts = sf.plan_options(split_precision=True)
        batch = 1 if len(shape) == 2 else 4
        p = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction.forward, opts)
        d = p.describe()
        if shape == [4096, 4096]:
            # the contiguous 4096-point axis runs on the tensor cores; the strided one is FP32
            assert len(tc_passes(d)) == 1
        else:
            assert not tc_passes(d), (shape, d)
        n = int(np.prod(shape))
        dt = np.complex128 if dbl else np.complex64
        x = uniform_complex(n * batch, n + batch, dt)
        xi = torch.from_numpy(x).cuda()
        out = torch.empty_like(xi)
        p.execute(xi, out).synchronize()
        tol = (1e-12 if dbl else 1e-5) * max(1.0, math.log2(n))
        assert rel_l2(out.cpu().numpy(), fp64_fft(x, shape, batch, -1)) <= tol


def test_split_precision_batch_and_override(torch):
    """execute_batch (first b transforms) and execute_ex (direction / normalization
    override) on a tensor-core plan."""
    from syclfft_b200 import _provider
    lib = _provider.load()
    api = _provider.provider(lib)
    err = ctypes.create_string_buffer(1024)
    cfg = _provider.make_config([256], 64, -1, double=False, normalization=0)
    h = lib.syclfft_b200_create_ex(ctypes.byref(cfg), _provider.CREATE_SYNC | _provider.CREATE_SPLIT_BF16, err, 1024)
    assert h, err.value
    x = uniform_complex(256 * 64, 99, np.complex64)
    xi = torch.from_numpy(x).cuda()
    out = torch.zeros_like(xi)
    s = torch.cuda.current_stream().cuda_stream
    assert lib.syclfft_b200_execute_batch(h, xi.data_ptr(), out.data_ptr(), 20, s, err, 1024) == 0, err.value
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert rel_l2(got[: 256 * 20], fp64_fft(x[: 256 * 20], [256], 20, -1)) <= 2e-5
    assert not np.any(got[256 * 20:])
    assert lib.syclfft_b200_execute_ex(h, xi.data_ptr(), out.data_ptr(), 64, 1, 3, s, err, 1024) == 0, err.value
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), fp64_fft(x, [256], 64, 1, 1 / 16)) <= 2e-5
    api.destroy(h)
