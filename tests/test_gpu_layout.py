"""GPU parity of strided ("advanced") layouts (syclfft_b200_create_strided via
plan_many_dft(layout=...)): the logical batch is read through the input layout and written
through the output layout; checked against numpy FFTs in FP64 at the complex tolerance of the
same shape (rel-L2 <= 1e-5 * log2(N) float, 1e-12 * log2(N) double), and every output
element outside the layout must keep its sentinel value."""
import math

import numpy as np
import pytest

from conftest import norm_scale, rel_l2

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


def offsets(shape, batch, strides, dist):
    idx = np.zeros([batch] + list(shape), dtype=np.int64)
    idx += (np.arange(batch) * dist).reshape([batch] + [1] * len(shape))
    for k, (n, s) in enumerate(zip(shape, strides)):
        view = [1] * (len(shape) + 1)
        view[k + 1] = n
        idx += (np.arange(n) * s).reshape(view)
    return idx


def run_layout(torch, sf, shape, batch, lay, d=-1, norm=0, dbl=False, in_place=False, seed=0):
    n = math.prod(shape)
    dt = np.complex128 if dbl else np.complex64
    rng = np.random.default_rng(seed + n + batch)
    ext_in = lay.extent(shape, batch, False)
    ext_out = lay.extent(shape, batch, True)
    buf = (rng.uniform(-1, 1, ext_in) + 1j * rng.uniform(-1, 1, ext_in)).astype(dt)
    oi = offsets(shape, batch, lay.in_strides, lay.in_distance)
    oo = offsets(shape, batch, lay.out_strides, lay.out_distance)
    x = buf[oi].astype(np.complex128)
    axes = tuple(range(1, len(shape) + 1))
    ref = (np.fft.fftn(x, axes=axes) if d == -1 else np.fft.ifftn(x, axes=axes) * n) * norm_scale(norm, d, n)
    opts = sf.plan_options(placement=sf.placement.in_place if in_place else sf.placement.out_of_place,
                           normalization=sf.normalization(norm))
    p = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction(d), opts, layout=lay)
    a = torch.from_numpy(buf).cuda()
    if in_place:
        p.execute(a).synchronize()
        out = a.cpu().numpy()
        untouched = np.ones(ext_in, bool)
        untouched[oo.reshape(-1)] = False
        assert np.array_equal(out[untouched], buf[untouched])
    else:
        sentinel = np.complex64(3 - 5j) if not dbl else np.complex128(3 - 5j)
        o = torch.full((ext_out,), complex(sentinel), dtype=a.dtype, device="cuda")
        p.execute(a, o).synchronize()
        out = o.cpu().numpy()
        untouched = np.ones(ext_out, bool)
        untouched[oo.reshape(-1)] = False
        assert np.all(out[untouched] == sentinel)
        assert np.array_equal(a.cpu().numpy(), buf), "out-of-place input modified"
    got = out[oo]
    tol = (1e-12 if dbl else 1e-5) * max(1.0, math.log2(max(n, 2)))
    assert rel_l2(got, ref) <= tol
    return p


def L(in_strides, in_dist, out_strides, out_dist):
    import syclfft_b200
    return syclfft_b200.data_layout(tuple(in_strides), in_dist, tuple(out_strides), out_dist)


CASES = [
    # (shape, batch, layout, direction, norm, double, in_place)
    ([64], 24, L([24], 1, [1], 64), -1, 0, False, False),          # columns of a row-major matrix -> rows
    ([64], 24, L([1], 64, [24], 1), 1, 2, False, False),           # rows -> columns
    ([4096], 96, L([96], 1, [96], 1), -1, 3, False, True),         # columns, in place
    ([1000], 5, L([1], 1037, [1], 1037), -1, 0, True, True),       # padded rows, in place (double)
    ([256], 10, L([2], 1, [1], 256), -1, 0, False, False),         # overlapping input reads (stride 2, distance 1)
    ([13440], 3, L([3], 1, [1], 13441), -1, 3, False, False),      # pipelined kernel behind a gather
    ([1009], 7, L([7], 1, [7], 1), -1, 1, False, False),           # Bluestein, columns both sides
    ([12, 10], 3, L([10, 1], 130, [1, 12], 120), -1, 0, False, False),  # transposed output
    ([16, 24], 4, L([1, 16], 384, [24, 1], 400), 1, 0, True, False),   # transposed input, padded out
    ([8, 12, 10], 2, L([130, 10, 1], 1100, [120, 10, 1], 960), -1, 3, False, False),  # padded 3D
    ([6, 5, 4], 3, L([1, 6, 30], 120, [20, 4, 1], 120), 1, 2, True, False),  # fully reversed axis order
    ([12, 10], 3, L([30, 3], 1, [30, 3], 1), -1, 0, False, False),  # 2D over 3 interleaved arrays (direct)
    ([1024], 300, L([300], 1, [300], 1), 1, 3, True, True),         # columns in place, double (direct)
]


@pytest.mark.parametrize("shape,batch,lay,d,norm,dbl,in_place", CASES, ids=str)
def test_strided_layout_parity(torch, sf, shape, batch, lay, d, norm, dbl, in_place):
    p = run_layout(torch, sf, shape, batch, lay, d, norm, dbl, in_place)
    desc = p.describe()
    assert "layout" in desc and "inner" in desc
    # an interleaved batch (distance 1, dense columns) on both sides runs the axis passes
    # straight on the user's array: no gather / scatter launches
    rank_dense = lay.in_distance == 1 and lay.in_strides == lay.out_strides and lay.out_distance == 1 and all(
        s == batch * math.prod(shape[k + 1:]) for k, s in enumerate(lay.in_strides) if shape[k] > 1)
    assert desc["layout"]["interleaved"] == (1 if rank_dense else 0)
    if rank_dense:
        assert p.launches() == len(desc["inner"]["passes"])


def test_large_column_transform(torch, sf):
    """4096-point transforms down the 4096 columns of a row-major 4096 x 4096 float matrix,
    written as contiguous rows; FP64 check on 8 sampled columns."""
    n = b = 4096
    lay = sf.data_layout((b,), 1, (1,), n)
    x = torch.randn(n * b, dtype=torch.complex64, device="cuda")
    p = sf.plan_many_dft("float", [n], b, sf.direction.forward, layout=lay)
    out = torch.empty_like(x)
    p.execute(x, out).synchronize()
    cols = [0, 1, 31, 32, 1000, 2047, 4094, 4095]
    xm = x.view(n, b).cpu().numpy()
    om = out.view(b, n).cpu().numpy()
    for c in cols:
        ref = np.fft.fft(xm[:, c].astype(np.complex128))
        assert rel_l2(om[c], ref) <= 1e-5 * 12


def test_contiguous_layout_is_a_plain_plan(torch, sf):
    lay = sf.data_layout.contiguous([32, 16])
    p = sf.plan_many_dft("float", [32, 16], 4, sf.direction.forward, layout=lay)
    assert "layout" not in p.describe()
    run_layout(torch, sf, [32, 16], 4, lay)


def test_partial_batch(torch, sf):
    """The first b of B transforms (execute_batch) through a gathered layout: columns of a
    matrix with 20 columns, 16 of them transformed."""
    import ctypes
    from syclfft_b200 import _provider
    n, batch, pitch, run = 128, 16, 20, 5
    lay = sf.data_layout((pitch,), 1, (pitch,), 1)
    x = torch.randn(n * pitch, dtype=torch.complex64, device="cuda")
    out = torch.zeros_like(x)
    p = sf.plan_many_dft("float", [n], batch, sf.direction.forward, layout=lay)
    err = ctypes.create_string_buffer(_provider.ERR_CAP)
    rc = p._lib.syclfft_b200_execute_batch(p._handle, x.data_ptr(), out.data_ptr(), run,
                                           torch.cuda.current_stream().cuda_stream, err, _provider.ERR_CAP)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    xm, om = x.view(n, pitch).cpu().numpy(), out.view(n, pitch).cpu().numpy()
    ref = np.fft.fft(xm[:, :run].astype(np.complex128), axis=0)
    assert rel_l2(om[:, :run], ref) <= 1e-5 * 7
    assert np.all(om[:, run:] == 0)
    # an interleaved-batch plan (stride = batch, distance 1) runs its whole batch only
    q = sf.plan_many_dft("float", [n], batch, sf.direction.forward, layout=sf.data_layout((batch,), 1, (batch,), 1))
    rc = q._lib.syclfft_b200_execute_batch(q._handle, x.data_ptr(), out.data_ptr(), run,
                                           torch.cuda.current_stream().cuda_stream, err, _provider.ERR_CAP)
    assert rc != 0 and b"whole batch" in err.value


def test_layout_errors(torch, sf):
    E = sf.error_code.invalid_argument
    bad = [
        ([8], 4, sf.data_layout((1,), 8, (1,), 4), False),           # output rows overlap
        ([8], 4, sf.data_layout((0,), 8, (1,), 8), False),           # zero stride
        ([8], 4, sf.data_layout((1,), 8, (4,), 1), True),            # in place, different layouts
        ([8, 8], 2, sf.data_layout((8,), 64, (8, 1), 64), False),    # one stride for two axes
    ]
    for shape, batch, lay, ip in bad:
        opts = sf.plan_options(placement=sf.placement.in_place if ip else sf.placement.out_of_place)
        with pytest.raises(sf.SyclfftError) as e:
            sf.plan_many_dft("float", shape, batch, sf.direction.forward, opts, layout=lay)
        assert e.value.code == E
    p = sf.plan_many_dft("float", [8], 4, sf.direction.forward, layout=sf.data_layout((4,), 1, (1,), 10))
    with pytest.raises(sf.SyclfftError) as e:
        p.execute(torch.zeros(32, dtype=torch.complex64, device="cuda"),
                  torch.zeros(37, dtype=torch.complex64, device="cuda"))   # output extent is 38
    assert e.value.code == E
