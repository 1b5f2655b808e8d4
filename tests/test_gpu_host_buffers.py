"""Page-locked host buffers through the plan API (host USM, which the reference's execute
accepts: src/sycl/sycl.cpp:72-85). With host tensors on both sides the batch streams through
the device in chunks (syclfft_b200_execute_host): copy in, the transform(s), copy out, on
overlapping streams. Results equal the device-buffer path of the same plan; chained stages
(forward then backward on one plan) equal running them one after the other on the device.
"""
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


@pytest.fixture(scope="module")
def sf():
    import syclfft_b200
    return syclfft_b200


# (shape, batch, double, in place): several 32 MiB chunks, a ragged last chunk, a line larger
# than a chunk (256^3 complex<float> is 128 MiB), Bluestein, four-step, multi-axis
CASES = [([4096], 3000, False, False), ([13440], 700, False, True), ([65536], 100, True, True),
         ([1009], 5000, False, False), ([256, 256, 256], 1, False, True), ([2048, 2048], 2, True, False),
         ([1024], 1, False, False)]


@pytest.mark.parametrize("shape,batch,dbl,in_place", CASES, ids=lambda v: str(v))
def test_host_buffers_match_device_path(sf, torch, shape, batch, dbl, in_place):
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 11 + n, dt)
    opts = sf.plan_options(placement=sf.placement.in_place if in_place else sf.placement.out_of_place,
                           normalization=sf.normalization.orthogonal)
    p = sf.plan_many_dft("double" if dbl else "float", shape, batch, sf.direction.forward, opts)
    dev = torch.from_numpy(x).cuda()
    if in_place:
        p.execute(dev).synchronize()
        expected = dev.cpu()
    else:
        dout = torch.empty_like(dev)
        p.execute(dev, dout).synchronize()
        expected = dout.cpu()
    hin = torch.from_numpy(x).pin_memory()
    if in_place:
        p.execute(hin).synchronize()
        got = hin
    else:
        hout = torch.empty_like(hin).pin_memory()
        p.execute(hin, hout).synchronize()
        got = hout
        assert torch.equal(hin, torch.from_numpy(x))  # the input of an out-of-place plan is kept
    tol = (1e-12 if dbl else 1e-6)
    assert rel_l2(got.numpy(), expected.numpy()) <= tol
    k = min(batch, 2)
    ref = fp64_fft(x[: k * n], shape, k, -1, norm_scale(3, -1, n))
    assert rel_l2(got.numpy()[: k * n], ref) <= (1e-12 if dbl else 1e-5) * max(1, math.log2(n))


def test_chained_stages_round_trip(sf, torch):
    """forward then backward (backward normalization) in one streamed call: the input back."""
    n, batch = 4096, 6000
    x = uniform_complex(n * batch, 5)
    p = sf.plan_many_dft("float", [n], batch, sf.direction.forward,
                         sf.plan_options(placement=sf.placement.in_place,
                                         normalization=sf.normalization.backward))
    hin = torch.from_numpy(x).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    ev = sf.execute_host([(p, sf.direction.forward), (p, sf.direction.backward)], hin, hout)
    ev.synchronize()
    assert rel_l2(hout.numpy(), x) <= 1e-5 * math.log2(n)
    # stage by stage on the device gives the same values
    dev = torch.from_numpy(x).cuda()
    p.execute(dev)
    lib, err = p._lib, p._err
    import ctypes
    rc = lib.syclfft_b200_execute_ex(p._handle, dev.data_ptr(), dev.data_ptr(), 0, 1, -1,
                                     torch.cuda.current_stream().cuda_stream, err, 1024)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    assert rel_l2(hout.numpy(), dev.cpu().numpy()) <= 1e-6


def test_host_buffer_errors(sf, torch):
    p = sf.plan_many_dft("float", [1024], 4, sf.direction.forward)
    pageable = torch.zeros(4096, dtype=torch.complex64)
    pinned = torch.zeros(4096, dtype=torch.complex64).pin_memory()
    with pytest.raises(sf.SyclfftError) as info:
        sf.execute_host([p], pageable, pinned)
    assert info.value.code == sf.error_code.invalid_pointer
    with pytest.raises(sf.SyclfftError) as info:
        p.execute(pageable, torch.zeros(4096, dtype=torch.complex64, device="cuda"))
    assert info.value.code == sf.error_code.invalid_pointer
    with pytest.raises(sf.SyclfftError) as info:
        sf.execute_host([p], torch.zeros(100, dtype=torch.complex64).pin_memory(), pinned)
    assert info.value.code == sf.error_code.invalid_argument
    q = sf.plan_many_dft("float", [2048], 4, sf.direction.forward)
    with pytest.raises(sf.SyclfftError) as info:
        sf.execute_host([p, q], pinned, pinned)
    assert info.value.code == sf.error_code.execution_failed and "transform size" in str(info.value)


def test_pinned_host_on_one_side_is_read_directly(sf, torch):
    """A page-locked host input with a device output: the kernels read the input over the bus."""
    n, batch = 4096, 8
    x = uniform_complex(n * batch, 9)
    p = sf.plan_many_dft("float", [n], batch, sf.direction.forward)
    hin = torch.from_numpy(x).pin_memory()
    out = torch.empty(n * batch, dtype=torch.complex64, device="cuda")
    p.execute(hin, out).synchronize()
    assert rel_l2(out.cpu().numpy(), fp64_fft(x, [n], batch, -1)) <= 1e-5 * math.log2(n)
