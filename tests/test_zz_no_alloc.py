"""The allocation-free entry point (syclfft_b200_execute_noalloc_c2c_f32), called
through the C ABI, against the plan entry point on the same inputs.

It serves callers that cannot allocate device memory when they transform (a framework
whose memory planner owns the device, a real-time loop that must not call cudaMalloc):
its scratch and twiddles live in fixed arrays inside the library. This file is named to
be collected last, so a run that stops at the first failure has run everything else.
It passes alone in a fresh process and after the other tests.
"""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    if not t.cuda.is_available():
        pytest.skip("no CUDA device")
    return t


def rel_l2(a, b):
    a = a.to(dtype=b.dtype)
    return float((a - b).abs().pow(2).sum().sqrt() / b.abs().pow(2).sum().sqrt())


def plan_reference(torch, x, n, batch, direction, norm):
    """The existing entry point: a plan of the provider's C ABI."""
    from syclfft_b200 import _provider
    api = _provider.provider()
    err = ctypes.create_string_buffer(1024)
    cfg = _provider.make_config([n], batch, direction, double=False, normalization=norm)
    h = api.create(ctypes.byref(cfg), err, 1024)
    assert h, err.value
    y = torch.empty_like(x)
    rc = api.execute(h, x.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream, err, 1024)
    assert rc == 0, err.value
    torch.cuda.synchronize()
    api.destroy(h)
    return y


def noalloc(torch, x, out, n, batch, direction, norm):
    from syclfft_b200 import _provider
    lib = _provider.load()
    err = ctypes.create_string_buffer(1024)
    rc = lib.syclfft_b200_execute_noalloc_c2c_f32(x.data_ptr(), out.data_ptr(), n, batch, direction, norm,
                                                  torch.cuda.current_stream().cuda_stream, err, 1024)
    return rc, err.value.decode()


def check_against_plan(torch, cases):
    for n, batch, direction, norm in cases:
        g = torch.Generator(device="cuda").manual_seed(n + batch)
        x = torch.complex(torch.rand(n * batch, device="cuda", generator=g) * 2 - 1,
                          torch.rand(n * batch, device="cuda", generator=g) * 2 - 1)
        keep = x.clone()
        out = torch.empty_like(x)
        rc, msg = noalloc(torch, x, out, n, batch, direction, norm)
        assert rc == 0, msg
        torch.cuda.synchronize()
        assert torch.equal(x, keep)  # out-of-place input untouched
        ref = plan_reference(torch, x, n, batch, direction, norm)
        tol = 1e-5 * math.log2(n)  # the float tolerance of the parity tests
        assert rel_l2(out, ref) <= tol
        # also against an FP64 FFT of the same input
        xs = x.view(batch, n)[:2].cpu().numpy().astype(np.complex128)
        f = np.fft.fft(xs, axis=1) if direction == -1 else np.fft.ifft(xs, axis=1) * n
        scale = {0: 1.0, 1: (1 / n if direction == -1 else 1.0), 2: (1 / n if direction == 1 else 1.0),
                 3: 1 / math.sqrt(n)}[norm]
        got = out.view(batch, n)[:2].cpu().numpy()
        assert np.linalg.norm(got - f * scale) / np.linalg.norm(f * scale) <= tol


def test_noalloc_matches_plan_entry_point_twice(torch):
    # two calls in a row, different length and direction
    check_against_plan(torch, [(65536, 8, -1, 3), (1 << 20, 2, 1, 2)])


@pytest.mark.parametrize("case", [(1 << 15, 1, 1, 0), (1 << 20, 4, -1, 1), (1 << 17, 3, 1, 2)])
def test_noalloc_boundary_cases(torch, case):
    # the shortest length (128 x 256 split), a batch exactly at the 4 Mi element limit, an odd
    # batch; every normalization in one direction or the other
    check_against_plan(torch, [case])


def test_noalloc_in_place_and_limits(torch):
    n, batch = 32768, 4
    x = torch.randn(n * batch, dtype=torch.complex64, device="cuda")
    ref = plan_reference(torch, x, n, batch, -1, 0)
    rc, msg = noalloc(torch, x, x, n, batch, -1, 0)
    assert rc == 0, msg
    torch.cuda.synchronize()
    assert rel_l2(x, ref) <= 1e-5 * math.log2(n)
    big = torch.empty(1, dtype=torch.complex64, device="cuda")
    rc, msg = noalloc(torch, big, big, 1 << 20, 8, -1, 0)  # 8 Mi elements > the 4 Mi limit
    assert rc != 0 and "limited" in msg
    rc, msg = noalloc(torch, big, big, 3 * 4096, 1, -1, 0)
    assert rc != 0 and "power-of-two" in msg
    # a view 4 bytes into a buffer: refused on the host before anything is launched
    raw = torch.zeros(2 * n + 2, dtype=torch.float32, device="cuda")
    base = raw.data_ptr()
    err = ctypes.create_string_buffer(1024)
    from syclfft_b200 import _provider
    rc = _provider.load().syclfft_b200_execute_noalloc_c2c_f32(base + 4, base + 4, n, 1, -1, 0,
                                                               torch.cuda.current_stream().cuda_stream, err, 1024)
    assert rc != 0 and "aligned" in err.value.decode()
    torch.cuda.synchronize()
    assert int(torch.count_nonzero(raw)) == 0
