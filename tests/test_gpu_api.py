"""Plan API semantics on the GPU: the reference's error-code cases
(tests/sycl_tests.cpp:508-538, host_tests.cpp:167-195), provider selection and
query_providers (sycl.cpp:447-475, 909-947), scratch size and the raw C ABI."""
import ctypes

import numpy as np
import pytest

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


def expect(sf, code, fn):
    with pytest.raises(sf.SyclfftError) as ei:
        fn()
    assert ei.value.code == code, str(ei.value)


def test_error_codes(sf, torch):
    E = sf.error_code
    fwd = sf.direction.forward
    expect(sf, E.invalid_argument, lambda: sf.plan_dft_1d("float", 8, 0))
    expect(sf, E.invalid_argument, lambda: sf.plan_dft_1d("float", 0, fwd))
    expect(sf, E.invalid_argument, lambda: sf.plan_many_dft("float", [2, 2, 2, 2], 1, fwd))
    expect(sf, E.invalid_argument, lambda: sf.plan_many_dft("float", [8], 0, fwd))
    expect(sf, E.invalid_argument, lambda: sf.plan_many_dft("float", [2 ** 63, 4], 1, fwd))
    expect(sf, E.provider_unavailable, lambda: sf.plan_dft_1d(
        "float", 8, fwd, sf.plan_options(preferred_provider=sf.provider.cufft)))
    expect(sf, E.provider_unavailable, lambda: sf.plan_dft_1d(
        "float", 8, fwd, sf.plan_options(preferred_provider=sf.provider.portable_sycl)))
    p = sf.plan_dft_1d("float", 8, fwd)
    expect(sf, E.invalid_pointer, lambda: p.execute(None, None))
    expect(sf, E.invalid_pointer, lambda: p.execute(torch.zeros(8, dtype=torch.complex64), torch.zeros(8, dtype=torch.complex64)))
    x = torch.zeros(8, dtype=torch.complex64, device="cuda")
    expect(sf, E.invalid_argument, lambda: p.execute(x))
    expect(sf, E.invalid_argument, lambda: p.execute(x, x))
    expect(sf, E.invalid_argument, lambda: p.execute(x.to(torch.complex128), torch.zeros_like(x)))
    ip = sf.plan_dft_1d("float", 8, fwd, sf.plan_options(placement=sf.placement.in_place))
    expect(sf, E.invalid_argument, lambda: ip.execute(x, torch.zeros_like(x)))
    moved = ip.move()
    expect(sf, E.invalid_state, lambda: ip.execute(x))
    moved.execute(x).synchronize()
    assert ip.shape() == [] and moved.shape() == [8]


def test_provider_selection_and_query(sf, torch):
    p = sf.plan_dft_1d("float", 8, sf.direction.forward)
    assert p.selected_provider() == sf.provider.b200
    rows = sf.query_providers()
    b200 = [r for r in rows if r["name"] == "b200"][0]
    assert b200["built"] and b200["available"], b200["reason"]
    assert all(r["reason"] for r in rows if not r["available"])


def test_scratch_size(sf, torch, monkeypatch):
    assert sf.plan_many_dft("float", [4096], 16, sf.direction.forward).scratch_size_bytes() == 0
    assert sf.plan_many_dft("double", [65536], 4, sf.direction.forward).scratch_size_bytes() >= 65536 * 4 * 16
    monkeypatch.setenv("SYCLFFT_B200_CLUSTER", "8")
    assert sf.plan_many_dft("double", [65536], 4, sf.direction.forward).scratch_size_bytes() == 0  # cluster kernel
    monkeypatch.delenv("SYCLFFT_B200_CLUSTER")
    assert sf.plan_many_dft("double", [65536, 3], 1, sf.direction.forward).scratch_size_bytes() >= 65536 * 3 * 16
    # Rader: the convolution of a prime length L runs over L - 1 (65536) points
    assert sf.plan_many_dft("float", [65537], 2, sf.direction.forward).scratch_size_bytes() == 2 * 65536 * 8
    # Bluestein: over M >= 2L - 2 (131072 for L = 65521)
    assert sf.plan_many_dft("float", [65521], 2, sf.direction.forward).scratch_size_bytes() >= 2 * 131072 * 8


def test_raw_c_abi(sf, torch):
    from syclfft_b200 import _provider
    api = _provider.provider()
    err = ctypes.create_string_buffer(1024)
    assert api.supports(torch.cuda.current_device(), err, 1024) == 1
    cfg = _provider.make_config([1024], 4, -1, double=False, normalization=3)
    h = api.create(ctypes.byref(cfg), err, 1024)
    assert h, err.value
    x = torch.randn(4096, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    s = torch.cuda.current_stream()
    assert api.execute(h, x.data_ptr(), y.data_ptr(), s.cuda_stream, err, 1024) == 0, err.value
    torch.cuda.synchronize()
    ref = np.fft.fft(x.cpu().numpy().reshape(4, 1024).astype(np.complex128), axis=1, norm="ortho")
    assert np.abs(y.cpu().numpy().reshape(4, 1024) - ref).max() < 1e-4
    # in-place plan given distinct pointers -> error status, no exception across the ABI
    assert api.execute(h, x.data_ptr(), x.data_ptr(), s.cuda_stream, err, 1024) != 0
    assert b"distinct" in err.value
    api.destroy(h)
    bad = _provider.make_config([16], 1, -1)
    bad.abi_version = 2
    assert not api.create(ctypes.byref(bad), err, 1024) and b"ABI" in err.value
    bad = _provider.make_config([16], 1, 0)
    assert not api.create(ctypes.byref(bad), err, 1024) and b"direction" in err.value


@pytest.mark.parametrize("shape,batch,dbl", [([4096], 512, False), ([13440], 64, False), ([65536], 8, True),
                                             ([1009], 32, False), ([64, 64], 4, True)], ids=str)
def test_autotuned_plans(sf, torch, shape, batch, dbl, tmp_path, monkeypatch):
    """planning_mode::measure times candidate kernels, reports them, keeps the fastest, and
    reuses the decision from the on-disk cache."""
    from conftest import fp64_fft, rel_l2, uniform_complex
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("SYCLFFT_B200_TUNE_CACHE", str(cache))
    opts = sf.plan_options(planning=sf.planning_mode.measure)
    kind = "double" if dbl else "float"
    p = sf.plan_many_dft(kind, shape, batch, sf.direction.forward, opts)
    tuning = p.describe()["tuning"]
    assert tuning["choice"] and (tuning.get("cached") or len(tuning["candidates"]) >= 1), tuning
    n = int(np.prod(shape))
    x = uniform_complex(n * batch, n, np.complex128 if dbl else np.complex64)
    xt = torch.from_numpy(x).cuda()
    out = torch.empty_like(xt)
    p.execute(xt, out).synchronize()
    tol = (1e-12 if dbl else 1e-5) * max(1.0, np.log2(n))
    assert rel_l2(out.cpu().numpy(), fp64_fft(x, shape, batch, -1)) <= tol
    assert cache.exists()
