"""Failure detection on the GPU without a fault: a bounded device wait that gives up.

Every wait on an mbarrier in the provider's kernels is bounded. A plan's wait limit can be
set from the host (syclfft_b200_plan_set_wait_limit, or SYCLFFT_B200_WAIT_POLLS for new
plans); with 0 polls every such wait of the next execution gives up at once. The block then
records the failure in the plan's status word, lets the copy or tensor-core product it gave
up on finish (bounded), frees what it holds and exits, so the context stays usable. The
execution's event raises execution_failed -- the reference's code for a failed provider
execution (src/sycl/sycl.cpp:671-676) -- once; later executions with the default limit are
correct.
"""
import ctypes
import math

import numpy as np
import pytest

from conftest import fp64_fft, rel_l2, uniform_complex

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


# (shape, batch, split precision, pass kind that waits): the copy-pipelined kernel (bulk-copy
# waits), the tensor-core kernel (MMA-commit waits) and the fused four-step (dependency waits
# on counters between its column and row tiles)
WAITING = [([13440], 32, False, "piped"), ([256], 512, True, "tc"), ([65536], 16, False, "fused_fourstep")]


@pytest.mark.parametrize("shape,batch,split,kind", WAITING, ids=lambda v: str(v))
def test_wait_that_gives_up_raises_execution_failed(sf, torch, monkeypatch, shape, batch, split, kind):
    monkeypatch.setenv("SYCLFFT_B200_FUSED4", "1")  # the fused kernels are opt-in
    n = int(np.prod(shape))
    x = uniform_complex(n * batch, 77 + n)
    xt = torch.from_numpy(x).cuda()
    out = torch.empty_like(xt)
    p = sf.plan_many_dft("float", shape, batch, sf.direction.forward, sf.plan_options(split_precision=split))
    desc = p.describe()
    runs = {"piped": any(ps["piped_id"] >= 0 for ps in desc["passes"]),
            "tc": any(ps["tc_id"] >= 0 for ps in desc["passes"]),
            "fused_fourstep": bool(desc.get("fused_fourstep"))}
    assert runs[kind], desc
    lib = p._lib
    assert lib.syclfft_b200_plan_set_wait_limit(p._handle, 0) == 0
    ev = p.execute(xt, out)
    with pytest.raises(sf.SyclfftError) as info:
        ev.synchronize()
    assert info.value.code == sf.error_code.execution_failed
    assert lib.syclfft_b200_plan_status(p._handle) == 0  # reported once, then cleared
    ev.synchronize()
    # the context and the plan are still usable: the default limit gives a correct result
    assert lib.syclfft_b200_plan_set_wait_limit(p._handle, -1) == 0
    p.execute(xt, out).synchronize()
    tol = (2e-5 if split else 1e-5) * math.log2(n)
    assert rel_l2(out.cpu().numpy(), fp64_fft(x, shape, batch, -1)) <= tol


def test_wait_limit_from_environment(sf, torch, monkeypatch):
    n, batch = 13440, 16
    xt = torch.ones(n * batch, dtype=torch.complex64, device="cuda")
    out = torch.empty_like(xt)
    monkeypatch.setenv("SYCLFFT_B200_WAIT_POLLS", "0")
    impatient = sf.plan_many_dft("float", [n], batch, sf.direction.forward)
    monkeypatch.delenv("SYCLFFT_B200_WAIT_POLLS")
    healthy = sf.plan_many_dft("float", [n], batch, sf.direction.forward)
    with pytest.raises(sf.SyclfftError) as info:
        impatient.execute(xt, out).synchronize()
    assert info.value.code == sf.error_code.execution_failed
    healthy.execute(xt, out).synchronize()
    got = out.view(batch, n).cpu().numpy()
    assert np.allclose(got[:, 0], n, rtol=1e-5) and np.abs(got[:, 1:]).max() < 1e-2


def test_misaligned_buffers_are_refused_before_launch(sf, torch):
    """Kernels move whole complex elements; an address off the element boundary is refused on
    the host (a device-side misaligned access would leave the context unusable)."""
    for dbl, n in ((False, 4096), (True, 2048)):
        el = 16 if dbl else 8
        raw = torch.zeros(2 * n * el + 64, dtype=torch.uint8, device="cuda")
        base = raw.data_ptr()
        p = sf.plan_many_dft("double" if dbl else "float", [n], 1, sf.direction.forward)
        err = ctypes.create_string_buffer(1024)
        rc = p._api.execute(p._handle, base + el // 2, base + n * el + el, torch.cuda.current_stream().cuda_stream,
                            err, 1024)
        assert rc != 0 and b"aligned" in err.value
        torch.cuda.synchronize()
        assert int(torch.count_nonzero(raw)) == 0
