"""CPU checks of the fused four-step kernel's tile schedule (no GPU): the schedule code the
kernel runs (sycl-fft_b200/csrc/fused4_schedule.h) hands every column and row tile of every
line out exactly once, every dependency wait points at an earlier ticket (so blocks that claim
tickets in order cannot deadlock, whatever their number), the ring and the control words fit
the plan's scratch, and a simulation with the kernel's counter targets finishes."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native")


@pytest.fixture(scope="module")
def lib():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    L = ctypes.CDLL(os.path.join(HERE, "libfused4_check.so"))
    L.f4_check.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int64,
                           ctypes.c_int64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_int64)]
    return L


CTRL_BYTES = (2 + 2 * 64) * 4  # kFused4CtrlWords 32-bit words


@pytest.mark.parametrize("tc,tr,line_bytes", [(32, 32, 65536 * 16), (16, 16, 65536 * 8)])
@pytest.mark.parametrize("lines", [3, 4, 5, 7, 16, 33, 100, 512, 1000])
@pytest.mark.parametrize("blocks", [1, 2, 64, 592, 1184])
def test_schedule(lib, tc, tr, line_bytes, lines, blocks):
    lag, ring, waits = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
    rc = lib.f4_check(lines, blocks, tc, tr, 64, CTRL_BYTES, line_bytes, ctypes.byref(lag), ctypes.byref(ring),
                      ctypes.byref(waits))
    assert rc == 0, (rc, lag.value, ring.value)
    assert 0 <= lag.value < ring.value <= min(lines - 1, 64)


def test_full_config_lag_leaves_few_waits(lib):
    """c128 65536 x 512 on 148 SMs x 4 blocks: the lag covers the tiles in flight."""
    lag, ring, waits = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
    assert lib.f4_check(512, 592, 32, 32, 64, CTRL_BYTES, 65536 * 16, ctypes.byref(lag), ctypes.byref(ring),
                        ctypes.byref(waits)) == 0
    assert ring.value * 65536 * 16 <= 64 << 20  # the ring stays far inside the 126 MB L2
    assert waits.value < 0.05 * 512 * 64
