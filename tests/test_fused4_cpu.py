"""CPU checks of the fused multi-pass kernels' tile schedule (no GPU): the schedule code the
kernels run (sycl-fft_b200/csrc/fused4_schedule.h) hands every tile of every phase of every
line out exactly once, every dependency wait points at an earlier ticket (so blocks that
claim tickets in order cannot deadlock, whatever their number), the ring and the control
words fit the plan's scratch, and a simulation with the kernels' counter targets finishes."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native")
CTRL_BYTES = (2 + 3 * 64) * 4  # control words: ticket, abort, 3 phases x 64 ring slots


@pytest.fixture(scope="module")
def lib():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    L = ctypes.CDLL(os.path.join(HERE, "libfused4_check.so"))
    L.f4_check.argtypes = [ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                           ctypes.c_int64, ctypes.c_int64, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_int64)]
    return L


def check(lib, lines, blocks, tiles, line_bytes):
    lag, ring, waits = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
    arr = (ctypes.c_int * len(tiles))(*tiles)
    rc = lib.f4_check(lines, blocks, len(tiles), arr, 64, CTRL_BYTES, line_bytes, ctypes.byref(lag),
                      ctypes.byref(ring), ctypes.byref(waits))
    return rc, lag.value, ring.value, waits.value


# four-step (column tiles, row tiles) and Bluestein (forward columns, row convolution, inverse
# columns) tile counts, with their line sizes in bytes
SHAPES = [((32, 32), 65536 * 16), ((16, 16), 65536 * 8), ((8, 15), 13440 * 8), ((32, 20, 32), 163840 * 8),
          ((16, 10, 16), 163840 * 16)]


@pytest.mark.parametrize("tiles,line_bytes", SHAPES, ids=str)
@pytest.mark.parametrize("lines", [3, 4, 5, 7, 16, 33, 100, 512, 1000])
@pytest.mark.parametrize("blocks", [1, 2, 64, 592, 1184])
def test_schedule(lib, tiles, line_bytes, lines, blocks):
    rc, lag, ring, _ = check(lib, lines, blocks, tiles, line_bytes)
    assert rc == 0, (rc, lag, ring)
    if lines >= len(tiles) + 1:
        assert 1 <= lag and (len(tiles) - 1) * lag < ring <= min(lines - 1, 64)


def test_capped_ring_keeps_reuse_gap(lib):
    """c64 65536 x 1024 on 1184 blocks in flight: the wanted ring (80 slots) exceeds the cap of
    64, so lag and reuse gap share it instead of the lag taking all of it (a slot's next user
    then waits right behind its last one)."""
    rc, lag, ring, waits = check(lib, 1024, 1184, (16, 16), 65536 * 8)
    assert rc == 0 and ring == 64 and lag == 32
    assert waits < 0.25 * 1024 * 32  # not one wait per tile: the lag and the reuse gap share the ring


def test_full_config_lag_leaves_few_waits(lib):
    """c128 65536 x 512 on 148 SMs x 4 blocks: the lag covers the tiles in flight."""
    rc, lag, ring, waits = check(lib, 512, 592, (32, 32), 65536 * 16)
    assert rc == 0
    assert ring * 65536 * 16 <= 64 << 20  # the ring stays far inside the 126 MB L2
    assert waits < 0.05 * 512 * 64
