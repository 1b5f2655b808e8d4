"""The CPython fast-call shim (sycl-fft_b200/csrc/fastcall.c) that Plan.execute uses for the
provider's execute entry: arguments arrive in order and unchanged, the return code comes back,
and bad arguments raise instead of calling. Runs without a GPU: the entry is a ctypes callback
with the provider table's execute signature."""
import ctypes
import os
import sys

import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sycl-fft_b200"))

EXEC_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_char_p, ctypes.c_size_t)


def test_fastcall_passes_arguments_and_return_code():
    from syclfft_b200 import _fastcall
    seen = []

    def entry(plan, inp, out, stream, err, cap):
        seen.append((plan, inp, out, stream, cap))
        return 7

    cb = EXEC_FN(entry)
    addr = ctypes.cast(cb, ctypes.c_void_p).value
    err = ctypes.create_string_buffer(64)
    rc = _fastcall.execute(addr, 0x1000, 0x7f0000001000, 0x7f0000002000, 0, ctypes.addressof(err), 64)
    assert rc == 7
    assert seen == [(0x1000, 0x7f0000001000, 0x7f0000002000, None, 64)]


def test_fastcall_rejects_bad_arguments():
    from syclfft_b200 import _fastcall
    with pytest.raises(TypeError):
        _fastcall.execute(1, 2, 3)
    with pytest.raises(ValueError):
        _fastcall.execute(0, 1, 2, 3, 4, 5, 6)  # no entry to call
    with pytest.raises((TypeError, OverflowError)):
        _fastcall.execute(1, "plan", 2, 3, 4, 5, 6)
