"""ctypes wrapper around the CPU restatement of the syclfft portable provider.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` as the
checker, and by bench.py's CPU-baseline / reference arm. The product library never
imports this module. The restated algorithm (src/sycl/sycl.cpp:34-339, 509-569,
688-775 of Vaskozlov/sycl-fft) lives in oracle/portable_ref.cpp.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle_portable.so")
_lib = None

NORMALIZATIONS = {"none": 0, "forward": 1, "backward": 2, "orthogonal": 3}
DIRECTIONS = {"forward": -1, "backward": 1}


def build() -> str:
    """Compile the restatement with its Makefile (g++ -O3 -fopenmp)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_plan_create.restype = ctypes.c_void_p
        L.oracle_plan_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint64,
                                         ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_plan_execute.restype = ctypes.c_int
        L.oracle_plan_execute.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_plan_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_plan_scratch_bytes.restype = ctypes.c_uint64
        L.oracle_plan_scratch_bytes.argtypes = [ctypes.c_void_p]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


class OraclePlan:
    """A plan of the restated portable provider (plan creation = table build)."""

    def __init__(self, lengths, batch: int, direction: str | int, normalization: str | int = "none",
                 double: bool = False):
        L = lib()
        self.lengths = [int(v) for v in lengths]
        self.batch = int(batch)
        self.double = bool(double)
        d = DIRECTIONS[direction] if isinstance(direction, str) else int(direction)
        n = NORMALIZATIONS[normalization] if isinstance(normalization, str) else int(normalization)
        padded = (self.lengths + [0, 0, 0])[:max(3, len(self.lengths))]
        arr = (ctypes.c_uint64 * len(padded))(*padded)
        err = ctypes.create_string_buffer(1024)
        self._h = L.oracle_plan_create(int(self.double), d, n, len(self.lengths), arr,
                                       self.batch, err, 1024)
        if not self._h:
            raise ValueError(err.value.decode())
        self.count = self.batch * int(np.prod(self.lengths))
        self.dtype = np.complex128 if self.double else np.complex64

    def scratch_bytes(self) -> int:
        return int(lib().oracle_plan_scratch_bytes(self._h))

    def execute(self, x: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=self.dtype).reshape(-1)
        if x.size != self.count:
            raise ValueError("input size mismatch")
        if out is None:
            out = np.empty_like(x)
        err = ctypes.create_string_buffer(1024)
        rc = lib().oracle_plan_execute(self._h, x.ctypes.data, out.ctypes.data, err, 1024)
        if rc != 0:
            raise RuntimeError(err.value.decode())
        return out

    def close(self):
        if getattr(self, "_h", None):
            lib().oracle_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def portable_fft(x, lengths, batch, direction, normalization="none", double=None):
    """One-shot helper: plan + execute on a host array."""
    if double is None:
        double = np.asarray(x).dtype == np.complex128
    p = OraclePlan(lengths, batch, direction, normalization, double)
    try:
        return p.execute(x)
    finally:
        p.close()
