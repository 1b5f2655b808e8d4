"""Loaders for the test-only host libraries in tests/native (built with its Makefile)."""
import ctypes
import json
import os
import subprocess

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "native")
_cache = {}


def _load(name):
    if name not in _cache:
        subprocess.run(["make", "-s", "-C", HERE], check=True)
        _cache[name] = ctypes.CDLL(os.path.join(HERE, name))
    return _cache[name]


def butterfly(radix, x, double=True):
    L = _load("libbutterfly_check.so")
    dt = np.float64 if double else np.float32
    xin = np.ascontiguousarray(np.stack([x.real, x.imag], -1).reshape(-1).astype(dt))
    out = np.zeros_like(xin)
    fn = L.sfb_check_dft_f64 if double else L.sfb_check_dft_f32
    rc = fn(int(radix), ctypes.c_void_p(xin.ctypes.data), ctypes.c_void_p(out.ctypes.data))
    assert rc == 0
    return out[0::2] + 1j * out[1::2]


def twiddle_powers(mode, radix, w, x, double=True):
    """u[r] * w^r (r = 1..radix-1, u[0] unchanged) through the size-specialised kernels'
    twiddle_powers (mode 0: the balanced product tree)."""
    L = _load("libbutterfly_check.so")
    dt = np.float64 if double else np.float32
    xin = np.ascontiguousarray(np.stack([x.real, x.imag], -1).reshape(-1).astype(dt))
    out = np.zeros_like(xin)
    fn = L.sfb_check_powers_f64 if double else L.sfb_check_powers_f32
    real = ctypes.c_double if double else ctypes.c_float
    fn.argtypes = [ctypes.c_int, ctypes.c_int, real, real, ctypes.c_void_p, ctypes.c_void_p]
    rc = fn(int(mode), int(radix), w.real, w.imag, ctypes.c_void_p(xin.ctypes.data), ctypes.c_void_p(out.ctypes.data))
    assert rc == 0
    return out[0::2] + 1j * out[1::2]


def emulate(x, shape, batch, direction, norm=0, double=False, in_place=False, force_maxv=0, smem_limit=0):
    """Run a plan through the FP64 pass emulator; returns (output, plan description)."""
    L = _load("libplan_emulator.so")
    L.emu_run.argtypes = [ctypes.c_int] * 4 + [ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                               ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
    sh = (ctypes.c_uint64 * 3)(*(list(shape) + [0] * (3 - len(shape))))
    xin = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
    out = np.zeros_like(xin)
    desc = ctypes.create_string_buffer(1 << 18)
    err = ctypes.create_string_buffer(1024)
    rc = L.emu_run(int(double), int(direction), int(norm), int(in_place), len(shape), sh, int(batch),
                   int(force_maxv), int(smem_limit), xin.ctypes.data, out.ctypes.data, desc, 1 << 18, err, 1024)
    if rc:
        raise RuntimeError(err.value.decode())
    return out, json.loads(desc.value.decode())


def emulate_skip(x, shape, batch, direction, skip_axes, norm=0, double=False, in_place=False):
    """emulate() with the axes in the bit mask `skip_axes` left untransformed."""
    L = _load("libplan_emulator.so")
    L.emu_run_skip.argtypes = [ctypes.c_int] * 4 + [ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint,
                                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                                                    ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t]
    sh = (ctypes.c_uint64 * 3)(*(list(shape) + [0] * (3 - len(shape))))
    xin = np.ascontiguousarray(np.asarray(x, dtype=np.complex128))
    out = np.zeros_like(xin)
    desc = ctypes.create_string_buffer(1 << 18)
    err = ctypes.create_string_buffer(1024)
    rc = L.emu_run_skip(int(double), int(direction), int(norm), int(in_place), len(shape), sh, int(batch),
                        int(skip_axes), xin.ctypes.data, out.ctypes.data, desc, 1 << 18, err, 1024)
    if rc:
        raise RuntimeError(err.value.decode())
    return out, json.loads(desc.value.decode())


def describe(shape, batch, direction=-1, norm=0, double=False, in_place=False, smem_limit=232448, split_bf16=False):
    """The planner's plan for a request (no execution), as the provider describes it."""
    L = _load("libplan_emulator.so")
    L.emu_describe.argtypes = [ctypes.c_int] * 4 + [ctypes.c_uint, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int,
                                                    ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_size_t,
                                                    ctypes.c_char_p, ctypes.c_size_t]
    sh = (ctypes.c_uint64 * 3)(*(list(shape) + [0] * (3 - len(shape))))
    desc = ctypes.create_string_buffer(1 << 18)
    err = ctypes.create_string_buffer(1024)
    rc = L.emu_describe(int(double), direction, norm, int(in_place), len(shape), sh, batch, 0, smem_limit,
                        int(split_bf16), desc, len(desc), err, len(err))
    if rc != 0:
        raise ValueError(err.value.decode())
    return json.loads(desc.value.decode())


def primitive_root(p):
    """The planner's primitive root mod the prime p (the generator of its Rader tables)."""
    L = _load("libplan_emulator.so")
    L.emu_primitive_root.restype = ctypes.c_uint64
    L.emu_primitive_root.argtypes = [ctypes.c_uint64]
    return int(L.emu_primitive_root(int(p)))
