"""ctypes binding of the B200 provider's C ABI (include/syclfft_b200_provider.h).

This is the raw drop-in boundary: plan configs, the provider table and device
pointers on a CUDA stream. The higher-level mirror of syclfft's plan API lives in
``syclfft_b200.api``.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_DIR = os.path.join(PKG_ROOT, "lib")
PROVIDER_DIR = os.path.join(LIB_DIR, "syclfft", "providers")
PROVIDER_PATH = os.path.join(PROVIDER_DIR, "syclfft_provider_b200.so")

ABI_VERSION = 1
CREATE_STREAM_SCRATCH = 1
CREATE_SYNC = 2
CREATE_SPLIT_BF16 = 4
REAL_R2C = 1
REAL_C2R = 2
SCALAR_FLOAT = 1
SCALAR_DOUBLE = 2
ERR_CAP = 1024


class PlanConfigV1(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32),
        ("scalar", ctypes.c_uint32),
        ("direction", ctypes.c_int32),
        ("rank", ctypes.c_uint32),
        ("lengths", ctypes.c_uint64 * 3),
        ("batch_count", ctypes.c_uint64),
        ("in_place", ctypes.c_uint32),
        ("normalization", ctypes.c_uint32),
        ("measure", ctypes.c_uint32),
        ("device", ctypes.c_int32),
    ]


_SUPPORTS = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t)
_CREATE = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.POINTER(PlanConfigV1), ctypes.c_char_p, ctypes.c_size_t)
_DESTROY = ctypes.CFUNCTYPE(None, ctypes.c_void_p)
_EXECUTE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_char_p, ctypes.c_size_t)
_SCRATCH = ctypes.CFUNCTYPE(ctypes.c_uint64, ctypes.c_void_p)


class LayoutV1(ctypes.Structure):
    _fields_ = [
        ("in_strides", ctypes.c_int64 * 3),
        ("in_distance", ctypes.c_int64),
        ("out_strides", ctypes.c_int64 * 3),
        ("out_distance", ctypes.c_int64),
    ]


class GroupItemV1(ctypes.Structure):
    _fields_ = [
        ("in_", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("batch", ctypes.c_uint64),
        ("direction", ctypes.c_int32),
        ("normalization", ctypes.c_uint32),
    ]


class FamilyItemV1(ctypes.Structure):
    _fields_ = [
        ("in_", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("n", ctypes.c_uint64),
        ("batch", ctypes.c_uint64),
        ("direction", ctypes.c_int32),
        ("normalization", ctypes.c_uint32),
    ]


class ExecItemV1(ctypes.Structure):
    _fields_ = [
        ("plan", ctypes.c_void_p),
        ("in_", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("batch", ctypes.c_uint64),
        ("direction", ctypes.c_int32),
        ("normalization", ctypes.c_int32),
    ]


class FillItemV1(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("count", ctypes.c_uint64),
        ("seed", ctypes.c_uint64),
        ("scalar", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


class HostStageV1(ctypes.Structure):
    _fields_ = [
        ("plan", ctypes.c_void_p),
        ("direction", ctypes.c_int32),
        ("normalization", ctypes.c_int32),
    ]


class ProviderV1(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32),
        ("name", ctypes.c_char_p),
        ("supports", _SUPPORTS),
        ("create", _CREATE),
        ("destroy", _DESTROY),
        ("execute", _EXECUTE),
        ("scratch_bytes", _SCRATCH),
    ]


# Every symbol include/syclfft_b200_provider.h declares.
EXPORTED_SYMBOLS = (
    "syclfft_b200_get_provider_v1",
    "syclfft_b200_describe_plan",
    "syclfft_b200_plan_launches",
    "syclfft_b200_version",
    "syclfft_b200_plan_status",
    "syclfft_b200_plan_device_bytes",
    "syclfft_b200_plan_take_status",
    "syclfft_b200_plan_set_wait_limit",
    "syclfft_b200_execute_host",
    "syclfft_b200_create_ex",
    "syclfft_b200_execute_batch",
    "syclfft_b200_execute_ex",
    "syclfft_b200_group_supports",
    "syclfft_b200_group_create",
    "syclfft_b200_group_execute",
    "syclfft_b200_group_destroy",
    "syclfft_b200_execute_noalloc_c2c_f32",
    "syclfft_b200_family_supports",
    "syclfft_b200_family_create",
    "syclfft_b200_family_execute",
    "syclfft_b200_execute_many",
    "syclfft_b200_fill_uniform",
    "syclfft_b200_release_stream_scratch",
    "syclfft_b200_family_destroy",
    "syclfft_b200_create_real",
    "syclfft_b200_create_strided",
)

_lib = None


def load(path: str | None = None):
    """dlopen the provider module (RTLD_LOCAL, like provider_loader.cpp:209) and bind its symbols."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or PROVIDER_PATH
    if not os.path.exists(p):
        raise OSError(f"B200 provider module not built: {p}")
    lib = ctypes.CDLL(p, mode=ctypes.RTLD_LOCAL)
    lib.syclfft_b200_get_provider_v1.restype = ctypes.POINTER(ProviderV1)
    lib.syclfft_b200_get_provider_v1.argtypes = []
    lib.syclfft_b200_describe_plan.restype = ctypes.c_int
    lib.syclfft_b200_describe_plan.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_plan_launches.restype = ctypes.c_int
    lib.syclfft_b200_plan_launches.argtypes = [ctypes.c_void_p]
    lib.syclfft_b200_version.restype = ctypes.c_char_p
    lib.syclfft_b200_version.argtypes = []
    lib.syclfft_b200_execute_batch.restype = ctypes.c_int
    lib.syclfft_b200_execute_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                               ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_create_ex.restype = ctypes.c_void_p
    lib.syclfft_b200_create_ex.argtypes = [ctypes.POINTER(PlanConfigV1), ctypes.c_uint32, ctypes.c_char_p,
                                           ctypes.c_size_t]
    lib.syclfft_b200_execute_ex.restype = ctypes.c_int
    lib.syclfft_b200_execute_ex.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_char_p,
                                            ctypes.c_size_t]
    lib.syclfft_b200_plan_device_bytes.restype = ctypes.c_uint64
    lib.syclfft_b200_plan_device_bytes.argtypes = [ctypes.c_void_p]
    lib.syclfft_b200_plan_status.restype = ctypes.c_int
    lib.syclfft_b200_plan_status.argtypes = [ctypes.c_void_p]
    lib.syclfft_b200_plan_take_status.restype = ctypes.c_int
    lib.syclfft_b200_plan_take_status.argtypes = [ctypes.c_void_p]
    lib.syclfft_b200_plan_set_wait_limit.restype = ctypes.c_int
    lib.syclfft_b200_plan_set_wait_limit.argtypes = [ctypes.c_void_p, ctypes.c_int64]
    lib.syclfft_b200_execute_host.restype = ctypes.c_int
    lib.syclfft_b200_execute_host.argtypes = [ctypes.POINTER(HostStageV1), ctypes.c_uint32, ctypes.c_void_p,
                                              ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_char_p,
                                              ctypes.c_size_t]
    lib.syclfft_b200_group_supports.restype = ctypes.c_int
    lib.syclfft_b200_group_supports.argtypes = [ctypes.c_uint32, ctypes.c_uint64]
    lib.syclfft_b200_group_create.restype = ctypes.c_void_p
    lib.syclfft_b200_group_create.argtypes = [ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int32, ctypes.c_char_p,
                                              ctypes.c_size_t]
    lib.syclfft_b200_group_execute.restype = ctypes.c_int
    lib.syclfft_b200_group_execute.argtypes = [ctypes.c_void_p, ctypes.POINTER(GroupItemV1), ctypes.c_uint32,
                                               ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_family_supports.restype = ctypes.c_int
    lib.syclfft_b200_family_supports.argtypes = [ctypes.c_uint32, ctypes.c_uint64]
    lib.syclfft_b200_family_create.restype = ctypes.c_void_p
    lib.syclfft_b200_family_create.argtypes = [ctypes.c_uint32, ctypes.c_int32, ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_family_execute.restype = ctypes.c_int
    lib.syclfft_b200_family_execute.argtypes = [ctypes.c_void_p, ctypes.POINTER(FamilyItemV1), ctypes.c_uint32,
                                                ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_execute_many.restype = ctypes.c_int
    lib.syclfft_b200_execute_many.argtypes = [ctypes.POINTER(ExecItemV1), ctypes.c_uint32, ctypes.c_void_p,
                                              ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_release_stream_scratch.restype = None
    lib.syclfft_b200_release_stream_scratch.argtypes = [ctypes.c_void_p, ctypes.c_int32]
    lib.syclfft_b200_fill_uniform.restype = ctypes.c_int
    lib.syclfft_b200_fill_uniform.argtypes = [ctypes.POINTER(FillItemV1), ctypes.c_uint32, ctypes.c_void_p,
                                              ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_family_destroy.restype = None
    lib.syclfft_b200_family_destroy.argtypes = [ctypes.c_void_p]
    lib.syclfft_b200_group_destroy.restype = None
    lib.syclfft_b200_group_destroy.argtypes = [ctypes.c_void_p]
    lib.syclfft_b200_create_real.restype = ctypes.c_void_p
    lib.syclfft_b200_create_real.argtypes = [ctypes.POINTER(PlanConfigV1), ctypes.c_int32, ctypes.c_uint32,
                                             ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_create_strided.restype = ctypes.c_void_p
    lib.syclfft_b200_create_strided.argtypes = [ctypes.POINTER(PlanConfigV1), ctypes.POINTER(LayoutV1), ctypes.c_uint32,
                                                ctypes.c_char_p, ctypes.c_size_t]
    lib.syclfft_b200_execute_noalloc_c2c_f32.restype = ctypes.c_int
    lib.syclfft_b200_execute_noalloc_c2c_f32.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                                         ctypes.c_uint64, ctypes.c_int32, ctypes.c_uint32,
                                                         ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    if path is None:
        _lib = lib
    return lib


def provider(lib=None):
    lib = lib or load()
    api = lib.syclfft_b200_get_provider_v1()
    if not api:
        raise RuntimeError("syclfft_b200_get_provider_v1 returned NULL")
    return api.contents


def make_config(lengths, batch, direction, double=False, in_place=False, normalization=0, measure=False,
                device=-1) -> PlanConfigV1:
    lengths = [int(v) for v in lengths]
    cfg = PlanConfigV1()
    cfg.abi_version = ABI_VERSION
    cfg.scalar = SCALAR_DOUBLE if double else SCALAR_FLOAT
    cfg.direction = int(direction)
    cfg.rank = len(lengths)
    for i in range(3):
        cfg.lengths[i] = lengths[i] if i < len(lengths) else 0
    cfg.batch_count = int(batch)
    cfg.in_place = 1 if in_place else 0
    cfg.normalization = int(normalization)
    cfg.measure = 1 if measure else 0
    cfg.device = int(device)
    return cfg
