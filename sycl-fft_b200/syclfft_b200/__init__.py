"""syclfft_b200: B200-native FFT provider for the syclfft plan API.

Python mirror of the reference's plan surface (include/syclfft/syclfft.hpp:90-130,
include/syclfft/common.hpp:34-110): ``plan_dft_1d/2d/3d``, ``plan_many_dft``,
``plan_options``, ``plan.execute(...)``, with the same enum values, error codes and
validation rules, running on the B200 provider module through its C ABI. Device
buffers are CUDA torch tensors (complex64 / complex128) or raw device pointers;
execution is ordered on a CUDA stream (the stand-in for the SYCL queue) and returns
a CUDA event (the stand-in for sycl::event).
"""
from .api import (  # noqa: F401
    Plan,
    RealPlan,
    SyclfftError,
    data_layout,
    direction,
    error_code,
    execute_host,
    normalization,
    placement,
    plan_dft_1d,
    plan_dft_2d,
    plan_dft_3d,
    plan_dft_c2r,
    plan_dft_c2r_1d,
    plan_dft_r2c,
    plan_dft_r2c_1d,
    plan_many_dft,
    plan_options,
    planning_mode,
    provider,
    query_providers,
)
from . import _provider  # noqa: F401

__all__ = [
    "Plan", "RealPlan", "SyclfftError", "data_layout", "direction", "error_code", "execute_host", "normalization", "placement", "plan_dft_1d",
    "plan_dft_2d", "plan_dft_3d", "plan_dft_r2c_1d", "plan_dft_c2r_1d", "plan_dft_r2c", "plan_dft_c2r", "plan_many_dft", "plan_options", "planning_mode", "provider",
    "query_providers",
]
