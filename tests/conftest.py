"""Shared test setup: the `gpu` marker, import paths, and seeded input helpers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "sycl-fft_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")


def uniform_complex(n, seed, dtype=np.complex64):
    """re, im ~ U[-1, 1) from a seeded PCG64 generator."""
    rng = np.random.default_rng(seed)
    return (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(dtype)


def gaussian_complex(n, seed, dtype=np.complex64):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(dtype)


def fp64_fft(x, shape, batch, direction, scale=1.0):
    """FP64 oracle: numpy pocketfft in complex128 over the transform axes."""
    a = np.asarray(x, dtype=np.complex128).reshape([batch] + list(shape))
    axes = tuple(range(1, len(shape) + 1))
    n = int(np.prod(shape))
    y = np.fft.fftn(a, axes=axes) if direction == -1 else np.fft.ifftn(a, axes=axes) * n
    return (y * scale).reshape(-1)


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128).reshape(-1)
    b = np.asarray(b, dtype=np.complex128).reshape(-1)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def norm_scale(norm, direction, n):
    if norm == 0:
        return 1.0
    if norm == 1:
        return 1.0 / n if direction == -1 else 1.0
    if norm == 2:
        return 1.0 / n if direction == 1 else 1.0
    return 1.0 / np.sqrt(n)


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import portable
    portable.build()
    return portable
