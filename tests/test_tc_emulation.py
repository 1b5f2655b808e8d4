"""CPU restatement of the split-precision tensor-core pass (sycl-fft_b200/csrc/tc_kernel.cuh).

The kernel's bookkeeping is restated in numpy row by row: the Stockham butterfly rows
(line l, butterfly j), the padded exchange buffer (index i stored at i + i // R, line pitch
N + N/R + 1), the twiddle exponent e = r * (j mod ns) * N / (ns * R) of W_N^e, the real
2R x 2R DFT matrix, the two-level twiddle product hi[e >> 6] * lo[e & 63], the BF16 hi/lo splitting and the three products hi*hi + hi*lo + lo*hi.
Products are summed in FP64 and rounded to FP32 (the tensor core accumulates in FP32, so
its error can only be a little larger). The tests pin the index arithmetic against FP64
FFTs and give the error level the GPU tests then hold the kernel to.
"""
import math

import numpy as np
import pytest


def bf16(x):
    """float32 -> nearest BF16 (ties to even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def split(x):
    hi = bf16(x)
    lo = bf16((np.asarray(x, np.float32) - hi).astype(np.float32))
    return hi, lo


def dft_real(R):
    """Rows: outputs [re, im] interleaved; columns: inputs [re, im] interleaved."""
    m = np.arange(R)[:, None]
    n = np.arange(R)[None, :]
    ang = -2.0 * np.pi * ((m * n) % R) / R
    c = np.cos(ang).astype(np.float32)
    s = np.sin(ang).astype(np.float32)
    B = np.zeros((2 * R, 2 * R), np.float32)
    B[0::2, 0::2] = c
    B[0::2, 1::2] = -s
    B[1::2, 0::2] = s
    B[1::2, 1::2] = c
    return B


def tc_lines(x, R, S, products=3):
    """Forward FFT of each row of x (complex64, shape (L, R**S)) as the kernel computes it."""
    L, N = x.shape
    assert N == R ** S
    NB = N // R
    pitch = N + N // R + 1
    Bh, Bl = split(dft_real(R))
    tw_hi = np.exp(-2j * np.pi * 64 * np.arange((N + 63) // 64) / N).astype(np.complex64)
    tw_lo = np.exp(-2j * np.pi * np.arange(64) / N).astype(np.complex64)
    z = np.zeros((L, pitch), np.complex64)
    out = np.zeros((L, N), np.complex64)
    l_idx, j_idx = (a.ravel() for a in np.meshgrid(np.arange(L), np.arange(NB), indexing="ij"))
    r = np.arange(R)
    for s in range(S):
        ns = R ** s
        jm = j_idx % ns
        idx = j_idx[:, None] + r[None, :] * NB
        if s == 0:
            v = x[l_idx[:, None], idx]
        else:
            v = z[l_idx[:, None], idx + idx // R]
            e = r[None, :] * jm[:, None] * (N // (ns * R))
            h, q = tw_hi[e >> 6], tw_lo[e & 63]
            w = ((h.real * q.real - h.imag * q.imag).astype(np.float32)
                 + 1j * (h.real * q.imag + h.imag * q.real).astype(np.float32)).astype(np.complex64)
            re = (v.real * w.real - v.imag * w.imag).astype(np.float32)
            im = (v.real * w.imag + v.imag * w.real).astype(np.float32)
            v = (re + 1j * im).astype(np.complex64)
        A = np.empty((v.shape[0], 2 * R), np.float32)
        A[:, 0::2] = v.real
        A[:, 1::2] = v.imag
        Ah, Al = split(A)
        f64 = np.float64
        D = Ah.astype(f64) @ Bh.T.astype(f64) + Ah.astype(f64) @ Bl.T.astype(f64) + Al.astype(f64) @ Bh.T.astype(f64)
        if products == 4:
            D += Al.astype(f64) @ Bl.T.astype(f64)
        D = D.astype(np.float32)
        y = (D[:, 0::2] + 1j * D[:, 1::2]).astype(np.complex64)  # (rows, R): output m
        m = np.arange(R)[None, :]
        if s + 1 < S:
            oidx = (j_idx - jm)[:, None] * R + jm[:, None] + m * ns
            z[l_idx[:, None], oidx + oidx // R] = y
        else:
            out[l_idx[:, None], j_idx[:, None] + m * NB] = y
    return out


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("R,S,L", [(16, 2, 16), (16, 3, 1), (4, 2, 3), (8, 3, 2)])
def test_tc_restatement_matches_fp64(R, S, L):
    N = R ** S
    rng = np.random.default_rng(N + L)
    x = (rng.uniform(-1, 1, (L, N)) + 1j * rng.uniform(-1, 1, (L, N))).astype(np.complex64)
    got = tc_lines(x, R, S)
    ref = np.fft.fft(x.astype(np.complex128), axis=1)
    err = rel_l2(got, ref)
    # BF16 hi + lo keeps 16 bits: about 2^-17 relative per operand, a few 1e-6 per stage
    assert err < 1e-5 * max(1.0, math.log2(N)), err
    assert err < 2e-5, err


def test_tc_error_level_and_lo_lo_term():
    """The dropped lo*lo product changes the error by far less than the error itself."""
    R, S = 16, 2
    rng = np.random.default_rng(7)
    x = (rng.uniform(-1, 1, (8, 256)) + 1j * rng.uniform(-1, 1, (8, 256))).astype(np.complex64)
    ref = np.fft.fft(x.astype(np.complex128), axis=1)
    e3 = rel_l2(tc_lines(x, R, S, products=3), ref)
    e4 = rel_l2(tc_lines(x, R, S, products=4), ref)
    assert e3 < 1e-5 and e4 < 1e-5
    assert abs(e3 - e4) < 0.5 * e3


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.14159, 1e-30], np.float32)
    h = bf16(x)
    assert h[0] == 1.0 and h[1] == 1.0  # halfway: ties to the even neighbour
    hi, lo = split(x)
    assert np.all(np.abs((hi.astype(np.float64) + lo) - x) <= np.abs(x) * 2.0 ** -16)
