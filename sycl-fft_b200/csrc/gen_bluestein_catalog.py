#!/usr/bin/env python
"""Writes bluestein_catalog.h: the size-specialised Bluestein kernels (fixed_kernel.cuh
features kFeatPremul / kFeatConv / kFeatPostmul) instantiated by bluestein_variants.cu.

Convolution lengths are 2^a * f, f in {1, 3, 5, 7}: a Bluestein axis of length L takes the
smallest catalog length (or product of a column and a row length) >= 2L - 2, so the padding
stays within about 25% of the smallest 7-smooth length while every stage is a large radix.
Run: python gen_bluestein_catalog.py > bluestein_catalog.h
"""
import math

KINDS = {"fused": 0, "cols_fwd": 1, "rows_conv": 2, "cols_inv": 3}


def sizes(lo, hi):
    out = set()
    for f in (1, 3, 5, 7):
        n = f
        while n <= hi:
            if n >= lo:
                out.add(n)
            n *= 2
    return sorted(out)


def radices(n, dbl):
    maxr = 8 if dbl else 16
    f = n
    while f % 2 == 0:
        f //= 2
    p2 = n // f
    rs = []
    while p2 >= maxr:
        rs.append(maxr)
        p2 //= maxr
    if p2 > 1:
        rs.append(p2)
    if f > 1:
        rs.append(f)
    return rs


def tpl(n, rs, dbl):
    maxv = 8 if dbl else 16
    t = 1
    while True:
        if all(math.ceil(n // r / t) * r <= maxv for r in rs):
            return t
        t += 1


def maxt(threads):
    for m in (256, 512, 1024):
        if threads <= m:
            return m
    return None


def entries():
    out = []
    for dbl in (0, 1):
        for n in sizes(64, 8192 if dbl else 16384):
            rs = radices(n, dbl)
            t = tpl(n, rs, dbl)
            if t > 1024:
                continue
            out.append((dbl, "fused", n, t, 1, maxt(t), rs))
        for n in sizes(64, 1024):
            rs = radices(n, dbl)
            t = tpl(n, rs, dbl)
            out.append((dbl, "rows_conv", n, t, 1, maxt(t), rs))
        w = 8 if dbl else 16
        for n in (64, 128, 256, 512, 1024):
            rs = radices(n, dbl)
            t = tpl(n, rs, dbl)
            for kind in ("cols_fwd", "cols_inv"):
                out.append((dbl, kind, n, t, w, maxt(t * w), rs))
    return out


def main():
    print("// Generated by gen_bluestein_catalog.py: size-specialised Bluestein pass kernels.")
    print("//")
    print("// X(ID, DOUBLE, KIND, N, TPL, W, MAXT, RADICES...)")
    print("//   KIND 0 fused single pass (contiguous lines: chirp pre-multiply, FFT_N, spectrum")
    print("//          multiply, inverse FFT_N, chirp post-multiply), 1 column pass of the")
    print("//          zero-padded pre-multiplied line (four-step twiddle on the store), 2 row pass")
    print("//          (FFT, spectrum multiply, inverse FFT, inverse twiddle), 3 inverse column")
    print("//          pass (chirp post-multiply, truncation)")
    print("//   N FFT length, TPL threads per line, W columns per CTA (column passes), MAXT the")
    print("//   CTA-size bound of the instantiation, RADICES the Stockham stages.")
    print("#pragma once")
    print()
    print("#define SFB_BLUESTEIN_CATALOG(X) \\")
    es = entries()
    lines = []
    for i, (dbl, kind, n, t, w, mt, rs) in enumerate(es):
        lines.append(f"    X({i}, {dbl}, {KINDS[kind]}, {n}, {t}, {w}, {mt}, {', '.join(map(str, rs))})")
    print(" \\\n".join(lines))
    print()
    print(f"#define SFB_BLUESTEIN_COUNT {len(es)}")


if __name__ == "__main__":
    main()
