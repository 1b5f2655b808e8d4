"""Generate the golden known-answer fixtures of the reference's own tests.

The reference (Vaskozlov/sycl-fft) pins its portable provider with direct-DFT
known-answer tests. This script restates those cases -- the same sizes,
directions, normalizations, placements and closed-form inputs -- and stores the
inputs and the exact (float64 direct DFT) expected outputs in golden.npz:

  tests/sycl_tests.cpp:91-112   direct_dft (the 1-D oracle)
  tests/sycl_tests.cpp:115-151  reference_many (per-axis direct DFT, multi-dim)
  tests/sycl_tests.cpp:154-193  run_many inputs ((i*11+2)%17)/8, ((i*3+1)%13)/7, tol 8e-4 float
  tests/sycl_tests.cpp:196-262  run_1d inputs ((i*5+1)%9)/4, ((i*3+2)%7)/5, tol 4e-4 float / 2e-11 double
  tests/sycl_tests.cpp:318-365  1-D and multi-dim case list
  tests/sycl_tests.cpp:367-399  N=13 float round trip, input (i/7, (i%3)/5), tol 2e-3 absolute
  tests/sycl_tests.cpp:410-435  two concurrent impulse plans
  tests/sycl_tests.cpp:483-506  event-span dependency: impulse -> all ones
  tests/host_tests.cpp:84-131   run_case inputs ((i*7)%13)/7, ((i*5+3)%11)/9, tol 2e-4 / 1e-11
  tests/host_tests.cpp:133-165  host case list and the N=13 double round trip

Run: python tests/golden/make_golden.py   (writes tests/golden/golden.npz)
"""
from __future__ import annotations

import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

NORM = ["none", "forward", "backward", "orthogonal"]


def norm_scale(norm: str, direction: int, n: int) -> float:
    # src/core/provider_loader.cpp:134-147
    if norm == "none":
        return 1.0
    if norm == "forward":
        return 1.0 / n if direction == -1 else 1.0
    if norm == "backward":
        return 1.0 / n if direction == 1 else 1.0
    return 1.0 / np.sqrt(n)


def direct_axis(x: np.ndarray, shape, batch: int, axis: int, direction: int) -> np.ndarray:
    """Exact per-axis DFT in float64 (the reference's direct oracle, in higher precision)."""
    a = x.reshape([batch] + list(shape)).astype(np.complex128)
    n = shape[axis]
    k = np.arange(n)
    w = np.exp(direction * 2j * np.pi * np.outer(k, k) / n)
    return np.moveaxis(np.tensordot(w, np.moveaxis(a, axis + 1, 0), axes=(1, 0)), 0, axis + 1).reshape(-1)


def expected(x, shape, batch, direction, norm):
    y = x.astype(np.complex128)
    for ax in range(len(shape)):
        y = direct_axis(y, shape, batch, ax, direction)
    return y * norm_scale(norm, direction, int(np.prod(shape)))


def input_1d(n):  # sycl_tests.cpp:202-205
    i = np.arange(n)
    return ((i * 5 + 1) % 9) / 4.0 + 1j * (((i * 3 + 2) % 7) / 5.0)


def input_many(n):  # sycl_tests.cpp:162-165
    i = np.arange(n)
    return ((i * 11 + 2) % 17) / 8.0 + 1j * (((i * 3 + 1) % 13) / 7.0)


def input_host(n):  # host_tests.cpp:95-97
    i = np.arange(n)
    return ((i * 7) % 13) / 7.0 + 1j * (((i * 5 + 3) % 11) / 9.0)


def cases():
    out = []

    def add(name, shape, batch, direction, norm, placement, double, tol, src, x):
        out.append(dict(name=name, shape=list(shape), batch=batch, direction=direction, norm=norm,
                        placement=placement, double=double, tol=tol, source=src, x=x))

    for norm in NORM:  # sycl_tests.cpp:318-325
        add(f"sycl_1d_n8_fwd_{norm}", [8], 1, -1, norm, "out_of_place", False, 4e-4,
            "tests/sycl_tests.cpp:318-325", input_1d(8))
    add("sycl_1d_n7_bwd_inplace", [7], 1, 1, "none", "in_place", False, 4e-4,
        "tests/sycl_tests.cpp:326-331", input_1d(7))
    add("sycl_1d_n6_fwd", [6], 1, -1, "none", "out_of_place", False, 4e-4,
        "tests/sycl_tests.cpp:332-337", input_1d(6))
    add("sycl_1d_n15_bwd", [15], 1, 1, "none", "out_of_place", False, 4e-4,
        "tests/sycl_tests.cpp:338-343", input_1d(15))
    add("sycl_1d_n35_fwd", [35], 1, -1, "none", "out_of_place", False, 4e-4,
        "tests/sycl_tests.cpp:344-349", input_1d(35))
    add("sycl_1d_n11_bwd_inplace", [11], 1, 1, "none", "in_place", False, 4e-4,
        "tests/sycl_tests.cpp:350-355", input_1d(11))
    add("sycl_many_3x4_b2", [3, 4], 2, -1, "none", "out_of_place", False, 8e-4,
        "tests/sycl_tests.cpp:356", input_many(24))
    add("sycl_many_2x3x5", [2, 3, 5], 1, -1, "none", "out_of_place", False, 8e-4,
        "tests/sycl_tests.cpp:357", input_many(30))
    add("sycl_many_11x3", [11, 3], 1, -1, "none", "out_of_place", False, 8e-4,
        "tests/sycl_tests.cpp:358", input_many(33))
    add("sycl_1d_n11_double_ortho", [11], 1, -1, "orthogonal", "out_of_place", True, 2e-11,
        "tests/sycl_tests.cpp:359-365", input_1d(11))
    for norm in NORM:  # host_tests.cpp:133-148
        add(f"host_8_b2_fwd_{norm}", [8], 2, -1, norm, "out_of_place", False, 2e-4,
            "tests/host_tests.cpp:139-140", input_host(16))
        add(f"host_3x5_double_bwd_inplace_{norm}", [3, 5], 1, 1, norm, "in_place", True, 1e-11,
            "tests/host_tests.cpp:141-142", input_host(15))
    add("host_2x3x4_b2_bwd", [2, 3, 4], 2, 1, "none", "out_of_place", False, 2e-4,
        "tests/host_tests.cpp:144-148", input_host(48))
    for c in out:
        c["y"] = expected(c["x"], c["shape"], c["batch"], c["direction"], c["norm"])
    return out


def main():
    cs = cases()
    arrays = {}
    meta = []
    for c in cs:
        arrays[c["name"] + "__x"] = c["x"].astype(np.complex128)
        arrays[c["name"] + "__y"] = c["y"].astype(np.complex128)
        meta.append({k: c[k] for k in ("name", "shape", "batch", "direction", "norm", "placement",
                                       "double", "tol", "source")})
    # N=13 round trips (sycl_tests.cpp:372-399 float; host_tests.cpp:150-165 double)
    i = np.arange(13)
    arrays["roundtrip13__x"] = (i / 7.0 + 1j * ((i % 3) / 5.0)).astype(np.complex128)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"cases": meta,
                   "roundtrip13": {"source": ["tests/sycl_tests.cpp:372-399",
                                              "tests/host_tests.cpp:150-165"],
                                   "tol_float_abs": 2e-3, "tol_double": 2e-11}},
                  f, indent=1)
    print(f"wrote {len(meta)} cases")


if __name__ == "__main__":
    main()
