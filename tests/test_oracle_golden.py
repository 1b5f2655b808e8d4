"""The oracle (CPU restatement of the portable provider) pinned against the
reference's own known-answer tests (tests/golden, generated by make_golden.py from
tests/sycl_tests.cpp and tests/host_tests.cpp of the reference)."""
import json
import os

import numpy as np
import pytest

from conftest import fp64_fft, rel_l2, uniform_complex

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load_cases():
    meta = json.load(open(os.path.join(GOLDEN, "golden.json")))
    return meta["cases"]


@pytest.mark.parametrize("case", load_cases(), ids=lambda c: c["name"])
def test_oracle_matches_reference_known_answers(oracle_mod, case):
    g = np.load(os.path.join(GOLDEN, "golden.npz"))
    x, y = g[case["name"] + "__x"], g[case["name"] + "__y"]
    dt = np.complex128 if case["double"] else np.complex64
    p = oracle_mod.OraclePlan(case["shape"], case["batch"], case["direction"], case["norm"], case["double"])
    out = p.execute(x.astype(dt))
    err = np.abs(out - y)
    # the reference tests' bound: |actual - expected| <= tol * (1 + |expected|)
    assert np.all(err <= case["tol"] * (1 + np.abs(y))), case["source"]


def test_oracle_round_trip_13(oracle_mod):
    # tests/sycl_tests.cpp:372-399 (float, backward normalization) and host_tests.cpp:150-165 (double)
    x = np.load(os.path.join(GOLDEN, "golden.npz"))["roundtrip13__x"]
    for dbl, tol in ((False, 2e-3), (True, 2e-11)):
        dt = np.complex128 if dbl else np.complex64
        spec = oracle_mod.OraclePlan([13], 1, "forward", "none", dbl).execute(x.astype(dt))
        back = oracle_mod.OraclePlan([13], 1, "backward", "backward", dbl).execute(spec)
        assert np.max(np.abs(back - x)) < tol * (1 if not dbl else 1 + np.max(np.abs(x)))


def test_oracle_impulses(oracle_mod):
    # sycl_tests.cpp:410-435 and 483-506: impulse at 0 -> all ones; impulse at 1 -> X[0] = 1
    a = np.zeros(8, np.complex64); a[0] = 1
    b = np.zeros(8, np.complex64); b[1] = 1
    ya = oracle_mod.portable_fft(a, [8], 1, "forward")
    yb = oracle_mod.portable_fft(b, [8], 1, "forward")
    assert np.allclose(ya, 1, atol=1e-5) and abs(yb[0].real - 1) < 1e-5


@pytest.mark.parametrize("shape,batch,dbl", [([1024], 4, False), ([4096], 3, False), ([13440], 1, False),
                                             ([1009], 2, True), ([4099], 1, False), ([16, 12, 10], 2, False),
                                             ([11, 3], 3, True), ([1], 4, False)])
def test_oracle_vs_fp64(oracle_mod, shape, batch, dbl):
    n = int(np.prod(shape))
    dt = np.complex128 if dbl else np.complex64
    x = uniform_complex(n * batch, 7, dt)
    for d in (-1, 1):
        y = oracle_mod.portable_fft(x, shape, batch, d, double=dbl)
        e = rel_l2(y, fp64_fft(x, shape, batch, d))
        # Bluestein float carries the reference's float chirp error (~1e-4 at N=1009, 4e-4 at 4099).
        assert e < (1e-12 if dbl else 1e-3)


def test_oracle_rejects_invalid(oracle_mod):
    with pytest.raises(ValueError):
        oracle_mod.OraclePlan([0], 1, "forward")
    with pytest.raises(ValueError):
        oracle_mod.OraclePlan([2, 2, 2, 2], 1, "forward")
    with pytest.raises(ValueError):
        oracle_mod.OraclePlan([4], 0, "forward")
