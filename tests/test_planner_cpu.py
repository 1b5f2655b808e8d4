"""Host-side checks of the provider's building blocks, no GPU needed:
register butterflies vs a direct DFT, and every plan decomposition (single pass,
four-step, fused and three-pass Bluestein, strided axes, copy) run through the FP64
pass emulator against numpy's FP64 FFT."""
import os

import numpy as np
import pytest

from conftest import fp64_fft, gaussian_complex, norm_scale, rel_l2
from native_libs import butterfly, emulate, twiddle_powers


@pytest.mark.parametrize("radix", [1, 2, 3, 4, 5, 7, 8, 15, 16])
def test_butterflies_fp64(radix):
    x = gaussian_complex(radix, radix, np.complex128)
    assert np.max(np.abs(butterfly(radix, x) - np.fft.fft(x))) < 1e-14 * max(1, radix)


@pytest.mark.parametrize("radix", [2, 3, 4, 5, 7, 8, 15, 16])
def test_butterflies_fp32(radix):
    x = gaussian_complex(radix, radix + 100, np.complex128)
    assert np.max(np.abs(butterfly(radix, x, double=False) - np.fft.fft(x))) < 2e-6 * radix


@pytest.mark.parametrize("mode", [0])
@pytest.mark.parametrize("radix", [2, 3, 4, 5, 7, 8, 16])
def test_twiddle_powers(mode, radix):
    """The size-specialised kernels form a butterfly's twiddles from one base twiddle
    W_(Ns*R)^jm by a balanced product tree: u[r] * w^r, exact in FP64 up to rounding and within
    a few float roundings in FP32."""
    rng = np.random.default_rng(radix + 10 * mode)
    for ns in (7, 45, 1024):
        for jm in (0, 1, ns - 1, int(rng.integers(0, ns))):
            w = np.exp(-2j * np.pi * jm / (ns * radix))
            x = gaussian_complex(radix, radix + 7 * jm, np.complex128)
            want = x * w ** np.arange(radix)
            got = twiddle_powers(mode, radix, w, x)
            assert np.max(np.abs(got - want)) < 1e-14 * np.max(np.abs(x)), (ns, jm)
            w32 = np.complex64(w)
            got32 = twiddle_powers(mode, radix, w32, x, double=False)
            assert np.max(np.abs(got32 - want)) < 1e-6 * np.max(np.abs(x)), (ns, jm)


SHAPES = [
    ([8], 2), ([1024], 3), ([4096], 2), ([13440], 1), ([16384], 1), ([11], 3), ([1009], 2), ([4099], 1),
    ([16, 12, 10], 2), ([11, 3], 1), ([3, 4], 2), ([2, 3, 5], 1), ([1], 5), ([1, 1], 2), ([32768], 2),
    ([65536], 1), ([65537], 1), ([30000], 2), ([64, 2048], 1), ([3, 40000], 1), ([40000, 3], 1),
    ([65537, 2], 1), ([257, 5], 2), ([7, 1, 9], 3), ([2048, 2048 // 64], 1), ([131072], 1), ([65536, 3], 1),
]


@pytest.mark.parametrize("double", [False, True])
@pytest.mark.parametrize("shape,batch", SHAPES, ids=lambda v: str(v))
def test_plan_decompositions_emulated(shape, batch, double):
    n = int(np.prod(shape))
    x = gaussian_complex(n * batch, n + batch, np.complex128)
    for d, norm in ((-1, 3), (1, 2)):
        y, desc = emulate(x, shape, batch, d, norm, double)
        ref = fp64_fft(x, shape, batch, d, norm_scale(norm, d, n))
        assert rel_l2(y, ref) < 1e-13, desc


def test_plan_kinds():
    _, d = emulate(np.zeros(4096 * 2), [4096], 2, -1)
    assert [p["kind"] for p in d["passes"]] == ["single"]
    _, d = emulate(np.zeros(65536), [65536], 1, -1, double=True)
    assert [p["kind"] for p in d["passes"]] == ["fourstep_cols", "fourstep_rows"]
    assert all(p["fixed_id"] >= 0 for p in d["passes"])
    _, d = emulate(np.zeros(2 * 65536), [65536, 2], 1, -1, double=True)
    assert [p["kind"] for p in d["passes"]][1:] == ["fourstep_cols", "fourstep_rows"]
    _, d = emulate(np.zeros(1009), [1009], 1, -1)
    assert [p["kind"] for p in d["passes"]] == ["bluestein_fused"]
    _, d = emulate(np.zeros(65537), [65537], 1, -1)  # prime, 65536 = 256 x 256: Rader
    assert [p["kind"] for p in d["passes"]] == ["rader_cols_fwd", "rader_rows_conv", "rader_cols_inv"]
    assert d["scratch_elements"] == 65536
    _, d = emulate(np.zeros(65539), [65539], 1, -1)  # prime, 65538 = 2 * 3 * 29 * 113: Bluestein
    assert [p["kind"] for p in d["passes"]] == ["bluestein_cols_fwd", "bluestein_rows_conv", "bluestein_cols_inv"]
    assert d["scratch_elements"] >= 2 * 65539 - 2


def test_in_place_emulated():
    x = gaussian_complex(3 * 40000, 5, np.complex128)
    y, _ = emulate(x, [40000], 3, -1, 0, False, in_place=True)
    assert rel_l2(y, fp64_fft(x, [40000], 3, -1)) < 1e-13


def test_small_smem_limit_forces_fourstep():
    x = gaussian_complex(4096, 9, np.complex128)
    y, d = emulate(x, [4096], 1, -1, smem_limit=16 * 1024)
    assert d["passes"][0]["kind"] == "fourstep_cols"
    assert rel_l2(y, fp64_fft(x, [4096], 1, -1)) < 1e-13


def test_split_precision_pass_selection():
    """The tensor-core kernels replace plain single passes of float plans whose axis length
    has one (256, 4096 contiguous; 256 strided); everything else keeps its FP32/FP64 pass."""
    from native_libs import describe

    def tc(shape, batch, double=False, split=True):
        return [p["tc_id"] for p in describe(shape, batch, double=double, split_bf16=split)["passes"]]

    assert tc([256], 64) == [0]
    assert tc([4096], 8) == [2]
    assert tc([256, 256, 256], 1) == [0, 1, 1]        # last axis contiguous, then strided columns
    assert tc([4096, 4096], 1)[0] == 2 and all(t < 0 for t in tc([4096, 4096], 1)[1:])
    assert all(t < 0 for t in tc([256], 64, double=True))    # double plans stay FP64
    assert all(t < 0 for t in tc([256], 64, split=False))    # opt-in only
    assert all(t < 0 for t in tc([1009], 8))                 # Bluestein passes stay FP32
    assert all(t < 0 for t in tc([13440], 8))                # no tensor-core kernel for this length


def test_bluestein_on_catalog_kernels():
    """Contiguous Bluestein axes take the smallest catalog convolution length >= 2L - 2: one
    fused pass where it fits a CTA, else three passes over M = n1 * n2; strided axes and
    the generic-kernel switch keep the runtime-parameterised passes."""
    from native_libs import describe, emulate

    def kinds(shape, dbl=False, batch=2):
        d = describe(shape, batch, double=dbl)
        return [(p["kind"], p["n"], p["blue_id"] >= 0) for p in d["passes"]]

    assert kinds([1009]) == [("bluestein_fused", 2048, True)]
    assert kinds([4099]) == [("bluestein_fused", 10240, True)]
    os.environ["SYCLFFT_B200_RADER"] = "0"  # 65537 is a Rader length; Bluestein on request
    try:
        k = kinds([65537])
    finally:
        del os.environ["SYCLFFT_B200_RADER"]
    assert [x[0] for x in k] == ["bluestein_cols_fwd", "bluestein_rows_conv", "bluestein_cols_inv"]
    assert all(x[2] for x in k) and k[0][1] * k[1][1] == 2 * 65537 - 2  # M = 2L - 2 = 2^17
    assert all(x[2] for x in kinds([4099], dbl=True))
    assert not any(x[2] for x in kinds([1009, 6]))           # strided prime axis: generic passes
    rng = np.random.default_rng(9)
    for shape, dbl in (([1009], False), ([4099], True), ([12289], False)):
        n = int(np.prod(shape))
        x = rng.standard_normal(2 * n) + 1j * rng.standard_normal(2 * n)
        out, _ = emulate(x, shape, 2, -1, norm=1, double=dbl)
        ref = np.fft.fft(x.reshape(2, n), axis=1).reshape(-1) / n
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-13


@pytest.mark.parametrize("shape,batch,dbl,kinds", [
    ([257], 3, False, ["rader_fused"]),
    ([641], 2, True, ["rader_fused"]),
    ([12289], 2, False, ["rader_fused"]),
    ([12289], 2, True, ["rader_cols_fwd", "rader_rows_conv", "rader_cols_inv"]),
    ([65537], 2, False, ["rader_cols_fwd", "rader_rows_conv", "rader_cols_inv"]),
    ([65537], 1, True, ["rader_cols_fwd", "rader_rows_conv", "rader_cols_inv"]),
    ([5, 257], 2, False, ["rader_fused", "single"]),
    ([257, 6], 1, False, ["single", "generic_or_bluestein"]),
    ([7681], 1, False, ["bluestein_fused"]),
])
def test_rader_plans_emulated(shape, batch, dbl, kinds, monkeypatch):
    """Prime lengths L whose L - 1 the Bluestein catalog covers run Rader's algorithm on the
    catalog kernels (gather through generator powers, length-(L-1) convolution with the x[0]
    term at bin 0, scatter); the FP64 emulation of those passes is the DFT in both directions,
    for every normalization, in place and out of place. Strided prime axes and primes whose
    L - 1 is not a catalog length (7680 = 2^9 * 15) stay on Bluestein."""
    from native_libs import describe
    d = describe(shape, batch, double=dbl)
    got = [p["kind"] for p in d["passes"]]
    if kinds[-1] == "generic_or_bluestein":
        assert got[0] == "single" and not any(k.startswith("rader") for k in got)
    else:
        assert got == kinds
    assert all(p["rader"] == p["kind"].startswith("rader") for p in d["passes"])
    n = int(np.prod(shape))
    rng = np.random.default_rng(n + batch)
    x = rng.standard_normal(n * batch) + 1j * rng.standard_normal(n * batch)
    for direction, norm, ip in ((-1, 0, False), (1, 2, True), (-1, 3, True), (1, 1, False)):
        out, _ = emulate(x, shape, batch, direction, norm=norm, double=dbl, in_place=ip)
        ref = fp64_fft(x, shape, batch, direction, norm_scale(norm, direction, n))
        assert rel_l2(out, ref) < 1e-13, (direction, norm, ip)
    # the same plan on Bluestein's convolution agrees
    monkeypatch.setenv("SYCLFFT_B200_RADER", "0")
    out_b, d_b = emulate(x, shape, batch, -1, double=dbl)
    assert not any(p["rader"] for p in d_b["passes"])
    assert rel_l2(out_b, fp64_fft(x, shape, batch, -1, 1.0)) < 1e-13


def test_primitive_roots():
    """The generator the Rader tables are built from: its powers run through every residue."""
    from native_libs import primitive_root
    for p in (3, 5, 7, 257, 641, 12289, 65537, 786433):
        g = primitive_root(p)
        seen, v = set(), 1
        for _ in range(p - 1):
            seen.add(v)
            v = v * g % p
        assert len(seen) == p - 1 and v == 1, p


def test_fused_single_routes_13440_through_a_catalogued_split(monkeypatch):
    """With SYCLFFT_B200_FUSED4_SINGLE=1 a length that fits one block but has a fused four-step
    kernel (13440 = 112 x 120) is planned as that four-step, on the catalog's radix sequences
    (16, 7) and (8, 15); the FP64 emulation of its passes is the DFT. Without it the single pass
    stays."""
    import numpy as np
    import native_libs as nl
    n, b = 13440, 3
    x = np.random.default_rng(3).standard_normal(n * b) + 1j * np.random.default_rng(4).standard_normal(n * b)
    out, desc = nl.emulate(x, [n], b, -1)
    assert [p["kind"] for p in desc["passes"]] == ["single"]
    monkeypatch.setenv("SYCLFFT_B200_FUSED4_SINGLE", "1")
    out, desc = nl.emulate(x, [n], b, -1)
    assert [(p["kind"], p["radices"]) for p in desc["passes"]] == [("fourstep_cols", [16, 7]),
                                                                    ("fourstep_rows", [8, 15])]
    ref = np.fft.fft(x.reshape(b, n), axis=1).reshape(-1)
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-14


def test_lean_passes_marked():
    """Runtime-length passes over contiguous lines (whole lines, and the column and row passes of
    a contiguous four-step) run on the lean kernel; strided axes, size-specialised, Bluestein and
    single-stage passes do not. The lean kernel has the general kernel's semantics (plus the
    radix-15 stage), so the FP64 emulation of these plans (the SHAPES cases above) covers them."""
    from native_libs import describe

    def lean(shape, dbl=False):
        return [(p["kind"], p["lean"]) for p in describe(shape, 4, double=dbl)["passes"]]

    assert lean([3000]) == [("single", 1)]
    assert lean([680400]) == [("fourstep_cols", 1), ("fourstep_rows", 1)]
    assert lean([784000], True) == [("fourstep_cols", 1), ("fourstep_rows", 1)]
    assert lean([3000, 6]) == [("single", 1), ("single", 0)]  # the strided axis stays general
    assert lean([4096]) == [("single", 0)]                     # size-specialised
    assert lean([1009]) == [("bluestein_fused", 0)]
    for p in describe([680400], 4)["passes"]:
        assert p["w"] & (p["w"] - 1) == 0 and len(p["radices"]) >= 2


def test_lean_radix15_stages():
    """Float lean passes run each (3, 5) pair of stages as one radix-15 stage (a radix-3, -5 or
    -15 stage all need n / 15 threads per line at 16 values a thread, so the tile is the same);
    double lean passes (8 values a thread) keep 3 and 5; a pass is never fused down to a single
    stage, and the order stays 16, 8, 4, 2, 15, 3, 5, 7."""
    from native_libs import describe

    def first(n, dbl=False):
        p = describe([n], 4, double=dbl)["passes"][0]
        return p["lean"], p["radices"], p["threads"]

    assert first(3000) == (1, [8, 15, 5, 5], 224)
    assert first(810)[1] == [2, 15, 3, 3, 3]
    assert first(1125)[1] == [15, 15, 5]
    assert first(105)[1] == [15, 7]
    assert first(15)[1] == [3, 5]                      # one radix-15 stage would be a single stage
    assert first(840, True)[1] == [8, 3, 5, 7]         # double: no radix 15
    assert first(2187)[1] == [3] * 7                    # no 5 to pair with
    order = [16, 8, 4, 2, 15, 3, 5, 7]
    for n in (810, 1125, 3000, 12000, 6125, 30000, 680400):
        for p in describe([n], 2)["passes"]:
            if p["lean"]:
                pos = [order.index(r) for r in p["radices"]]
                assert pos == sorted(pos), (n, p["radices"])
