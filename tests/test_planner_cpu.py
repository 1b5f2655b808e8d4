"""Host-side checks of the provider's building blocks, no GPU needed:
register butterflies vs a direct DFT, and every plan decomposition (single pass,
four-step, fused and three-pass Bluestein, strided axes, copy) run through the FP64
pass emulator against numpy's FP64 FFT."""
import numpy as np
import pytest

from conftest import fp64_fft, gaussian_complex, norm_scale, rel_l2
from native_libs import butterfly, emulate


@pytest.mark.parametrize("radix", [1, 2, 3, 4, 5, 7, 8, 15, 16])
def test_butterflies_fp64(radix):
    x = gaussian_complex(radix, radix, np.complex128)
    assert np.max(np.abs(butterfly(radix, x) - np.fft.fft(x))) < 1e-14 * max(1, radix)


@pytest.mark.parametrize("radix", [2, 3, 4, 5, 7, 8, 15, 16])
def test_butterflies_fp32(radix):
    x = gaussian_complex(radix, radix + 100, np.complex128)
    assert np.max(np.abs(butterfly(radix, x, double=False) - np.fft.fft(x))) < 2e-6 * radix


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
    _, d = emulate(np.zeros(65537), [65537], 1, -1)
    assert [p["kind"] for p in d["passes"]] == ["bluestein_cols_fwd", "bluestein_rows_conv", "bluestein_cols_inv"]
    assert d["scratch_elements"] >= 2 * 65537 - 1


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
    """Contiguous Bluestein axes take the smallest catalog convolution length >= 2L - 1: one
    fused pass where it fits a CTA, else three passes over M = n1 * n2; strided axes and
    the generic-kernel switch keep the runtime-parameterised passes."""
    from native_libs import describe, emulate

    def kinds(shape, dbl=False, batch=2):
        d = describe(shape, batch, double=dbl)
        return [(p["kind"], p["n"], p["blue_id"] >= 0) for p in d["passes"]]

    assert kinds([1009]) == [("bluestein_fused", 2048, True)]
    assert kinds([4099]) == [("bluestein_fused", 10240, True)]
    k = kinds([65537])
    assert [x[0] for x in k] == ["bluestein_cols_fwd", "bluestein_rows_conv", "bluestein_cols_inv"]
    assert all(x[2] for x in k) and k[0][1] * k[1][1] >= 2 * 65537 - 1
    assert all(x[2] for x in kinds([4099], dbl=True))
    assert not any(x[2] for x in kinds([1009, 6]))           # strided prime axis: generic passes
    rng = np.random.default_rng(9)
    for shape, dbl in (([1009], False), ([4099], True), ([12289], False)):
        n = int(np.prod(shape))
        x = rng.standard_normal(2 * n) + 1j * rng.standard_normal(2 * n)
        out, _ = emulate(x, shape, 2, -1, norm=1, double=dbl)
        ref = np.fft.fft(x.reshape(2, n), axis=1).reshape(-1) / n
        assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-13


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
