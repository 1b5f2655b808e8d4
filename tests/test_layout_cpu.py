"""data_layout on the CPU: extents, the output-overlap test and in-place rules (no device)."""
import pytest

import syclfft_b200 as sf


def test_contiguous_layout():
    lay = sf.data_layout.contiguous([4, 5, 6])
    assert lay.in_strides == (30, 6, 1) and lay.in_distance == 120
    assert lay.extent([4, 5, 6], 3, False) == 360
    lay.check([4, 5, 6], 3, True)


@pytest.mark.parametrize("strides,dist,shape,batch,ok", [
    ((1,), 8, [8], 4, True),
    ((4,), 1, [8], 4, True),          # columns
    ((1,), 4, [8], 4, False),         # rows overlap
    ((2,), 1, [8], 4, False),         # interleave of 2 for 4 signals overlaps
    ((2,), 1, [8], 2, True),
    ((1, 12), 120, [12, 10], 3, True),  # transposed
    ((1, 11), 120, [12, 10], 3, False),
    ((0,), 8, [8], 1, False),
    ((3,), 0, [8], 2, False),
    ((3,), 0, [8], 1, True),          # distance unused for a single transform
])
def test_output_layout_check(strides, dist, shape, batch, ok):
    lay = sf.data_layout(tuple(strides), dist, tuple(strides), dist)
    if ok:
        lay.check(shape, batch, False)
    else:
        with pytest.raises(sf.SyclfftError) as e:
            lay.check(shape, batch, False)
        assert e.value.code == sf.error_code.invalid_argument


def test_extent_and_in_place_rule():
    lay = sf.data_layout((96,), 1, (1,), 4096)
    assert lay.extent([4096], 96, False) == 4095 * 96 + 95 + 1
    assert lay.extent([4096], 96, True) == 4096 * 96
    with pytest.raises(sf.SyclfftError):
        lay.check([4096], 96, True)


@pytest.mark.parametrize("shape,skip,d,norm,in_place", [
    ([64, 24], 0b10, -1, 0, False),        # 64-point transforms down 24 columns
    ([4096, 96], 0b10, 1, 2, True),
    ([1009, 7], 0b10, -1, 1, False),       # Bluestein on a strided axis
    ([12, 10, 3], 0b100, -1, 3, False),    # 2D transforms of 3 interleaved arrays
    ([13440, 3], 0b10, -1, 0, True),
    ([1024, 300], 0b10, 1, 0, False),
])
def test_skipped_axes_on_the_emulator(shape, skip, d, norm, in_place):
    """Plans with untransformed (batch) axes, run pass by pass by the FP64 emulator of the
    planner's kernels, against numpy over the transformed axes only; the normalization scale
    counts transformed axes only."""
    import math
    import numpy as np
    from native_libs import emulate_skip
    rng = np.random.default_rng(sum(shape))
    n_all = math.prod(shape)
    x = rng.uniform(-1, 1, n_all) + 1j * rng.uniform(-1, 1, n_all)
    out, desc = emulate_skip(x, shape, 1, d, skip, norm, False, in_place)
    axes = tuple(a for a in range(len(shape)) if not (skip >> a) & 1)
    n = math.prod(shape[a] for a in axes)
    a = x.reshape(shape)
    ref = np.fft.fftn(a, axes=axes) if d == -1 else np.fft.ifftn(a, axes=axes) * n
    scale = {0: 1.0, 1: 1.0 / n if d == -1 else 1.0, 2: 1.0 / n if d == 1 else 1.0, 3: n ** -0.5}[norm]
    ref = (ref * scale).reshape(-1)
    assert np.linalg.norm(out - ref) / np.linalg.norm(ref) < 1e-12
    assert all(p["axis"] in axes for p in desc["passes"])
