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
