"""Host logic of the batched path (no GPU): the layout offsets that the
batched kernels index with, and the argument checks."""
import pytest

from lig_b200 import _lib
from lig_b200.batch import BatchLayout


def test_offsets_follow_concatenation_order():
    L = BatchLayout([64, 130, 16], [96, 77, 16], [10, 0, 5], 16)
    assert L.g_off == [0, 10, 10, 15]
    assert L.pix_off == [0, 64 * 96, 64 * 96 + 130 * 77, 64 * 96 + 130 * 77 + 256]
    tiles = [(96 // 16) * (64 // 16), 5 * 9, 1]
    assert L.tile_off == [0, tiles[0], tiles[0] + tiles[1], sum(tiles)]
    assert (L.points, L.pixels, L.tiles) == (15, L.pix_off[-1], sum(tiles))
    n, h, w, c = L.args()
    assert n == 3 and h.value and w.value and c.value


@pytest.mark.parametrize("kw", [
    dict(heights=[], widths=[], counts=[]),
    dict(heights=[8] * (_lib.LIG_MAX_BATCH + 1), widths=[8] * (_lib.LIG_MAX_BATCH + 1),
         counts=[1] * (_lib.LIG_MAX_BATCH + 1)),
    dict(heights=[8, 8], widths=[8], counts=[1, 1]),
    dict(heights=[0], widths=[8], counts=[1]),
    dict(heights=[8], widths=[8], counts=[-1]),
])
def test_bad_layouts_raise(kw):
    with pytest.raises(ValueError):
        BatchLayout(block=16, **kw)


def test_block_range_and_index_width():
    with pytest.raises(ValueError):
        BatchLayout([8], [8], [1], 33)
    with pytest.raises(ValueError):
        BatchLayout([8], [8], [1], 1)
    with pytest.raises(ValueError):
        BatchLayout([30000, 30000], [30000, 30000], [1, 1], 16)  # 3*pixels >= 2^31
