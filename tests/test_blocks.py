"""Block, neighbour and work tables of the corrected scheme (bhgrid.blocks;
no CUDA): every work list covers its index space exactly once."""
import numpy as np
import pytest

from bhgrid.blocks import (CHUNK, TILE, TILE_MIN, balanced_levels, box_size, flux_item_positions, flux_items,
                           index_count, leveled_blocks, torus_levels, uniform_blocks, work_items)


def _covered(n, items):
    seen = np.zeros((n + 2,) * 3, dtype=np.int32)
    for _, e in items:
        p = flux_item_positions(n, int(e)) + 1
        np.add.at(seen, (p[:, 0], p[:, 1], p[:, 2]), 1)
    return seen


@pytest.mark.parametrize("n", [4, 8, 16, 32, 64, 128])
def test_flux_items_cover_every_position_once(n):
    blocks, _ = leveled_blocks(-1.0, 1.0, np.zeros((1, 1, 1), np.int32), n)
    items = flux_items(blocks)
    assert (items[:, 0] == 0).all()
    tiled = n >= TILE_MIN
    assert ((items[:, 1] >= 0) == tiled).all()
    if tiled:
        m = n + 2
        assert len(items) == -(-m // TILE[0]) * -(-m // TILE[1]) * -(-m // TILE[2])
    else:
        assert len(items) == -(-(n + 2) ** 3 // CHUNK)
    assert (_covered(n, items) == 1).all()


def test_flux_items_of_a_mixed_grid():
    blocks, _ = leveled_blocks(-40.0, 40.0, np.array([[[0, 1], [1, 1]], [[0, 0], [1, 0]]]), 16)
    items = flux_items(blocks, tile_min=32)
    for b, blk in enumerate(blocks):
        mine = items[items[:, 0] == b]
        assert ((mine[:, 1] >= 0) == (int(blk["n"]) >= 32)).all()
        assert (_covered(int(blk["n"]), mine) == 1).all()


@pytest.mark.parametrize("kind", ["cell", "pos", "ghost"])
def test_work_items_chunk_the_index_space(kind):
    blocks, _ = uniform_blocks(-1.0, 1.0, 16, 8)
    items = work_items(blocks, kind)
    for b in range(len(blocks)):
        starts = items[items[:, 0] == b, 1]
        assert (starts == np.arange(0, index_count(8, kind), CHUNK)).all()


def test_boxes_and_offsets():
    blocks, nbr = uniform_blocks(-1.0, 1.0, 16, 8)
    assert len(blocks) == 8 and nbr.shape == (8, 27)
    assert (np.diff(blocks["off"]) == box_size(8)).all()
    assert (nbr[:, 13] == np.arange(8)).all()


def test_torus_levels_are_two_to_one_balanced():
    lv = torus_levels()
    assert (balanced_levels(lv) == lv).all()
    blocks, _ = leveled_blocks(-40.0, 40.0, lv, 8)
    assert sorted(set(int(v) for v in blocks["level"])) == [0, 1, 2]
