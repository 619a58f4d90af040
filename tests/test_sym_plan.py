"""The symmetric engine's work list (eb_sym_plan, host only): every ordered
pair of triangles of a mesh is covered exactly once, forward or transposed;
every partial slot of a row is written by exactly one work item; and the
slots a row holds (the ones the finalize folds) are exactly the slots its
items write, for meshes whose triangle count fills neither tiles nor cells,
at the single-mesh and the batch item sizes."""
import ctypes

import numpy as np
import pytest

from easybem_b200 import _lib

TILE, CELL = 128, 32


def _plan(ne, cells_per_item):
    L = _lib.lib()
    n, smax = ctypes.c_int(), ctypes.c_int()
    _lib.check(L.eb_sym_plan(ne, cells_per_item, ctypes.byref(n), ctypes.byref(smax), None, None))
    items = np.zeros((n.value, 4), dtype=np.int32)
    slots = np.zeros(ne, dtype=np.int32)
    _lib.check(L.eb_sym_plan(ne, cells_per_item, None, None, items.ctypes.data_as(ctypes.c_void_p),
                             slots.ctypes.data_as(ctypes.c_void_p)))
    return items, slots, smax.value


@pytest.mark.parametrize("ne", [1, 31, 127, 128, 129, 300, 1000, 2049, 5000])
@pytest.mark.parametrize("cells_per_item", [0, 2, 8, 32])
def test_symmetric_plan_covers_every_pair_once(ne, cells_per_item):
    items, slots, smax = _plan(ne, cells_per_item)
    cover = np.zeros((ne, ne), dtype=np.int32)
    written = [set() for _ in range(ne)]
    owner = {}
    for tgt0, c0, c1, split in items:
        tile = tgt0 // TILE
        rows = np.arange(tgt0, min(ne, tgt0 + TILE))
        src = np.arange(c0 * CELL, min(ne, c1 * CELL))
        upper = c0 * CELL >= tgt0 + TILE
        assert upper or (c0 * CELL == tgt0 and src.size == min(TILE, ne - tgt0))
        cover[np.ix_(rows, src)] += 1
        if upper:
            cover[np.ix_(src, rows)] += 1
        for i in rows:
            assert (i, split) not in owner
            owner[(i, split)] = 1
            written[i].add(split)
        if upper:
            for j in src:
                assert (j, tile) not in owner
                owner[(j, tile)] = 1
                written[j].add(tile)
    assert (cover == 1).all()
    for s in range(ne):
        assert written[s] == set(range(slots[s])), s
    assert slots.max() <= smax


def test_symmetric_plan_rejects_bad_sizes():
    L = _lib.lib()
    n = ctypes.c_int()
    assert L.eb_sym_plan(0, 0, ctypes.byref(n), None, None, None) == _lib.EB_ERR_INVALID
    assert L.eb_sym_plan(10, -1, ctypes.byref(n), None, None, None) == _lib.EB_ERR_INVALID
