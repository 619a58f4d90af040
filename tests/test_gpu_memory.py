"""The device memory pool behind the library's buffers: a released mesh
leaves its memory in the pool, a new mesh of the same size reuses it, and
eb_release_cached_memory gives the unused part back to the driver."""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2
from easybem_b200 import meshes

pytestmark = pytest.mark.gpu


def _cached(lib):
    b = ctypes.c_longlong()
    assert lib.eb_cached_memory_bytes(ctypes.byref(b)) == 0
    return b.value


def test_released_blocks_are_reused_and_trimmed(gpu_lib):
    from easybem_b200 import _lib
    L = _lib.lib()
    assert L.eb_release_cached_memory() == 0
    base = _cached(L)
    nodes, elems = meshes.perturbed_icosphere(4, seed=2)
    rng = np.random.default_rng(1)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    with gpu_lib.Mesh(nodes, elems) as m:
        v0, q0 = m.apply_sl_dl(t, u)
    held = _cached(L)
    assert held > base
    # the same mesh again: served from the cache, same results
    with gpu_lib.Mesh(nodes, elems) as m:
        assert _cached(L) < held
        v1, q1 = m.apply_sl_dl(t, u)
    assert rel_l2(v1, v0) == 0.0 and rel_l2(q1, q0) == 0.0
    assert L.eb_release_cached_memory() == 0
    assert _cached(L) < held
