"""The allocation-free apply, eb_apply_sl_dl_noalloc, through the C ABI.

It exists for callers that cannot allocate device memory when they apply the
operator: applications whose GPU memory belongs to their own pool or
framework allocator (an unplanned cudaMalloc would break the budget that
allocator enforces) and loops that must not enter the driver's allocator
because it can synchronise the device. Such a caller hands in device buffers
it already owns; the entry point keeps its scratch in a fixed device array.

Checked here: two calls in a row agree with the allocating entry point
(eb_apply_sl_dl_device) on the same inputs, in both precisions; after one
warm-up call, further calls change neither the device's free memory nor the
library's memory pool nor torch's caching allocator; and a mesh whose scratch
exceeds the fixed array is refused with a clear error.
"""
import ctypes

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _ptr(x):
    return ctypes.c_void_p(x.data_ptr())


@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-6)])
def test_noalloc_matches_allocating_apply_twice(gpu_lib, precision, tol):
    import torch

    from easybem_b200 import _lib, meshes
    L = _lib.lib()
    nodes, elems = meshes.perturbed_icosphere(4, seed=9)
    rng = np.random.default_rng(precision)
    t = torch.from_numpy(rng.normal(size=elems.shape[0])).cuda()
    u = torch.from_numpy(rng.normal(size=nodes.shape[0])).cuda()
    with gpu_lib.Mesh(nodes, elems) as m:
        v_ref = torch.empty_like(t)
        q_ref = torch.empty_like(t)
        _lib.check(L.eb_apply_sl_dl_device(m.handle, precision, _ptr(t), _ptr(u), _ptr(v_ref), _ptr(q_ref), None))
        torch.cuda.synchronize()
        for _ in range(2):
            v = torch.full_like(t, np.nan)
            q = torch.full_like(t, np.nan)
            _lib.check(L.eb_apply_sl_dl_noalloc(m.handle, precision, _ptr(t), _ptr(u), _ptr(v), _ptr(q), None))
            torch.cuda.synchronize()
            assert rel_l2(v.cpu().numpy(), v_ref.cpu().numpy()) <= tol
            assert rel_l2(q.cpu().numpy(), q_ref.cpu().numpy()) <= tol
        # one operator only: the DL output buffer is left untouched
        v = torch.empty_like(t)
        q = torch.full_like(t, 7.0)
        _lib.check(L.eb_apply_sl_dl_noalloc(m.handle, precision, _ptr(t), None, _ptr(v), None, None))
        torch.cuda.synchronize()
        v_sl = torch.empty_like(t)
        _lib.check(L.eb_apply_sl_dl_device(m.handle, precision, _ptr(t), None, _ptr(v_sl), None, None))
        torch.cuda.synchronize()
        assert rel_l2(v.cpu().numpy(), v_sl.cpu().numpy()) <= tol
        assert torch.all(q == 7.0)


def test_noalloc_calls_take_no_device_memory(gpu_lib):
    import torch

    from easybem_b200 import _lib, meshes
    L = _lib.lib()
    nodes, elems = meshes.perturbed_icosphere(4, seed=11)
    rng = np.random.default_rng(5)
    t = torch.from_numpy(rng.normal(size=elems.shape[0])).cuda()
    u = torch.from_numpy(rng.normal(size=nodes.shape[0])).cuda()
    v = torch.empty_like(t)
    q = torch.empty_like(t)
    cached = ctypes.c_longlong(0)
    with gpu_lib.Mesh(nodes, elems) as m:
        # the first call on the device places the fixed array (lazy module loading)
        _lib.check(L.eb_apply_sl_dl_noalloc(m.handle, 1, _ptr(t), _ptr(u), _ptr(v), _ptr(q), None))
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        reserved0 = torch.cuda.memory_reserved()
        _lib.check(L.eb_cached_memory_bytes(ctypes.byref(cached)))
        pool0 = cached.value
        for precision in (1, 0, 1, 0):
            _lib.check(L.eb_apply_sl_dl_noalloc(m.handle, precision, _ptr(t), _ptr(u), _ptr(v), _ptr(q), None))
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        _lib.check(L.eb_cached_memory_bytes(ctypes.byref(cached)))
        assert free1 == free0
        assert torch.cuda.memory_reserved() == reserved0
        assert cached.value == pool0


def test_noalloc_rejects_meshes_beyond_its_scratch(gpu_lib):
    import torch

    from easybem_b200 import _lib, meshes
    L = _lib.lib()
    nodes, elems = meshes.icosphere(6)  # FP64 SL+DL records alone need ~37 MB
    t = torch.zeros(elems.shape[0], dtype=torch.float64, device="cuda")
    u = torch.zeros(nodes.shape[0], dtype=torch.float64, device="cuda")
    v = torch.empty_like(t)
    q = torch.empty_like(t)
    with gpu_lib.Mesh(nodes, elems) as m:
        st = L.eb_apply_sl_dl_noalloc(m.handle, 0, _ptr(t), _ptr(u), _ptr(v), _ptr(q), None)
        assert st == _lib.EB_ERR_INVALID
        assert b"bytes of apply scratch" in L.eb_last_error()
