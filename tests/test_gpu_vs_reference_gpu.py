"""The reference's own GPU path beside this library on the same mesh.

The reference's FP32 kernels with host-packed pairs (initGPU,
applyGPULaplace3d1Layer/2Layer, src/BEM3dLaplaceGPU.cu:830-1551), compiled
from its sources into oracle/_ref by `make -C oracle refgpu`, run on an L4
sphere. Both are checked against the FP64 oracle; this library's FP64 apply
must be at least as accurate as the reference's FP32 one and faster than it
(a regression guard; measured about 1,000x at FP64 and 3,000x mixed).
"""
import time

import numpy as np
import pytest

from conftest import rel_l2
from easybem_b200 import meshes
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not O.refgpu_available(), reason="reference GPU library not built (make -C oracle refgpu)")
def test_reference_gpu_path_is_slower_and_less_accurate(gpu_lib, oracle):
    nodes, elems = meshes.perturbed_icosphere(4, seed=1)
    rng = np.random.default_rng(3)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    v_ref, q_ref, t_sl, t_dl, _ = O.refgpu_apply(nodes, elems, t, u, 4, repeats=1)
    rows = np.arange(0, elems.shape[0], 37, dtype=np.int32)
    oracle.set_order(4)
    vo, qo = oracle.apply_rows(nodes, elems, t, u, rows)
    with gpu_lib.Mesh(nodes, elems) as m:
        m.apply_sl_dl(t, u)
        a = time.perf_counter()
        v, q = m.apply_sl_dl(t, u)
        ours = time.perf_counter() - a
        pairs = m.far_quad_pairs
    err_ref = max(rel_l2(v_ref[rows], vo), rel_l2(q_ref[rows], qo))
    err_ours = max(rel_l2(v[rows], vo), rel_l2(q[rows], qo))
    print(f"reference GPU FP32: {pairs / (t_sl + t_dl) / 1e9:.2f} Gpairs/s, rel err {err_ref:.1e}; "
          f"this library FP64: {pairs / ours / 1e9:.0f} Gpairs/s, rel err {err_ours:.1e}")
    assert err_ref < 1e-5  # the reference's FP32 path is a valid (if coarser) operator
    assert err_ours < 1e-12 and err_ours < err_ref
    assert ours * 20 < t_sl + t_dl
