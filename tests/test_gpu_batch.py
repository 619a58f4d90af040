"""Batched SL+DL applies (eb_batch_create_sl_dl / eb_batch_apply_sl_dl).

A batch shaped like the 256-surface workload, cut to 40 surfaces: icospheres
of level 2-5 drawn uniformly (320-20,480 triangles), scaled to triaxial
ellipsoids, rotated and offset, each with its own seeded SL and DL
densities, applied in one persistent launch. Checked against the CPU oracle
on sampled rows of every mesh (FP64 <= 1e-12, mixed <= 1e-6 relative L2 over
the sampled rows of the whole batch and per mesh) and against the
single-mesh fused apply (rounding only: the batch's shared-memory tile is
the smallest of its meshes'), with the far field on the CUDA cores and, for
the mixed apply, on the tensor cores and on the symmetric engine (every
unordered pair once; in FP64 too).
"""
import numpy as np
import pytest

from conftest import rel_l2
from easybem_b200 import meshes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def batch40(gpu_lib):
    items = meshes.ellipsoid_batch(40, seed=31, levels=(2, 3, 4, 5), nrhs=1)
    ms = [gpu_lib.Mesh(b["nodes"], b["elems"]) for b in items]
    rng = np.random.default_rng(4)
    ts = [rng.normal(size=m.nelems) for m in ms]
    us = [rng.normal(size=b["nodes"].shape[0]) for b in items]
    yield items, ms, ts, us
    for m in ms:
        m.close()


def test_batched_sl_dl_matches_oracle_on_sampled_rows(gpu_lib, batch40, oracle):
    items, ms, ts, us = batch40
    assert sorted({b["level"] for b in items}) == [2, 3, 4, 5]
    rng = np.random.default_rng(12)
    oracle.set_order(4)
    ref_v, ref_q, rows = [], [], []
    for b, t, u in zip(items, ts, us):
        r = np.sort(rng.choice(b["elems"].shape[0], 6, replace=False)).astype(np.int32)
        vo, qo = oracle.apply_rows(b["nodes"], b["elems"], t, u, r)
        ref_v.append(vo)
        ref_q.append(qo)
        rows.append(r)
    for prec, tol, engine in (("fp64", 1e-12, "cuda"), ("mixed", 1e-6, "cuda"), ("mixed", 1e-6, "tensor"),
                              ("mixed", 1e-6, "sym"), ("fp64", 1e-12, "sym_all")):
        for m in ms:
            m.set_far_engine(engine)
        bt = gpu_lib.Batch(ms, precision=prec, sl_dl=True)
        for rep in range(2):  # the second call replays the captured graph
            vs, qs = bt.apply_sl_dl(ts, us)
            v_all = np.concatenate([v[r] for v, r in zip(vs, rows)])
            q_all = np.concatenate([q[r] for q, r in zip(qs, rows)])
            assert rel_l2(v_all, np.concatenate(ref_v)) < tol, (prec, rep)
            assert rel_l2(q_all, np.concatenate(ref_q)) < tol, (prec, rep)
            for v, q, r, vo, qo in zip(vs, qs, rows, ref_v, ref_q):
                assert rel_l2(v[r], vo) < tol and rel_l2(q[r], qo) < tol, prec
        bt.close()


def test_batched_sl_dl_equals_single_mesh_applies(gpu_lib, batch40):
    items, ms, ts, us = batch40
    for prec, tol, engine in (("fp64", 1e-14, "cuda"), ("mixed", 1e-7, "cuda"), ("mixed", 1e-7, "tensor"),
                              ("mixed", 1e-7, "sym"), ("fp64", 1e-14, "sym_all")):
        for m in ms:
            m.set_far_engine(engine)
        bt = gpu_lib.Batch(ms, precision=prec, sl_dl=True)
        vs, qs = bt.apply_sl_dl(ts, us)
        bt.close()
        for m, t, u, v, q in zip(ms, ts, us, vs, qs):
            v1, q1 = m.apply_sl_dl(t, u, precision=prec)
            assert rel_l2(v, v1) <= tol and rel_l2(q, q1) <= tol, prec


def test_batch_kinds_are_not_mixed_up(gpu_lib, batch40):
    import ctypes

    from easybem_b200 import _lib
    _, ms, _, _ = batch40
    bt = gpu_lib.Batch(ms[:2], precision="mixed", sl_dl=True)
    null = (ctypes.c_void_p * 2)()
    assert _lib.lib().eb_batch_apply(bt._h, null, null, None) == _lib.EB_ERR_INVALID
    bt.close()
    bs = gpu_lib.Batch(ms[:2], ncols=1, precision="mixed")
    assert _lib.lib().eb_batch_apply_sl_dl(bs._h, null, null, null, null, None) == _lib.EB_ERR_INVALID
    bs.close()
