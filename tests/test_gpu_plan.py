"""Launch plans and the plan autotuner on the GPU.

A plan changes how the far-field work is cut (work items per SM) and staged
(source triangles per shared-memory tile); the operator must not change
beyond rounding. Tolerances (relative L2) as in the parity tests: FP64 plans
agree to 1e-13 with each other, mixed plans to 1e-6 with FP64, and every plan
meets the pinned oracle on sampled rows.
"""
import numpy as np
import pytest

from conftest import rel_l2
from easybem_b200 import EasyBemError, meshes

pytestmark = pytest.mark.gpu


def test_every_plan_gives_the_same_operator(gpu_lib, oracle):
    nodes, elems = meshes.perturbed_icosphere(4, seed=4)
    rng = np.random.default_rng(5)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    rows = np.sort(rng.choice(elems.shape[0], 64, replace=False)).astype(np.int32)
    oracle.set_order(4)
    vo, qo = oracle.apply_rows(nodes, elems, t, u, rows)
    with gpu_lib.Mesh(nodes, elems) as m:
        v0, q0 = m.apply_sl_dl(t, u)
        for ips, tile in [(1, 0), (4, 16), (13, 32), (128, 0), (4096, 7)]:
            m.set_plan(ips, tile)
            p = m.plan()
            assert p["items_per_sm"] == ips and p["src_tile"] == tile
            assert p["work_items"] >= 1 and p["nsplit"] >= 1
            v, q = m.apply_sl_dl(t, u)
            assert rel_l2(v, v0) < 1e-13 and rel_l2(q, q0) < 1e-13, (ips, tile)
            assert rel_l2(v[rows], vo) < 1e-12 and rel_l2(q[rows], qo) < 1e-12, (ips, tile)
            v32, q32 = m.apply_sl_dl(t, u, precision="mixed")
            assert rel_l2(v32, v0) < 1e-6 and rel_l2(q32, q0) < 1e-6, (ips, tile)
            # the other operators that share the far kernel
            assert rel_l2(m.apply_sl(t), v0) < 1e-13
            assert m.apply_sl_p1(u).shape == (nodes.shape[0],)


def test_invalid_plans_are_rejected(gpu_lib):
    nodes, elems = meshes.icosphere(2)
    with gpu_lib.Mesh(nodes, elems) as m:
        before = m.plan()
        for ips, tile in [(0, 0), (-1, 0), (5000, 0), (8, -1), (8, 65)]:
            with pytest.raises(EasyBemError):
                m.set_plan(ips, tile)
        assert m.plan() == before


def test_autotune_keeps_the_fastest_and_seeds_new_meshes(gpu_lib, tmp_path):
    gpu_lib.clear_plans()
    nodes, elems = meshes.perturbed_icosphere(5, seed=6)
    rng = np.random.default_rng(1)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    with gpu_lib.Mesh(nodes, elems) as m:
        v0, q0 = m.apply_sl_dl(t, u, precision="mixed")
        r = m.autotune(precision="mixed", reps=3)
        assert r["items_per_sm"] in (4, 8, 16, 32, 64, 128, 256, 512)
        assert r["src_tile"] in (0, 16, 32)
        assert 0 < r["ms"] <= r["start_ms"]
        p = m.plan()
        assert (p["items_per_sm"], p["src_tile"]) == (r["items_per_sm"], r["src_tile"])
        v, q = m.apply_sl_dl(t, u, precision="mixed")
        assert rel_l2(v, v0) < 1e-6 and rel_l2(q, q0) < 1e-6
    # a new mesh in the same size bucket starts from the tuned plan
    nodes2, elems2 = meshes.perturbed_icosphere(5, seed=7)
    with gpu_lib.Mesh(nodes2, elems2) as m2:
        p2 = m2.plan()
        assert (p2["items_per_sm"], p2["src_tile"]) == (r["items_per_sm"], r["src_tile"])
    # the table survives a save / clear / load round trip
    path = str(tmp_path / "plans.txt")
    gpu_lib.save_plans(path)
    gpu_lib.clear_plans()
    with gpu_lib.Mesh(nodes2, elems2) as m3:
        assert m3.plan()["items_per_sm"] == 32
    assert gpu_lib.load_plans(path) == 1
    with gpu_lib.Mesh(nodes2, elems2) as m4:
        assert m4.plan()["items_per_sm"] == r["items_per_sm"]
    gpu_lib.clear_plans()


def test_batch_follows_a_changed_plan(gpu_lib):
    import torch
    ms = [gpu_lib.Mesh(*meshes.perturbed_icosphere(3, seed=s)) for s in (1, 2)]
    rng = np.random.default_rng(3)
    ts = [rng.normal(size=m.nelems) for m in ms]
    ref = [m.apply_sl(t) for m, t in zip(ms, ts)]
    ms[0].set_plan(128, 16)
    b = gpu_lib.Batch(ms, ncols=1, precision="fp64")
    d_t = [torch.tensor(t, device="cuda") for t in ts]
    d_v = [torch.empty_like(x) for x in d_t]
    b.apply_device([x.data_ptr() for x in d_t], [x.data_ptr() for x in d_v])
    torch.cuda.synchronize()
    for v, r in zip(d_v, ref):
        assert rel_l2(v.cpu().numpy(), r) < 1e-13
    b.close()
    for m in ms:
        m.close()
