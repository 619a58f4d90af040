"""The symmetric far field (eb_mesh_set_far_engine(EB_FAR_SYMMETRIC)).

The fused mixed SL+DL apply with every unordered quadrature-point pair
evaluated once and added to both rows of its triangle pair, against the CPU
oracle (relative L2 <= 1e-6, the mixed-precision bar) and against the
CUDA-core kernel that evaluates every ordered pair. The meshes exercise a
partial last target tile and source cell (ne not a multiple of 128 or 32),
small meshes whose every cell is near (masks, the direct-difference form,
the per-lane plane distance), an open surface, two components, and larger
meshes where most cells are well separated. Results are bitwise
reproducible: every partial slot is written by one work item and folded in
slot order. The FP64 form (EB_FAR_SYMMETRIC_ALL, opt-in) is held to the FP64
bar (1e-12 against the oracle).
"""
import numpy as np
import pytest

from conftest import rel_l2
from easybem_b200 import meshes

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-6


def _cases(golden_ops):
    z = golden_ops
    out = [(n, z[f"{n}_nodes"], z[f"{n}_elems"]) for n in ("ico2", "pico2", "torus16", "cap", "pair")]
    v, f = meshes.perturbed_icosphere(4, seed=13)
    out.append(("pico4", v, f))
    v, f = meshes.torus(100, 0.3)  # 5,000 triangles: neither tiles nor cells divide it
    out.append(("torus100", v, f))
    v, f = meshes.icosphere(3)  # stretched: close, nearly parallel sheets
    out.append(("ellipsoid3", v * np.array([2.0, 0.7, 0.25]), f))
    return out


def test_symmetric_far_field_matches_oracle_and_cuda_cores(gpu_lib, golden_ops, oracle):
    oracle.set_order(4)
    for name, nodes, elems in _cases(golden_ops):
        rng = np.random.default_rng(len(name))
        t = rng.normal(size=elems.shape[0])
        u = rng.normal(size=nodes.shape[0])
        ne = elems.shape[0]
        rows = np.arange(ne) if ne <= 1280 else np.sort(rng.choice(ne, 96, replace=False))
        vo, qo = oracle.apply_rows(nodes, elems, t, u, rows.astype(np.int32))
        with gpu_lib.Mesh(nodes, elems) as m:
            m.set_far_engine("cuda")
            vc, qc = m.apply_sl_dl(t, u, precision="mixed")
            m.set_far_engine("sym")
            assert m.far_engine("mixed") == "sym" and m.far_engine("fp64") == "cuda"
            prev = None
            for rep in range(2):
                v, q = m.apply_sl_dl(t, u, precision="mixed")
                ev, eq = rel_l2(v[rows], vo), rel_l2(q[rows], qo)
                print(f"{name} ({ne} triangles): symmetric SL {ev:.2e} DL {eq:.2e}; "
                      f"vs CUDA cores SL {rel_l2(v, vc):.2e} DL {rel_l2(q, qc):.2e}")
                assert ev < MIXED_TOL and eq < MIXED_TOL, name
                assert rel_l2(v, vc) < MIXED_TOL and rel_l2(q, qc) < MIXED_TOL, name
                if prev is not None:
                    assert np.array_equal(v, prev[0]) and np.array_equal(q, prev[1]), name
                prev = (v, q)
            # FP64 and the single operators keep the CUDA-core kernels
            v64, q64 = m.apply_sl_dl(t, u)
            assert rel_l2(v64[rows], vo) < 1e-12 and rel_l2(q64[rows], qo) < 1e-12
            vs = m.apply_sl(t, precision="mixed")
            assert rel_l2(vs[rows], vo) < MIXED_TOL


def test_symmetric_far_field_at_level_6(gpu_lib, oracle):
    """The bench mesh (perturbed icosphere L6, 81,920 triangles): 24 sampled
    rows against the oracle, the CUDA-core kernel on every row, and the
    engine switched back and forth (scratch shared with the other engines)."""
    oracle.set_order(4)
    nodes, elems = meshes.perturbed_icosphere(6, seed=1)
    rng = np.random.default_rng(2024)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    rows = np.sort(rng.choice(elems.shape[0], 24, replace=False)).astype(np.int32)
    vo, qo = oracle.apply_rows(nodes, elems, t, u, rows)
    with gpu_lib.Mesh(nodes, elems) as m:
        m.set_far_engine("sym")
        v, q = m.apply_sl_dl(t, u, precision="mixed")
        assert rel_l2(v[rows], vo) < MIXED_TOL and rel_l2(q[rows], qo) < MIXED_TOL
        m.set_far_engine("cuda")
        vc, qc = m.apply_sl_dl(t, u, precision="mixed")
        assert rel_l2(v, vc) < MIXED_TOL and rel_l2(q, qc) < MIXED_TOL
        m.set_far_engine("sym")
        v2, q2 = m.apply_sl_dl(t, u, precision="mixed")
        assert np.array_equal(v, v2) and np.array_equal(q, q2)
        print(f"L6 symmetric: SL {rel_l2(v[rows], vo):.2e} DL {rel_l2(q[rows], qo):.2e}")


def test_symmetric_far_field_follows_plan_changes(gpu_lib):
    nodes, elems = meshes.perturbed_icosphere(4, seed=14)
    rng = np.random.default_rng(3)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    with gpu_lib.Mesh(nodes, elems) as m:
        m.set_far_engine("sym")
        v0, q0 = m.apply_sl_dl(t, u, precision="mixed")
        for ips in (4, 64, 512):
            m.set_plan(ips)
            v, q = m.apply_sl_dl(t, u, precision="mixed")
            # the symmetric work list does not depend on the forward plan
            assert np.array_equal(v, v0) and np.array_equal(q, q0), ips


def test_symmetric_far_field_in_fp64(gpu_lib, golden_ops, oracle):
    oracle.set_order(4)
    for name, nodes, elems in _cases(golden_ops)[3:]:
        rng = np.random.default_rng(len(name) + 7)
        t = rng.normal(size=elems.shape[0])
        u = rng.normal(size=nodes.shape[0])
        ne = elems.shape[0]
        rows = np.arange(ne) if ne <= 1280 else np.sort(rng.choice(ne, 96, replace=False))
        vo, qo = oracle.apply_rows(nodes, elems, t, u, rows.astype(np.int32))
        with gpu_lib.Mesh(nodes, elems) as m:
            v0, q0 = m.apply_sl_dl(t, u)  # the plain ordered-pair FP64 kernel (the default)
            m.set_far_engine("sym_all")
            assert m.far_engine("fp64") == "sym" and m.far_engine("mixed") == "sym"
            v, q = m.apply_sl_dl(t, u)
            v2, q2 = m.apply_sl_dl(t, u)
            print(f"{name} ({ne} triangles): symmetric FP64 SL {rel_l2(v[rows], vo):.2e} DL {rel_l2(q[rows], qo):.2e}")
            assert rel_l2(v[rows], vo) < 1e-12 and rel_l2(q[rows], qo) < 1e-12, name
            assert rel_l2(v, v0) < 1e-13 and rel_l2(q, q0) < 1e-13, name
            assert np.array_equal(v, v2) and np.array_equal(q, q2), name
            vm, qm = m.apply_sl_dl(t, u, precision="mixed")
            assert rel_l2(vm[rows], vo) < MIXED_TOL and rel_l2(qm[rows], qo) < MIXED_TOL, name


def test_symmetric_single_layer_columns(gpu_lib, oracle):
    """The single-layer-only symmetric kernels (1, 3 and 4 right-hand sides,
    the solver's batched applies): against the oracle and the ordered-pair
    kernel, and every column of a 3- or 4-column batch bitwise equal to the
    same column applied alone."""
    oracle.set_order(4)
    cases = [meshes.perturbed_icosphere(4, seed=5), meshes.torus(100, 0.3)]
    v, f = meshes.icosphere(3)
    cases.append((v * np.array([2.0, 0.7, 0.25]), f))
    ms = [gpu_lib.Mesh(n, e) for n, e in cases]
    rng = np.random.default_rng(77)
    for (nodes, elems), m in zip(cases, ms):
        t = rng.normal(size=elems.shape[0])
        rows = np.sort(rng.choice(elems.shape[0], 64, replace=False)).astype(np.int32)
        vo, _ = oracle.apply_rows(nodes, elems, t, np.zeros(nodes.shape[0]), rows)
        m.set_far_engine("cuda")
        vc = m.apply_sl(t, precision="mixed")
        m.set_far_engine("sym")
        vs = m.apply_sl(t, precision="mixed")
        assert rel_l2(vs[rows], vo) < MIXED_TOL and rel_l2(vs, vc) < MIXED_TOL
        assert np.array_equal(vs, m.apply_sl(t, precision="mixed"))
    _columns_alone_and_together(gpu_lib, ms, rng, "mixed", 1e-12)
    for m in ms:
        m.close()


def _batch_apply(gpu_lib, ms, ts, precision):
    import torch
    d_t = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in ts]
    d_v = [torch.empty_like(x) for x in d_t]
    bt = gpu_lib.Batch(ms, ts[0].shape[0], precision)
    bt.apply_device([x.data_ptr() for x in d_t], [x.data_ptr() for x in d_v])
    torch.cuda.synchronize()
    bt.close()
    return [x.cpu().numpy() for x in d_v]


def _columns_alone_and_together(gpu_lib, ms, rng, precision, tol):
    """Every column of a 3- or 4-column batch is bitwise the column applied in
    a 1-column batch, and agrees with the single-mesh apply (whose work items
    are finer: the same pairs, summed in other groups) to rounding."""
    for ncols in (3, 4):
        ts = [rng.normal(size=(ncols, m.nelems)) for m in ms]
        vs = _batch_apply(gpu_lib, ms, ts, precision)
        for c in range(ncols):
            alone = _batch_apply(gpu_lib, ms, [t[c:c + 1] for t in ts], precision)
            for m, t, v, a in zip(ms, ts, vs, alone):
                assert np.array_equal(v[c], a[0]), (ncols, c)
                assert rel_l2(v[c], m.apply_sl(t[c], precision=precision)) <= tol, (ncols, c)


def test_symmetric_single_layer_in_fp64(gpu_lib, oracle):
    """The FP64 single-layer symmetric kernels (the solver's FP64 residuals on
    the default engine; every FP64 SL apply on EB_FAR_SYMMETRIC_ALL): the FP64
    bar against the oracle and the plain kernel, and every column of a 3- or
    4-column batch bitwise equal to the same column alone."""
    oracle.set_order(4)
    cases = [meshes.perturbed_icosphere(4, seed=6), meshes.torus(100, 0.3)]
    ms = [gpu_lib.Mesh(n, e) for n, e in cases]
    rng = np.random.default_rng(78)
    for (nodes, elems), m in zip(cases, ms):
        t = rng.normal(size=elems.shape[0])
        rows = np.sort(rng.choice(elems.shape[0], 64, replace=False)).astype(np.int32)
        vo, _ = oracle.apply_rows(nodes, elems, t, np.zeros(nodes.shape[0]), rows)
        v0 = m.apply_sl(t)  # the plain ordered-pair FP64 kernel
        m.set_far_engine("sym_all")
        v = m.apply_sl(t)
        assert rel_l2(v[rows], vo) < 1e-12 and rel_l2(v, v0) < 1e-13
        assert np.array_equal(v, m.apply_sl(t))
    _columns_alone_and_together(gpu_lib, ms, rng, "fp64", 1e-14)
    for m in ms:
        m.close()
