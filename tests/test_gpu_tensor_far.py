"""The tensor-core far field (eb_mesh_set_far_engine(EB_FAR_TENSOR_CORES)).

The fused mixed SL+DL apply with |x - y|^2 and the double-layer numerator
as split-TF32 tcgen05 GEMMs, against the CPU oracle (relative L2 <= 1e-6,
the mixed-precision bar) and against the CUDA-core FP32 path, on meshes that
exercise a partial last target tile and source cell (ne not a multiple of
128 or 32), tiles with near cells (small meshes, an open surface, two
components) and a large mesh where most cells are well separated.
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
    return out


def test_tensor_far_field_matches_oracle_and_cuda_cores(gpu_lib, golden_ops, oracle):
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
            m.set_far_engine("tensor")
            assert m.far_engine("mixed") == "tensor" and m.far_engine("fp64") == "cuda"
            for rep in range(2):
                v, q = m.apply_sl_dl(t, u, precision="mixed")
                ev, eq = rel_l2(v[rows], vo), rel_l2(q[rows], qo)
                print(f"{name} ({ne} triangles): tensor SL {ev:.2e} DL {eq:.2e}; "
                      f"vs CUDA cores SL {rel_l2(v, vc):.2e} DL {rel_l2(q, qc):.2e}")
                assert ev < MIXED_TOL and eq < MIXED_TOL, name
                assert rel_l2(v, vc) < MIXED_TOL and rel_l2(q, qc) < MIXED_TOL, name
            # FP64 and the single operators keep the CUDA-core kernels
            v64, q64 = m.apply_sl_dl(t, u)
            assert rel_l2(v64[rows], vo) < 1e-12 and rel_l2(q64[rows], qo) < 1e-12
            # (the SL-only kernel packs target points, the fused one source
            # triangles: the same pairs summed in another order)
            vs = m.apply_sl(t, precision="mixed")
            assert rel_l2(vs[rows], vo) < MIXED_TOL and rel_l2(vs, vc) < MIXED_TOL


def test_tensor_far_field_follows_plan_changes(gpu_lib):
    nodes, elems = meshes.perturbed_icosphere(4, seed=14)
    rng = np.random.default_rng(3)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    with gpu_lib.Mesh(nodes, elems) as m:
        m.set_far_engine("tensor")
        v0, q0 = m.apply_sl_dl(t, u, precision="mixed")
        for ips in (4, 64, 512):
            m.set_plan(ips)
            v, q = m.apply_sl_dl(t, u, precision="mixed")
            assert rel_l2(v, v0) < 1e-7 and rel_l2(q, q0) < 1e-7, ips
