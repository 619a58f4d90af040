"""GPU parity at the meshes and quadrature indices the reference's own drivers run.

python/examples/laplace3dDirichletGPU.py:22-25, :30-35, :62 applies the GPU
operators on shaft-surface_verycoarse.vol (scaled by 1/100) refined 0..4
times at quadrature indices 9..13 (25- to 42-point triangle rules, 10- to
20-point line rules in the Sauter-Schwab near field); laplace3dNeumannGPU.py
runs the same mesh refined once at index 4. The fixture
tests/golden/reference_orders.npz holds the reference's own CPU outputs for
those cases (tests/golden/make_golden.py), plus index 7 on a perturbed
icosphere, index 18 (73-point rule) on the reference cube and sampled rows of
the 10,722-triangle shaft-surface.txt, whose thin, anisotropic triangles
give close but disjoint pairs.

Tolerances (relative L2 against the reference): plain FP64 <= 1e-12, mixed
(FP32 far field) <= 1e-6, hypersingular D u (FP64) <= 1e-11.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-6

CASES = [("shaft0", o) for o in (4, 9, 10, 11, 12, 13)] + [
    ("shaft1", 4), ("shaft1", 10), ("shaft2", 11), ("pico2", 7), ("cube", 18), ("shafttxt", 4)]


@pytest.fixture(scope="module")
def golden_orders():
    return np.load(os.path.join(GOLDEN, "reference_orders.npz"))


@pytest.mark.parametrize("name,order", CASES, ids=[f"{n}-o{o}" for n, o in CASES])
def test_reference_driver_meshes_and_orders(gpu_lib, golden_orders, name, order):
    z = golden_orders
    nodes, elems, t, u = z[f"{name}_nodes"], z[f"{name}_elems"], z[f"{name}_t"], z[f"{name}_u"]
    rows = z[f"{name}_rows"] if f"{name}_rows" in z else slice(None)
    vg, qg = z[f"{name}_o{order}_Vt"], z[f"{name}_o{order}_Ku"]
    with gpu_lib.Mesh(nodes, elems, order) as m:
        v, q = m.apply_sl_dl(t, u)
        ev, eq = rel_l2(v[rows], vg), rel_l2(q[rows], qg)
        v32, q32 = m.apply_sl_dl(t, u, precision="mixed")
        ev32, eq32 = rel_l2(v32[rows], vg), rel_l2(q32[rows], qg)
        print(f"{name} index {order} ({elems.shape[0]} triangles): FP64 SL {ev:.2e} DL {eq:.2e}; "
              f"mixed SL {ev32:.2e} DL {eq32:.2e}")
        assert ev < FP64_TOL and eq < FP64_TOL
        assert ev32 < MIXED_TOL and eq32 < MIXED_TOL


def test_hypersingular_on_the_neumann_driver_mesh(gpu_lib, golden_orders):
    z = golden_orders
    nodes, elems, u = z["shaft1_nodes"], z["shaft1_elems"], z["shaft1_u"]
    with gpu_lib.Mesh(nodes, elems, 4) as m:
        assert rel_l2(m.apply_hypersingular(u), z["shaft1_o4_Du"]) < 1e-11
        assert rel_l2(m.apply_hypersingular(u, precision="mixed"), z["shaft1_o4_Du"]) < MIXED_TOL


@pytest.mark.parametrize("order", [9, 13, 18])
def test_potential_at_large_rules(gpu_lib, golden_orders, oracle, order):
    """evaluateLaplace3d (src/BEM3dLaplace.cpp:784-843) at the reference
    driver's indices on its shaft mesh (25- to 73-point rules), points inside,
    outside and within a fraction of an element of the surface, against the
    oracle (pinned to the reference's evaluateLaplace3d on CPU)."""
    z = golden_orders
    nodes, elems, t, u = z["shaft0_nodes"], z["shaft0_elems"], z["shaft0_t"], z["shaft0_u"]
    c = nodes.mean(axis=0)
    rng = np.random.default_rng(order)
    tri = nodes[elems[rng.choice(elems.shape[0], 40)] - 1].mean(axis=1)
    n = rng.normal(size=(40, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    pts = np.vstack([tri + 0.02 * n, c + rng.normal(size=(20, 3)) * 0.3, c + rng.normal(size=(20, 3)) * 4.0])
    oracle.set_order(order)
    ref = oracle.evaluate(nodes, elems, pts, t, u)
    oracle.set_order(4)
    with gpu_lib.Mesh(nodes, elems, order) as m:
        assert rel_l2(m.evaluate(pts, t, u), ref) < 1e-12
        assert rel_l2(m.evaluate(pts, t, u, precision="mixed"), ref) < MIXED_TOL


def test_p1_single_layer_at_a_large_rule(gpu_lib, golden_orders, oracle):
    """applyGPULaplace3d1Layer(t, v, 1) (P1 x P1) at index 10 (25-point
    triangle rule, 12-point line rule) on the reference driver's shaft mesh,
    against the oracle's dense P1 matrix at the same index."""
    z = golden_orders
    nodes, elems, u = z["shaft0_nodes"], z["shaft0_elems"], z["shaft0_u"]
    oracle.set_order(10)
    ref = oracle.p1_dense(nodes, elems) @ u
    oracle.set_order(4)
    with gpu_lib.Mesh(nodes, elems, 10) as m:
        assert rel_l2(m.apply_sl_p1(u), ref) < 1e-12
        assert rel_l2(m.apply_sl_p1(u, precision="mixed"), ref) < MIXED_TOL
