"""The reference's own Python module running on this library.

oracle/Makefile (target refbind) compiles the reference's python/bindings.cpp
unchanged, with USE_CUDA, into a module named `easybem`, linked as the
reference's CMake links it except that the GPU half (initGPU, closeGPU,
applyGPULaplace3d1Layer/2Layer/HyperSing and the globals ne, nnodes declared
at bindings.cpp:6) is libeasybem_gpu.so instead of src/BEM3dLaplaceGPU.cu.
Its CPU half is the reference's own CPU library (get_laplace3d,
get_laplace3d_mass). These tests replay the call sequence of
python/examples/laplace3dDirichletGPU.py:48-83 and laplace3dNeumannGPU.py:
41-53 through that module and compare with the reference's outputs
(tests/golden/reference_orders.npz) and with its dense CPU operators.
"""
import importlib
import os
import sys

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel_l2

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


@pytest.fixture(scope="module")
def refmod(gpu_lib):
    import glob
    if not glob.glob(os.path.join(REF_DIR, "easybem*.so")):
        pytest.skip("the reference module was not built (make -C oracle refbind needs the reference sources)")
    sys.path.insert(0, REF_DIR)
    try:
        return importlib.import_module("easybem")
    finally:
        sys.path.remove(REF_DIR)


@pytest.fixture(scope="module")
def golden_orders():
    return np.load(os.path.join(GOLDEN, "reference_orders.npz"))


def _quiet(fn, *a):
    """Calls a reference function with its progress printing silenced."""
    from oracle.oracle import _quiet_stdout
    with _quiet_stdout():
        return fn(*a)


@pytest.mark.parametrize("name,order", [("shaft0", 9), ("shaft1", 10), ("shaft0", 4)])
def test_dirichlet_driver_sequence(refmod, golden_orders, name, order):
    eb = refmod
    z = golden_orders
    P, T = z[f"{name}_nodes"], z[f"{name}_elems"].astype(np.int64)  # int64: bindings.cpp force-casts
    t, u = z[f"{name}_t"], z[f"{name}_u"]
    ne, nv = T.shape[0], P.shape[0]
    eb.init_gpu(P, T, order, 240, 32)
    try:
        v = eb.apply_gpu_laplace3d_1layer(t)
        q = eb.apply_gpu_laplace3d_2layer(u)
        assert v.shape == (ne,) and q.shape == (ne,)  # sized by the globals ne (bindings.cpp:229, :240)
        assert rel_l2(v, z[f"{name}_o{order}_Vt"]) < 1e-12
        assert rel_l2(q, z[f"{name}_o{order}_Ku"]) < 1e-12
        # the driver's Dirichlet problem: b = 1/2 M u + K u, V t = b by CG
        # (laplace3dDirichletGPU.py:13-17, :61-81), against the reference's
        # dense CPU solve from the same module
        from scipy.sparse.linalg import LinearOperator, cg
        xstar = np.array([2.0, 2.0, 2.0])
        g = 1.0 / np.linalg.norm(P - xstar, axis=1)
        MM = _quiet(eb.get_laplace3d_mass, P, T)
        b = 0.5 * (MM @ g) + eb.apply_gpu_laplace3d_2layer(g)
        op = LinearOperator((ne, ne), matvec=eb.apply_gpu_laplace3d_1layer, dtype=np.float64)
        try:
            sol, info = cg(op, b, rtol=1e-12, maxiter=2000)
        except TypeError:  # SciPy before 1.12 names it tol
            sol, info = cg(op, b, tol=1e-12, maxiter=2000)
        assert info == 0
        if ne <= 600:
            V, K, _, M = _quiet(eb.get_laplace3d, P, T, order)
            # the Python V of get_laplace3d is the transpose of the C++ row order
            # (equal to ~1e-8); the GPU apply is V^T t in that convention
            sol_ref = np.linalg.solve(V.T, 0.5 * (M @ g) + K @ g)
            assert rel_l2(sol, sol_ref) < 1e-7
            assert rel_l2(b, 0.5 * (M @ g) + K @ g) < 1e-12
    finally:
        eb.close_gpu()


def test_neumann_driver_operators(refmod, golden_orders):
    """laplace3dNeumannGPU.py:41-53: the hypersingular operator and the P1
    single layer used as its preconditioner, on the shaft mesh refined once
    at index 4."""
    eb = refmod
    z = golden_orders
    P, T, u = z["shaft1_nodes"], z["shaft1_elems"], z["shaft1_u"]
    nv = P.shape[0]
    eb.init_gpu(P, T, 4, 240, 32)
    try:
        d = eb.apply_gpu_laplace3d_hypersing(u)
        assert d.shape == (nv,)  # sized by the global nnodes (bindings.cpp:252)
        assert rel_l2(d, z["shaft1_o4_Du"]) < 1e-11
        # the driver's curl form with the reference's CPU curls, applied with
        # the GPU single layer (laplace3dNeumannGPU.py:36-47)
        C1, C2, C3 = _quiet(eb.get_laplace3d_curl, P, T)
        A = P[T[:, 0] - 1]
        areas = 0.5 * np.linalg.norm(np.cross(P[T[:, 1] - 1] - A, P[T[:, 2] - 1] - A), axis=1)
        m = np.zeros(nv)
        np.add.at(m, T - 1, areas[:, None] / 3)
        dd = sum(C.T @ eb.apply_gpu_laplace3d_1layer(C @ u) for C in (C1, C2, C3)) + m * (m @ u)
        # getLaplace3d's D (src/BEM3dLaplace.cpp:767-771) has no m m^T term; the driver adds it
        assert rel_l2(d + m * (m @ u), dd) < 1e-11
        w = eb.apply_gpu_laplace3d_1layer_linears(u)
        assert w.shape == (nv,)
        from oracle.oracle import Oracle
        o = Oracle(4)
        assert rel_l2(w, o.p1_dense(P, T) @ u) < 1e-12
    finally:
        eb.close_gpu()
