"""GMRES with FP64 iterative refinement on the GPU (V x = b, P0 single layer).

The interior Dirichlet problem in the direct formulation of the reference
examples (python/examples/laplace3dDirichlet.py:31-35): V t = (1/2 M + K) g
with g(x) = 1/|x - x0|, x0 outside. Checks: the right-hand side against the
CPU oracle's dense K and M, the solution against a dense FP64 solve with the
oracle's V, the FP64 residual target 1e-8, the analytic Neumann data, and
that a system's solution is the same solved alone and in a batch.
"""
import numpy as np
import pytest

from conftest import rel_l2
from easybem_b200 import meshes

pytestmark = pytest.mark.gpu


def _mass(nodes, elems):
    P = nodes[elems - 1]
    J = np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
    M = np.zeros((elems.shape[0], nodes.shape[0]))
    for k in range(3):
        np.add.at(M, (np.arange(elems.shape[0]), elems[:, k] - 1), J / 6.0)
    return M


def test_dirichlet_solve_sphere_matches_dense_reference(gpu_lib, oracle):
    nodes, elems = meshes.icosphere(3)
    x0 = np.array([0.0, 0.0, 3.0])
    g = 1.0 / np.linalg.norm(nodes - x0, axis=1)
    oracle.set_order(4)
    V, K = oracle.dense(nodes, elems)
    b_ref = 0.5 * _mass(nodes, elems) @ g + K @ g
    t_ref = np.linalg.solve(V, b_ref)
    with gpu_lib.Mesh(nodes, elems) as m:
        b = m.dirichlet_rhs(g)
        assert rel_l2(b, b_ref) < 1e-12
        for prec in ("mixed", "fp64"):
            for pc in (True, False):
                [(t, stats)] = gpu_lib.solve([(m, b)], tol=1e-8, inner_precision=prec, precond=pc)
                assert stats[0]["converged"] and stats[0]["rel_residual"] <= 1e-8
                assert rel_l2(t, t_ref) < 1e-6
    # discretisation error against the exact Neumann data du/dn at centroids
    P = nodes[elems - 1]
    c = P.mean(axis=1)
    n = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    area = 0.5 * np.linalg.norm(n, axis=1)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    d = c - x0
    tex = -(d * n).sum(1) / np.linalg.norm(d, axis=1) ** 3
    err = np.sqrt(np.sum((t - tex) ** 2 * area) / np.sum(tex ** 2 * area))
    assert err < 0.05


def test_batched_solves_uneven_meshes_many_rhs(gpu_lib):
    batch = meshes.ellipsoid_batch(5, seed=11, levels=(1, 2, 3), nrhs=4)
    problems = []
    ms = []
    for item in batch:
        m = gpu_lib.Mesh(item["nodes"], item["elems"])
        ms.append(m)
        g = np.stack([1.0 / np.linalg.norm(item["nodes"] - p, axis=1) for p in item["sources"]])
        problems.append((m, m.dirichlet_rhs(g)))
    out = gpu_lib.solve(problems, tol=1e-8)
    for (m, b), (x, stats) in zip(problems, out):
        assert x.shape == b.shape
        for st in stats:
            assert st["converged"] and st["rel_residual"] <= 1e-8
        # independent FP64 residual check
        for r in range(b.shape[0]):
            assert rel_l2(m.apply_sl(x[r]), b[r]) <= 2e-8
    # the same system solved alone gives the same answer as in the batch
    m0, b0 = problems[2]
    [(x_alone, st_alone)] = gpu_lib.solve([(m0, b0[1:2])], tol=1e-8)
    assert rel_l2(x_alone[0], out[2][0][1]) <= 1e-12
    for m in ms:
        m.close()


def test_stepwise_solver_admits_systems_between_steps(gpu_lib):
    batch = meshes.ellipsoid_batch(3, seed=5, levels=(2, 3), nrhs=2)
    ms = [gpu_lib.Mesh(b["nodes"], b["elems"]) for b in batch]
    rhs = [m.dirichlet_rhs(np.stack([1.0 / np.linalg.norm(b["nodes"] - p, axis=1) for p in b["sources"]]))
           for m, b in zip(ms, batch)]
    s = gpu_lib.Solver(tol=1e-8)
    ids = s.add(ms[0], rhs[0])
    steps = 0
    late = None
    while True:
        n = s.step()
        steps += 1
        if steps == 3:
            late = s.add(ms[1], rhs[1]) + s.add(ms[2], rhs[2])  # join while others run
        if n == 0 and late is not None and all(s.done(i) for i in ids + late):
            break
        assert steps < 2000
    for i in ids + late:
        x, st = s.result(i)
        assert st["converged"] and st["rel_residual"] <= 1e-8
    # a late joiner equals the same system solved alone
    x_mix, _ = s.result(late[0])
    [(x_alone, _)] = gpu_lib.solve([(ms[1], rhs[1][0:1])], tol=1e-8)
    assert rel_l2(x_alone[0], x_mix) <= 1e-12
    s.close()
    for m in ms:
        m.close()


def test_near_field_preconditioner_cuts_iterations_not_accuracy(gpu_lib):
    # torus of the serving workload and a stretched ellipsoid: the same
    # solution (both reach the FP64 residual target) in far fewer iterations
    cases = [meshes.torus(64, 0.3)]
    v, f = meshes.icosphere(4)
    cases.append((v * np.array([2.0, 1.0, 0.5]), f))
    for nodes, elems in cases:
        x0 = np.array([0.3, -0.2, 4.0])
        g = 1.0 / np.linalg.norm(nodes - x0, axis=1)
        with gpu_lib.Mesh(nodes, elems) as m:
            b = m.dirichlet_rhs(g)
            [(t0, s0)] = gpu_lib.solve([(m, b)], tol=1e-8, precond=False)
            [(t1, s1)] = gpu_lib.solve([(m, b)], tol=1e-8, precond=True)
            assert s0[0]["converged"] and s1[0]["converged"]
            assert s1[0]["rel_residual"] <= 1e-8
            assert rel_l2(t1, t0) < 1e-6
            assert 3 * s1[0]["iterations"] <= s0[0]["iterations"], (s0[0]["iterations"], s1[0]["iterations"])


def test_preconditioner_matches_oracle_restatement(gpu_lib, oracle):
    # the GPU normal-equation build against a least-squares restatement on the
    # pinned FP64 near-field values, and its effect: V M close to identity
    from oracle.oracle import near_spai
    nodes, elems = meshes.perturbed_icosphere(2, seed=8)
    oracle.set_order(4)
    V, _ = oracle.dense(nodes, elems)
    M = near_spai(V, elems)
    rng = np.random.default_rng(4)
    with gpu_lib.Mesh(nodes, elems) as m:
        for _ in range(3):
            x = rng.normal(size=elems.shape[0])
            assert rel_l2(m.apply_near_precond(x), M @ x) < 1e-9
    VM = np.asarray(V) @ M
    ev = np.linalg.svd(VM, compute_uv=False)
    assert ev[0] / ev[-1] < np.linalg.cond(np.asarray(V)) / 3


def test_dirichlet_rhs_several_data_sets(gpu_lib, oracle):
    # 1, 2, 3 and 5 data sets: the one-column DL pass, a padded four-column
    # pass, and a full four-column pass plus a single one, all against the
    # oracle's dense K and M (FP64)
    nodes, elems = meshes.perturbed_icosphere(2, seed=6)
    oracle.set_order(4)
    V, K = oracle.dense(nodes, elems)
    M = _mass(nodes, elems)
    rng = np.random.default_rng(10)
    with gpu_lib.Mesh(nodes, elems) as m:
        for n in (1, 2, 3, 5):
            g = rng.normal(size=(n, nodes.shape[0]))
            b = m.dirichlet_rhs(g)
            ref = (0.5 * M @ g.T + np.asarray(K) @ g.T).T
            assert b.shape == (n, elems.shape[0])
            assert rel_l2(b, ref) < 1e-12, n
            for k in range(n):
                assert rel_l2(b[k], ref[k]) < 1e-12, (n, k)
            # K g with the FP32 far field (random data: no cancellation in b)
            b32 = m.dirichlet_rhs(g, precision="mixed")
            for k in range(n):
                assert rel_l2(b32[k], ref[k]) < 1e-6, (n, k)


def test_mixed_dirichlet_rhs_large_mesh(gpu_lib):
    # 5,120 triangles (far field over many cells): the FP32 one- and
    # four-column double-layer passes against the FP64 ones
    nodes, elems = meshes.perturbed_icosphere(4, seed=2)
    rng = np.random.default_rng(12)
    with gpu_lib.Mesh(nodes, elems) as m:
        for n in (1, 5):
            g = rng.normal(size=(n, nodes.shape[0]))
            b64 = m.dirichlet_rhs(g)
            b32 = m.dirichlet_rhs(g, precision="mixed")
            for k in range(n):
                assert rel_l2(b32[k], b64[k]) < 1e-6, (n, k)
            with pytest.raises(ValueError):
                m.dirichlet_rhs(g, precision="fp16")
