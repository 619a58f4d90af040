"""Generates the committed golden fixtures from the reference's own CPU code.

Run in a checkout where ``oracle/_ref/libeasybem_ref.so`` was built from the
reference sources (``make -C oracle ref``):

    python tests/golden/make_golden.py

Writes
* ``reference_quadrature.npz``: the reference quadrature tables per index
  (line rules 0..18, triangle rules 0..19), read from the compiled tables of
  src/quadrature.cpp;
* ``reference_ops.npz``: dense getLaplace3d V, K, M (src/BEM3dLaplace.cpp:
  561-781) on small meshes, and V t, K u for seeded densities, at several
  quadrature indices, plus evaluateLaplace3d (:784-843) at seeded points. The cube is the reference example mesh
  python/examples/cube01-surface.txt (8 vertices, 12 triangles).
* ``reference_orders.npz``: the meshes and quadrature indices the reference's
  own GPU driver runs (python/examples/laplace3dDirichletGPU.py:22-25, :30-35,
  :62: shaft-surface_verycoarse.vol scaled by 1/100, refined 1->4 per step,
  indices 9 + step) and its Neumann driver (laplace3dNeumannGPU.py:12-22:
  the same mesh refined once, index 4), plus index 7 on the perturbed
  icosphere, index 18 (the largest rule) on the cube, and sampled rows of the
  10,722-triangle shaft-surface.txt. V t, K u (and D u at index 4) come from
  the reference's dense getLaplace3d, or from its pair routines row by row
  (``rows`` arrays) where the dense matrices would be large.

``python tests/golden/make_golden.py orders`` rewrites only the second file.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from easybem_b200 import meshes  # noqa: E402
from oracle import oracle as O  # noqa: E402


def ref_example(name):
    """A mesh file of the reference's python/examples directory."""
    root = O.reference_root()
    if root is None:
        raise SystemExit("reference tree not found: set EASYBEM_REFERENCE")
    return os.path.join(root, "python", "examples", name)


def compact(nodes, elems1):
    """Drops unreferenced vertices and renumbers (1-based elements)."""
    used = np.unique(elems1 - 1)
    new = np.full(nodes.shape[0], -1, dtype=np.int64)
    new[used] = np.arange(used.size)
    return nodes[used].copy(), (new[elems1 - 1] + 1).astype(np.int32)


def open_cap():
    """An open surface: the perturbed level-2 icosphere without the triangles
    whose centroid lies above z = 0.6 (a shell with a hole, so some edges
    belong to one triangle only)."""
    v, f = meshes.perturbed_icosphere(2, seed=5)
    cz = v[f - 1][:, :, 2].mean(axis=1)
    return compact(v, f[cz < 0.6])


def two_spheres():
    """Two disjoint components: a level-1 icosphere and a scaled, rotated and
    shifted copy of it (pairs across the components are all regular)."""
    v, f = meshes.icosphere(1)
    rot = meshes.random_rotation(np.random.default_rng(11))
    w = (v @ rot.T) * np.array([1.3, 0.8, 1.0]) + np.array([2.5, 0.4, -0.3])
    return np.vstack([v, w]), np.vstack([f, f + v.shape[0]]).astype(np.int32)


def orders_cases():
    """Fixtures at the reference drivers' own meshes and quadrature indices."""
    out = {}

    def dense_case(name, nodes, elems, orders, hyper_at=()):
        rng = np.random.default_rng(17)
        t = rng.normal(size=elems.shape[0])
        u = rng.normal(size=nodes.shape[0])
        out[f"{name}_nodes"], out[f"{name}_elems"] = nodes, elems
        out[f"{name}_t"], out[f"{name}_u"] = t, u
        out[f"{name}_orders"] = np.array(orders)
        for o in orders:
            V, K, D, M = O.ref_dense(nodes, elems, o)
            out[f"{name}_o{o}_Vt"] = V @ t
            out[f"{name}_o{o}_Ku"] = K @ u
            if o in hyper_at:
                out[f"{name}_o{o}_Du"] = D @ u
                out[f"{name}_o{o}_Mu"] = M @ u

    def rows_case(name, nodes, elems, order, rows):
        rng = np.random.default_rng(19)
        t = rng.normal(size=elems.shape[0])
        u = rng.normal(size=nodes.shape[0])
        out[f"{name}_nodes"], out[f"{name}_elems"] = nodes, elems
        out[f"{name}_t"], out[f"{name}_u"] = t, u
        out[f"{name}_orders"] = np.array([order])
        out[f"{name}_rows"] = rows.astype(np.int32)
        v, q = O.ref_apply_rows(nodes, elems, t, u, rows=rows, order=order)
        out[f"{name}_o{order}_Vt"] = v
        out[f"{name}_o{order}_Ku"] = q

    P, T, _ = meshes.load_netgen_vol(ref_example("shaft-surface_verycoarse.vol"))
    P = P / 100.0  # laplace3dDirichletGPU.py:33
    T = T.astype(np.int32)
    dense_case("shaft0", P, T, [4, 9, 10, 11, 12, 13])
    P1, T1 = meshes.refine_mesh(P, T)[:2]
    T1 = T1.astype(np.int32)
    dense_case("shaft1", P1, T1, [4, 10], hyper_at=(4,))
    P2, T2 = meshes.refine_mesh(P1, T1)[:2]
    T2 = T2.astype(np.int32)
    rows_case("shaft2", P2, T2, 11, np.arange(0, T2.shape[0], 34))
    v, f = meshes.perturbed_icosphere(2, seed=3)
    dense_case("pico2", v, f.astype(np.int32), [7])
    cube_nodes, cube_elems, _ = meshes.load_surface_txt(ref_example("cube01-surface.txt"))
    dense_case("cube", cube_nodes, cube_elems.astype(np.int32), [18])
    S, ST, _ = meshes.load_surface_txt(ref_example("shaft-surface.txt"))
    S = S / 100.0
    ST = ST.astype(np.int32)
    rows_case("shafttxt", S, ST, 4, np.random.default_rng(23).choice(ST.shape[0], 256, replace=False))
    np.savez_compressed(os.path.join(HERE, "reference_orders.npz"), **out)


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libeasybem_ref.so is missing: run `make -C oracle ref` first")
    if sys.argv[1:] == ["orders"]:
        orders_cases()
        return
    lib = O.ref_lib()
    tabs = {}
    for o in range(20):
        nt = lib.ref_tri_size(o)
        xy, tw = np.zeros(2 * nt), np.zeros(nt)
        lib.ref_tri_rule(o, O._d(xy), O._d(tw))
        tabs[f"tx{o}"], tabs[f"ty{o}"], tabs[f"tw{o}"] = xy[0::2].copy(), xy[1::2].copy(), tw
        if o < 19:
            nl = lib.ref_line_size(o)
            lx, lw = np.zeros(nl), np.zeros(nl)
            lib.ref_line_rule(o, O._d(lx), O._d(lw))
            tabs[f"lx{o}"], tabs[f"lw{o}"] = lx, lw
    np.savez_compressed(os.path.join(HERE, "reference_quadrature.npz"), **tabs)

    cases = {}
    cube_nodes, cube_elems, _ = meshes.load_surface_txt(ref_example("cube01-surface.txt"))
    cases["cube"] = (cube_nodes, cube_elems, [4])
    v, f = meshes.icosphere(2)
    cases["ico2"] = (v, f, [4])
    v, f = meshes.perturbed_icosphere(2, seed=3)
    cases["pico2"] = (v, f, [0, 1, 2, 3, 4, 5, 6, 8])
    v, f = meshes.torus(16, 0.3)
    cases["torus16"] = (v, f, [4])
    cases["cap"] = (*open_cap(), [4])
    cases["pair"] = (*two_spheres(), [4])
    out = {}
    for name, (nodes, elems, orders) in cases.items():
        rng = np.random.default_rng(7)
        t = rng.normal(size=elems.shape[0])
        u = rng.normal(size=nodes.shape[0])
        out[f"{name}_nodes"] = nodes
        out[f"{name}_elems"] = elems
        out[f"{name}_t"] = t
        out[f"{name}_u"] = u
        out[f"{name}_orders"] = np.array(orders)
        for o in orders:
            V, K, D, M = O.ref_dense(nodes, elems, o)
            out[f"{name}_o{o}_Vt"] = V @ t
            out[f"{name}_o{o}_Ku"] = K @ u
            if elems.shape[0] <= 12:
                out[f"{name}_o{o}_V"] = V
                out[f"{name}_o{o}_K"] = K
                out[f"{name}_o{o}_D"] = D
            if o == 4:
                out[f"{name}_M1"] = M @ np.ones(nodes.shape[0])
                out[f"{name}_Du"] = D @ u
                # evaluateLaplace3d at points inside, outside and near the surface
                c = nodes.mean(axis=0)
                rad = np.max(np.linalg.norm(nodes - c, axis=1))
                prng = np.random.default_rng(13)
                dirs = prng.normal(size=(12, 3))
                dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
                scale = np.array([0.1, 0.4, 1.6, 3.0] * 3)[:, None]
                pts = c + dirs * rad * scale
                out[f"{name}_pts"] = pts
                out[f"{name}_eval"] = O.ref_evaluate(nodes, elems, pts, t, u, 4)
    np.savez_compressed(os.path.join(HERE, "reference_ops.npz"), **out)
    orders_cases()
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
