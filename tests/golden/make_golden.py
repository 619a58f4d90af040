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

REF_CUBE = "/root/reference/python/examples/cube01-surface.txt"


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


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libeasybem_ref.so is missing: run `make -C oracle ref` first")
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
    cube_nodes, cube_elems, _ = meshes.load_surface_txt(REF_CUBE)
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
    print("wrote", sorted(os.listdir(HERE)))


if __name__ == "__main__":
    main()
