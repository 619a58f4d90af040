"""Mesh generators, readers and refinement (host code, no GPU)."""
import numpy as np
import pytest

from easybem_b200 import meshes


def _check_closed_oriented(nodes, elems1, euler):
    f = np.asarray(elems1) - 1
    nv, ne = nodes.shape[0], f.shape[0]
    directed = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
    # every directed edge once, and its reverse once: closed and consistently oriented
    keys = set(map(tuple, directed))
    assert len(keys) == len(directed)
    assert all((b, a) in keys for a, b in keys)
    nedges = len(directed) // 2
    assert nv - nedges + ne == euler
    return f


def _signed_volume(nodes, f):
    a, b, c = nodes[f[:, 0]], nodes[f[:, 1]], nodes[f[:, 2]]
    return np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0


@pytest.mark.parametrize("level,ne,nv", [(0, 20, 12), (3, 1280, 642), (6, 81920, 40962)])
def test_icosphere_sizes_and_orientation(level, ne, nv):
    v, f = meshes.icosphere(level)
    assert f.shape == (ne, 3) and v.shape == (nv, 3) and f.min() == 1 and f.max() == nv
    assert np.allclose(np.linalg.norm(v, axis=1), 1.0)
    f0 = _check_closed_oriented(v, f, 2)
    assert _signed_volume(v, f0) > 0  # outward normals


def test_perturbed_icosphere_is_seeded():
    a, fa = meshes.perturbed_icosphere(3, seed=1)
    b, fb = meshes.perturbed_icosphere(3, seed=1)
    c, _ = meshes.perturbed_icosphere(3, seed=2)
    assert np.array_equal(a, b) and np.array_equal(fa, fb)
    assert not np.allclose(a, c)
    r = np.linalg.norm(a, axis=1)
    assert 0.5 < r.min() and r.max() < 1.5 and r.std() > 1e-3


@pytest.mark.parametrize("n_u", [32, 100, 256])
def test_torus_sizes(n_u):
    v, f = meshes.torus(n_u, 0.3)
    n_v = n_u // 4
    assert f.shape[0] == 2 * n_u * n_v and v.shape[0] == n_u * n_v
    f0 = _check_closed_oriented(v, f, 0)  # genus 1
    assert _signed_volume(v, f0) > 0


def test_refinement_splits_each_triangle_in_four():
    v, f = meshes.icosphere(1)
    tidx = np.arange(f.shape[0])
    v2, f2, t2 = meshes.refine_mesh(v, f, tidx)
    assert f2.shape[0] == 4 * f.shape[0] and v2.shape[0] == v.shape[0] + f.shape[0] * 3 // 2
    assert np.array_equal(t2, np.repeat(tidx, 4))
    area = lambda P, T: 0.5 * np.linalg.norm(np.cross(P[T[:, 1]] - P[T[:, 0]], P[T[:, 2]] - P[T[:, 0]]), axis=1)
    assert np.isclose(area(v2, f2 - 1).sum(), area(v, f - 1).sum())  # flat split keeps the area
    _check_closed_oriented(v2, f2, 2)


def test_surface_txt_reader(tmp_path):
    v, f = meshes.icosphere(1)
    lines = ["3", "3", str(v.shape[0])] + [" ".join(f"{x:.17g}" for x in p) for p in v]
    lines += [str(f.shape[0])] + [" ".join(map(str, t)) for t in f]
    lines += [str(f.shape[0])] + [f"{k + 1} {k % 3}" for k in range(f.shape[0])]
    path = tmp_path / "surf.txt"
    path.write_text("\n".join(lines) + "\n")
    P, T, tidx = meshes.load_surface_txt(str(path))
    assert np.array_equal(P, v) and np.array_equal(T, f)
    assert np.array_equal(tidx, np.arange(f.shape[0]) % 3)
    path.write_text("2\n3\n")
    with pytest.raises(ValueError):
        meshes.load_surface_txt(str(path))


def test_netgen_vol_reader(tmp_path):
    v, f = meshes.icosphere(0)
    out = ["mesh3d", "dimension", "3", "surfaceelementsgi", str(f.shape[0])]
    out += [f"{1 + k % 2} 1 1 0 3 {t[0]} {t[1]} {t[2]} 0 0 0" for k, t in enumerate(f)]
    out += ["points", str(v.shape[0])] + ["  ".join(f"{x:.17g}" for x in p) for p in v]
    path = tmp_path / "mesh.vol"
    path.write_text("\n".join(out) + "\n")
    P, T, tidx = meshes.load_netgen_vol(str(path))
    assert np.array_equal(P, v) and np.array_equal(T, f)
    assert np.array_equal(tidx, 1 + np.arange(f.shape[0]) % 2)


def test_workload_generators_match_their_configs():
    batch = meshes.ellipsoid_batch(32, seed=0)
    assert {b["level"] for b in batch} <= {2, 3, 4, 5}
    for b in batch:
        assert b["sources"].shape == (4, 3)
        c = b["nodes"].mean(axis=0)
        rad = np.linalg.norm(b["nodes"] - c, axis=1).max()
        assert np.all(np.linalg.norm(b["sources"] - c, axis=1) >= 2.0 * rad - 1e-9)
    reqs = list(meshes.serving_stream(50, seed=0))
    t = [r["t_arrival"] for r in reqs]
    assert t == sorted(t) and 0.05 < t[-1] < 0.5  # about 50 / 200 s
    for r in reqs:
        assert 32 <= r["n_u"] <= 256 and 0.2 <= r["r_minor"] <= 0.4
        assert r["elems"].shape[0] == 2 * r["n_u"] * (r["n_u"] // 4)
        assert 1 <= r["g"].shape[0] <= 8 and r["g"].shape[1] == r["nodes"].shape[0]
