"""Mesh ingestion through the C ABI (eb_read_surface_txt, eb_read_netgen_vol,
eb_mesh_refine; host code, no GPU): the reference's two file formats
(python/examples/surface3dMesh.py:51-146) and its 1->4 refinement
(:149-221), against this package's NumPy restatements of them
(easybem_b200/meshes.py) and, where the reference tree is present, its own
example files."""
import os

import numpy as np
import pytest

import easybem_b200 as eb
from conftest import GOLDEN
from easybem_b200 import meshes


def _write_txt(path, P, T, labels):
    with open(path, "w") as fh:
        fh.write("3\n3\n\n%d\n" % P.shape[0])
        for p in P:
            fh.write("%.17g %.17g %.17g\n" % tuple(p))
        fh.write("\n%d\n" % T.shape[0])
        for t in T:
            fh.write("%d %d %d\n" % tuple(t))
        fh.write("%d\n" % T.shape[0])
        for k, l in enumerate(labels):
            fh.write("%d %d\n" % (k + 1, l))


def _write_vol(path, P, T, labels):
    with open(path, "w") as fh:
        fh.write("mesh3d\ndimension\n3\n\nsurfaceelementsgi\n%d\n" % T.shape[0])
        for t, l in zip(T, labels):
            fh.write(" %d 1 1 0 3 %d %d %d 0 0 0\n" % (l, *t))
        fh.write("\npoints\n%d\n" % P.shape[0])
        for p in P:
            fh.write(" %.17g %.17g %.17g\n" % tuple(p))


@pytest.fixture(scope="module")
def shaft():
    z = np.load(os.path.join(GOLDEN, "reference_orders.npz"))
    return z["shaft0_nodes"], z["shaft0_elems"]


def test_readers_round_trip_both_formats(tmp_path, shaft):
    P, T = shaft
    labels = (np.arange(T.shape[0]) % 7 + 1).astype(np.int32)
    _write_txt(tmp_path / "s.txt", P, T, labels)
    _write_vol(tmp_path / "s.vol", P, T, labels)
    for name, pyread in (("s.txt", meshes.load_surface_txt), ("s.vol", meshes.load_netgen_vol)):
        P2, T2, L2 = eb.read_surface(tmp_path / name)
        P3, T3, L3 = pyread(str(tmp_path / name))
        assert np.array_equal(P2, P) and np.array_equal(T2, T) and np.array_equal(L2, labels)
        assert np.array_equal(P2, P3) and np.array_equal(T2, T3) and np.array_equal(L2, L3)


def test_readers_reject_malformed_files(tmp_path):
    from easybem_b200 import _lib
    (tmp_path / "bad.txt").write_text("2\n3\n0\n0\n0\n")
    (tmp_path / "bad.vol").write_text("mesh3d\npoints\n1\n0 0 0\n")
    for name in ("bad.txt", "bad.vol", "missing.txt"):
        with pytest.raises(_lib.EasyBemError):
            eb.read_surface(tmp_path / name)


def test_refinement_matches_the_numpy_restatement(shaft):
    P, T = shaft
    labels = np.arange(T.shape[0], dtype=np.int32)
    P2, T2, L2 = eb.refine_mesh(P, T, labels)
    P3, T3, _ = meshes.refine_mesh(P, T)
    assert np.array_equal(P2, P3) and np.array_equal(T2, T3)
    m = T.shape[0]
    assert np.array_equal(L2, np.tile(labels, 4))  # children k, m+k, 2m+k, 3m+k of triangle k
    # twice: the reference driver's second refinement step
    P4, T4, _ = eb.refine_mesh(P2, T2)
    assert T4.shape[0] == 16 * m and P4.shape[0] == P2.shape[0] + (3 * T2.shape[0]) // 2
    # every child lies in its parent: the four areas add up
    a = lambda P, T: 0.5 * np.linalg.norm(np.cross(P[T[:, 1] - 1] - P[T[:, 0] - 1], P[T[:, 2] - 1] - P[T[:, 0] - 1]), axis=1)
    assert np.allclose(a(P2, T2).reshape(4, m).sum(axis=0), a(P, T), rtol=1e-12)


def test_refinement_rejects_bad_indices():
    from easybem_b200 import _lib
    with pytest.raises(_lib.EasyBemError):
        eb.refine_mesh(np.zeros((3, 3)), np.array([[1, 2, 4]]))


def test_reference_example_files_when_present():
    from oracle.oracle import reference_root
    root = reference_root()
    if root is None:
        pytest.skip("reference tree not present")
    ex = os.path.join(root, "python", "examples")
    for name, pyread in (("shaft-surface_verycoarse.vol", meshes.load_netgen_vol),
                         ("shaft-surface.txt", meshes.load_surface_txt),
                         ("cube01-surface.txt", meshes.load_surface_txt)):
        P2, T2, L2 = eb.read_surface(os.path.join(ex, name))
        P3, T3, L3 = pyread(os.path.join(ex, name))
        assert np.array_equal(P2, P3) and np.array_equal(T2, T3) and np.array_equal(L2, L3), name
