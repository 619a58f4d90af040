"""Seeded synthetic surface meshes and mesh-file readers.

All meshes are closed, consistently oriented triangulations with outward
normals (counter-clockwise vertex order seen from outside). Elements are
returned 1-based (int32), nodes as float64 [n, 3], the convention of
easybem's Python API (python/examples/surface3dMesh.py:51-146,
python/bindings.cpp:186-202).

Generators cover the benchmark workloads:

* ``icosphere(level)``: icosahedron refined 1->4 ``level`` times with midpoints
  projected to the unit sphere (20*4^L triangles, 10*4^L+2 vertices);
* ``perturbed_icosphere(level, seed)``: radii r = 1 + 0.1 sum_{l<=4} a_lm Y_lm
  with real spherical harmonics and a_lm ~ N(0, 0.2^2);
* ``ellipsoid_batch(n, seed)``: icospheres of random level scaled to triaxial
  ellipsoids, randomly rotated and offset, with exterior point sources;
* ``torus(n_u, r_minor)``: structured n_u x n_u/4 torus, 2 triangles per quad.
"""
from __future__ import annotations

import math

import numpy as np


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
                  [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
                  [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
                  [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                  [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v, f


def refine(nodes, elems0, project=None):
    """Uniform 1->4 refinement (0-based elements in and out).

    Midpoint numbering follows unique sorted edges, the scheme of
    python/examples/surface3dMesh.py:149-221; ``project`` maps new points.
    """
    P = np.asarray(nodes, dtype=np.float64)
    T = np.asarray(elems0, dtype=np.int64)
    i0, i1, i2 = T[:, 0], T[:, 1], T[:, 2]
    e = np.sort(np.vstack([np.stack([i0, i1], 1), np.stack([i1, i2], 1), np.stack([i2, i0], 1)]), axis=1)
    eu, inv = np.unique(e, axis=0, return_inverse=True)
    inv = inv.reshape(-1)
    mid = 0.5 * (P[eu[:, 0]] + P[eu[:, 1]])
    if project is not None:
        mid = project(mid)
    n = P.shape[0]
    m = len(i0)
    m01 = n + inv[:m]
    m12 = n + inv[m:2 * m]
    m20 = n + inv[2 * m:]
    T2 = np.vstack([np.stack([i0, m01, m20], 1), np.stack([m01, i1, m12], 1),
                    np.stack([m20, m12, i2], 1), np.stack([m01, m12, m20], 1)])
    return np.vstack([P, mid]), T2


def icosphere(level: int):
    """Unit icosphere: returns (nodes [n,3] f64, elements [m,3] int32 1-based)."""
    v, f = _icosahedron()
    for _ in range(level):
        v, f = refine(v, f, project=lambda p: p / np.linalg.norm(p, axis=1, keepdims=True))
    return v, (f + 1).astype(np.int32)


def real_sph_harm(l: int, m: int, theta, phi):
    """Orthonormal real spherical harmonic Y_lm(theta = polar, phi = azimuth)."""
    from scipy.special import lpmv
    am = abs(m)
    norm = math.sqrt((2 * l + 1) / (4 * math.pi) * math.factorial(l - am) / math.factorial(l + am))
    p = lpmv(am, l, np.cos(theta)) * (-1) ** am  # remove the Condon-Shortley phase
    if m > 0:
        return math.sqrt(2.0) * norm * p * np.cos(am * phi)
    if m < 0:
        return math.sqrt(2.0) * norm * p * np.sin(am * phi)
    return norm * p


def perturbed_icosphere(level: int, seed: int = 0, amplitude: float = 0.1, lmax: int = 4, sigma: float = 0.2):
    """Icosphere with radii 1 + amplitude * sum_{l<=lmax} a_lm Y_lm, a_lm ~ N(0, sigma^2)."""
    v, f = icosphere(level)
    rng = np.random.default_rng(seed)
    theta = np.arccos(np.clip(v[:, 2], -1.0, 1.0))
    phi = np.arctan2(v[:, 1], v[:, 0])
    r = np.ones(len(v))
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            r += amplitude * rng.normal(0.0, sigma) * real_sph_harm(l, m, theta, phi)
    return v * r[:, None], f


def random_rotation(rng):
    q, rr = np.linalg.qr(rng.normal(size=(3, 3)))
    q = q * np.sign(np.diag(rr))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


def ellipsoid_batch(n: int = 256, seed: int = 0, levels=(2, 3, 4, 5), nrhs: int = 4):
    """Closed surfaces of uneven size with exterior point-source data.

    Each item: an icosphere of level L drawn uniformly from ``levels``, scaled
    to a triaxial ellipsoid with axes ~U[0.5, 2], rotated by a random rotation,
    offset by ~U[-5, 5]^3, plus ``nrhs`` point sources at distance
    ~U[2, 4] * max-axis from the centre. Returns a list of dicts with
    ``nodes``, ``elems`` (1-based), ``sources`` [nrhs, 3], ``level``.
    """
    rng = np.random.default_rng(seed)
    cache = {}
    out = []
    for _ in range(n):
        L = int(rng.choice(levels))
        if L not in cache:
            cache[L] = icosphere(L)
        v, f = cache[L]
        axes = rng.uniform(0.5, 2.0, size=3)
        R = random_rotation(rng)
        off = rng.uniform(-5.0, 5.0, size=3)
        nodes = (v * axes) @ R.T + off
        dirs = rng.normal(size=(nrhs, 3))
        dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
        dist = rng.uniform(2.0, 4.0, size=nrhs) * axes.max()
        out.append(dict(nodes=nodes, elems=f.copy(), sources=off + dirs * dist[:, None], level=L))
    return out


def torus(n_u: int, r_minor: float, r_major: float = 1.0):
    """Structured torus: n_u x n_v quads (n_v = n_u // 4), 2 triangles each."""
    n_v = max(3, n_u // 4)
    u = 2 * np.pi * np.arange(n_u) / n_u
    w = 2 * np.pi * np.arange(n_v) / n_v
    U, W = np.meshgrid(u, w, indexing="ij")
    x = (r_major + r_minor * np.cos(W)) * np.cos(U)
    y = (r_major + r_minor * np.cos(W)) * np.sin(U)
    z = r_minor * np.sin(W)
    nodes = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    i, j = np.meshgrid(np.arange(n_u), np.arange(n_v), indexing="ij")
    i, j = i.ravel(), j.ravel()
    a = i * n_v + j
    b = ((i + 1) % n_u) * n_v + j
    c = ((i + 1) % n_u) * n_v + (j + 1) % n_v
    d = i * n_v + (j + 1) % n_v
    tris = np.empty((2 * len(a), 3), dtype=np.int64)
    tris[0::2] = np.stack([a, b, c], 1)
    tris[1::2] = np.stack([a, c, d], 1)
    return nodes, (tris + 1).astype(np.int32)


def serving_stream(n: int = 2000, rate: float = 200.0, seed: int = 0, nu_range=(32, 256),
                   r_range=(0.2, 0.4), nrhs_range=(1, 8)):
    """The serving workload: Poisson arrivals of torus Dirichlet solves.

    Request k arrives at the k-th event of a Poisson process of rate ``rate``
    per second; its torus has major radius 1, minor radius ~U[r_range],
    n_u ~ U{nu_range} (n_v = n_u/4) and 1..8 right-hand sides from exterior
    point sources at distance ~U[2, 4] x (1 + r) from the origin. Yields dicts
    with ``t_arrival``, ``nodes``, ``elems`` (1-based) and ``g`` [nrhs, nnodes].
    """
    rng = np.random.default_rng(seed)
    t = 0.0
    for _ in range(n):
        t += rng.exponential(1.0 / rate)
        n_u = int(rng.integers(nu_range[0], nu_range[1] + 1))
        r = float(rng.uniform(*r_range))
        nrhs = int(rng.integers(nrhs_range[0], nrhs_range[1] + 1))
        nodes, elems = torus(n_u, r)
        d = rng.normal(size=(nrhs, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        src = d * rng.uniform(2.0, 4.0, size=(nrhs, 1)) * (1.0 + r)
        g = np.stack([1.0 / np.linalg.norm(nodes - p, axis=1) for p in src])
        yield dict(t_arrival=t, nodes=nodes, elems=elems, g=g, n_u=n_u, r_minor=r)


def point_source_data(nodes, elems, src):
    """Dirichlet data g(x) = 1/|x - src| at the vertices (P1) and centroids (P0)."""
    g_nodes = 1.0 / np.linalg.norm(nodes - src, axis=1)
    cent = nodes[elems - 1].mean(axis=1)
    g_cent = 1.0 / np.linalg.norm(cent - src, axis=1)
    return g_nodes, g_cent


def load_surface_txt(filename):
    """Reads easybem's plain-text surface format (python/examples/surface3dMesh.py:51-83)."""
    with open(filename) as fh:
        toks = [ln for ln in (l.strip() for l in fh) if ln]
    it = iter(toks)
    dim = int(next(it))
    npe = int(next(it))
    if dim != 3 or npe != 3:
        raise ValueError("expected a 3-D triangular surface")
    n = int(next(it))
    P = np.array([list(map(float, next(it).split())) for _ in range(n)], dtype=np.float64)
    m = int(next(it))
    T = np.array([list(map(int, next(it).split())) for _ in range(m)], dtype=np.int32)
    m2 = int(next(it))
    if m2 != m:
        raise ValueError("triangle count mismatch")
    tidx = np.array([int(next(it).split()[1]) for _ in range(m)], dtype=np.int32)
    return P, T, tidx


def load_netgen_vol(filename):
    """Reads the surface triangles of a Netgen .vol file (surface3dMesh.py:86-146)."""
    with open(filename) as fh:
        lines = fh.readlines()

    def find(name):
        for i, ln in enumerate(lines):
            if ln.strip().lower() == name:
                return i
        raise ValueError(f"section {name} not found")

    i = find("points")
    n = int(lines[i + 1])
    P = np.array([list(map(float, lines[i + 2 + k].split()[:3])) for k in range(n)], dtype=np.float64)
    i = find("surfaceelementsgi")
    m = int(lines[i + 1])
    T = np.zeros((m, 3), dtype=np.int32)
    tidx = np.zeros(m, dtype=np.int32)
    for k in range(m):
        parts = lines[i + 2 + k].split()
        nv = int(parts[4])
        T[k] = list(map(int, parts[5:5 + nv]))[:3]
        tidx[k] = int(parts[0])
    return P, T, tidx


def refine_mesh(nodes, elems1, tidx=None):
    """1->4 refinement with 1-based elements in and out (surface3dMesh.py:149-221)."""
    P2, T2 = refine(nodes, np.asarray(elems1) - 1)
    t2 = None if tidx is None else np.repeat(np.asarray(tidx), 4)
    return P2, (T2 + 1).astype(np.int32), t2
