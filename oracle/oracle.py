"""ORACLE loader — test infrastructure only.

Loads two CPU libraries through ctypes:

* ``liboracle.so``: this project's plain-C FP64 restatement of the reference
  operators (``oracle/bem_oracle.c``), built on demand with ``make``;
* ``_ref/libeasybem_ref.so``: the reference's own CPU sources compiled by
  ``oracle/Makefile`` (present when the reference tree was available at build
  time). It pins the restatement and serves as the reported CPU baseline.

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libeasybem_ref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libeasybem_ref_gpu.so")
TABLES_NPZ = os.path.join(os.path.dirname(HERE), "tests", "golden", "reference_quadrature.npz")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def reference_root():
    """The reference source tree, if one is available to build from.

    Taken from the environment variable ``EASYBEM_REFERENCE``, else a checkout
    named ``reference`` beside this repository's directory; None when neither
    holds ``src/BEM3dLaplace.cpp`` (the GPU box carries only the prebuilt
    ``_ref`` libraries).
    """
    cands = [os.environ.get("EASYBEM_REFERENCE", ""),
             os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")]
    for c in cands:
        if c and os.path.isfile(os.path.join(c, "src", "BEM3dLaplace.cpp")):
            return os.path.abspath(c)
    return None


def build():
    """Compiles the port (and the reference libraries when its sources exist)."""
    cmd = ["make", "-s", "-C", HERE, "all"]
    ref = reference_root()
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


_REF = None


def ref_lib():
    """The reference's own CPU code compiled from its sources (or None)."""
    global _REF
    if _REF is None and ref_available():
        lib = ctypes.CDLL(REF_SO)
        lib.ref_line_size.restype = ctypes.c_int
        lib.ref_tri_size.restype = ctypes.c_int
        for f in ("ref_sl_id", "ref_sl_edge", "ref_sl_vertex", "ref_sl_disjoint"):
            getattr(lib, f).restype = ctypes.c_double
        _REF = lib
    return _REF


def reference_rules(order: int):
    """Quadrature tables of the reference for index ``order``.

    Read from the compiled reference when present, else from the committed
    fixture ``tests/golden/reference_quadrature.npz`` made from it.
    """
    lib = ref_lib()
    if lib is not None:
        nl = lib.ref_line_size(order)
        lx, lw = np.zeros(nl), np.zeros(nl)
        lib.ref_line_rule(order, _d(lx), _d(lw))
        nt = lib.ref_tri_size(order)
        xy, tw = np.zeros(2 * nt), np.zeros(nt)
        lib.ref_tri_rule(order, _d(xy), _d(tw))
        xy = xy.reshape(nt, 2)
        l2x, l2w = np.zeros(2), np.zeros(2)
        lib.ref_line_rule(1, _d(l2x), _d(l2w))
        return dict(lx=lx, lw=lw, tx=xy[:, 0].copy(), ty=xy[:, 1].copy(), tw=tw, l2x=l2x, l2w=l2w)
    z = np.load(TABLES_NPZ)
    return dict(lx=z[f"lx{order}"], lw=z[f"lw{order}"], tx=z[f"tx{order}"], ty=z[f"ty{order}"],
                tw=z[f"tw{order}"], l2x=z["lx1"], l2w=z["lw1"])


class Oracle:
    """FP64 CPU restatement of the reference Galerkin SL/DL operators."""

    def __init__(self, order: int = 4):
        if not os.path.exists(PORT_SO) or (
                os.path.getmtime(PORT_SO) < os.path.getmtime(os.path.join(HERE, "bem_oracle.c"))):
            subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
        self.lib = ctypes.CDLL(PORT_SO)
        for f in ("orc_sl_id", "orc_sl_edge", "orc_sl_vertex", "orc_sl_disjoint"):
            getattr(self.lib, f).restype = ctypes.c_double
        self.order = None
        self.set_order(order)

    def set_order(self, order: int):
        r = reference_rules(order)
        self.rules = r
        self.lib.orc_set_rules(len(r["lx"]), _d(r["lx"]), _d(r["lw"]), len(r["tw"]), _d(r["tx"]),
                               _d(r["ty"]), _d(r["tw"]), _d(r["l2x"]), _d(r["l2w"]))
        self.order = order

    @staticmethod
    def _mesh(nodes, elems):
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        elems = np.ascontiguousarray(elems, dtype=np.int32)
        return nodes, elems

    def apply_rows(self, nodes, elems, t=None, u=None, rows=None, nthreads: int = 0):
        """Rows ``rows`` of V t and K u (elements 1-based)."""
        nodes, elems = self._mesh(nodes, elems)
        ne = elems.shape[0]
        rows = np.arange(ne, dtype=np.int32) if rows is None else np.ascontiguousarray(rows, dtype=np.int32)
        v = np.zeros(len(rows))
        q = np.zeros(len(rows))
        tt = None if t is None else np.ascontiguousarray(t, dtype=np.float64)
        uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
        self.lib.orc_apply_rows(_d(nodes), ne, _i(elems), _d(tt) if tt is not None else None,
                                _d(uu) if uu is not None else None, len(rows), _i(rows), _d(v), _d(q),
                                nthreads)
        return v, q

    def dense(self, nodes, elems, nthreads: int = 0):
        """Dense V (ne x ne, row = test triangle) and K (ne x nv)."""
        nodes, elems = self._mesh(nodes, elems)
        ne, nv = elems.shape[0], nodes.shape[0]
        V = np.zeros((ne, ne))
        K = np.zeros((ne, nv))
        self.lib.orc_dense(_d(nodes), nv, ne, _i(elems), _d(V), _d(K), nthreads)
        return V, K

    def evaluate(self, nodes, elems, points, t, u, nthreads: int = 0):
        """u(x) = V t - W u at points (the representation formula)."""
        nodes, elems = self._mesh(nodes, elems)
        pts = np.ascontiguousarray(points, dtype=np.float64)
        out = np.zeros(pts.shape[0])
        self.lib.orc_evaluate(_d(nodes), elems.shape[0], _i(elems), pts.shape[0], _d(pts),
                              _d(np.ascontiguousarray(t, dtype=np.float64)),
                              _d(np.ascontiguousarray(u, dtype=np.float64)), _d(out), nthreads)
        return out

    def p1_dense(self, nodes, elems):
        """Dense P1 x P1 single layer (nv x nv, row = test vertex)."""
        nodes, elems = self._mesh(nodes, elems)
        nv = nodes.shape[0]
        V1 = np.zeros((nv, nv))
        self.lib.orc_p1_dense(_d(nodes), nv, elems.shape[0], _i(elems), _d(V1))
        return V1

    def p1_pair(self, nodes, elems, i, j):
        nodes, elems = self._mesh(nodes, elems)
        I9 = np.zeros(9)
        ti = np.zeros(3, dtype=np.int32)
        tj = np.zeros(3, dtype=np.int32)
        ok = self.lib.orc_p1_pair(_d(nodes), _i(elems), int(i), int(j), _d(I9), _i(ti), _i(tj))
        return bool(ok), I9.reshape(3, 3), ti, tj

    def pair(self, nodes, elems, i, j):
        nodes, elems = self._mesh(nodes, elems)
        vij = ctypes.c_double()
        k = np.zeros(3)
        col = np.zeros(3, dtype=np.int32)
        self.lib.orc_pair(_d(nodes), _i(elems), int(i), int(j), ctypes.byref(vij), _d(k), _i(col))
        return vij.value, k, col


def near_spai(V, elems):
    """Sparse approximate inverse of the near field of V (dense FP64 [ne, ne],
    row = test triangle), as the solver's preconditioner defines it
    (easybem_b200/csrc/precond.cu): N keeps the entries of the triangle pairs
    that share a vertex; column j of M minimises ||N m - e_j||_2 over vectors
    supported on the triangles sharing a vertex with j. Solved here with a
    least-squares routine (the GPU forms the normal equations); returns M
    dense. Not from the reference, which has no preconditioner."""
    V = np.asarray(V, dtype=np.float64)
    f = np.asarray(elems) - 1
    ne = f.shape[0]
    by_vertex = {}
    for i, tri in enumerate(f):
        for v in tri:
            by_vertex.setdefault(int(v), []).append(i)
    ring = [sorted(set(k for v in f[i] for k in by_vertex[int(v)])) for i in range(ne)]
    N = np.zeros_like(V)
    for i in range(ne):
        N[i, ring[i]] = V[i, ring[i]]
    M = np.zeros_like(V)
    for j in range(ne):
        J = ring[j]
        I = sorted(set(i for k in J for i in ring[k]))
        e = np.zeros(len(I))
        e[I.index(j)] = 1.0
        m, *_ = np.linalg.lstsq(N[np.ix_(I, J)], e, rcond=None)
        M[J, j] = m
    return M


def ref_set_order(order: int):
    ref_lib().ref_set_order(order)


def ref_evaluate(nodes, elems, points, t, u, order: int = 4):
    """The reference's evaluateLaplace3d (src/BEM3dLaplace.cpp:784-843)."""
    lib = ref_lib()
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    pts = np.ascontiguousarray(points, dtype=np.float64)
    out = np.zeros(pts.shape[0])
    lib.ref_evaluate(_d(nodes), elems.shape[0], _i(elems), pts.shape[0], _d(pts),
                     _d(np.ascontiguousarray(t, dtype=np.float64)), _d(np.ascontiguousarray(u, dtype=np.float64)),
                     order, _d(out))
    return out


def ref_apply_rows(nodes, elems, t, u, rows=None, nthreads: int = 0, order: int = 4):
    """Rows of V t and K u computed by the reference's own pair routines."""
    lib = ref_lib()
    lib.ref_set_order(order)
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    ne = elems.shape[0]
    rows = np.arange(ne, dtype=np.int32) if rows is None else np.ascontiguousarray(rows, dtype=np.int32)
    v = np.zeros(len(rows))
    q = np.zeros(len(rows))
    lib.ref_apply_rows(nodes.shape[0], _d(nodes), ne, _i(elems), _d(np.ascontiguousarray(t, dtype=np.float64)),
                       _d(np.ascontiguousarray(u, dtype=np.float64)), len(rows), _i(rows), _d(v), _d(q),
                       nthreads)
    return v, q


def refgpu_available() -> bool:
    return os.path.exists(REF_GPU_SO)


def refgpu_apply(nodes, elems, t, u, order: int = 4, repeats: int = 1):
    """The reference's own GPU path (initGPU, applyGPULaplace3d1Layer/2Layer,
    src/BEM3dLaplaceGPU.cu:830-1551, FP32 kernels with host-packed pairs),
    built by `make -C oracle refgpu`. Returns (V t, K u, seconds of the
    fastest SL apply, seconds of the fastest DL apply, seconds of initGPU)."""
    import time
    lib = ctypes.CDLL(REF_GPU_SO)
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    t = np.ascontiguousarray(t, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.zeros(elems.shape[0])
    q = np.zeros(elems.shape[0])
    with _quiet_stdout():
        a = time.perf_counter()
        lib.refgpu_init(nodes.shape[0], _d(nodes), elems.shape[0], _i(elems), order)
        t_init = time.perf_counter() - a
        t_sl = t_dl = float("inf")
        for _ in range(repeats):
            a = time.perf_counter()
            lib.refgpu_apply_sl(_d(t), _d(v))
            t_sl = min(t_sl, time.perf_counter() - a)
            a = time.perf_counter()
            lib.refgpu_apply_dl(_d(u), _d(q))
            t_dl = min(t_dl, time.perf_counter() - a)
        lib.refgpu_close()
    return v, q, t_sl, t_dl, t_init


class _quiet_stdout:
    """Silences the reference's progress printing (std::cout) at the fd level."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        ctypes.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)


def ref_dense(nodes, elems, order: int = 4):
    """The reference's dense getLaplace3d: returns V (row = test), K, D, M."""
    with _quiet_stdout():
        return _ref_dense(nodes, elems, order)


def _ref_dense(nodes, elems, order):
    lib = ref_lib()
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    ne, nv = elems.shape[0], nodes.shape[0]
    V = np.zeros(ne * ne)
    K = np.zeros(ne * nv)
    D = np.zeros(nv * nv)
    M = np.zeros(ne * nv)
    lib.ref_get_laplace3d(nv, _d(nodes), ne, _i(elems), order, _d(V), _d(K), _d(D), _d(M))
    # getLaplace3d writes V[i*ne+j] (i = test), K[i+node*ne], D[a+b*nv], M[i+node*ne]
    return (V.reshape(ne, ne), K.reshape(nv, ne).T.copy(), D.reshape(nv, nv).T.copy(),
            M.reshape(nv, ne).T.copy())
