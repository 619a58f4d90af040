"""easybem-b200: B200-native matrix-free Galerkin Laplace layer potentials.

Two Python surfaces over the CUDA library ``libeasybem_gpu.so``:

* the module functions of easybem's pybind module for the GPU path
  (python/bindings.cpp:186-253): ``init_gpu``, ``close_gpu``,
  ``apply_gpu_laplace3d_1layer``, ``apply_gpu_laplace3d_1layer_linears``,
  ``apply_gpu_laplace3d_2layer``, ``apply_gpu_laplace3d_hypersing`` and
  ``version`` — same names, arguments (1-based elements, the ``order``
  index, ignored ``nblocks``/``nthreads``) and result sizes, over one
  process-global mesh;
* ``Mesh``: a handle-based form with an explicit precision
  (``"fp64"``, the default, or ``"mixed"``) and device-pointer applies.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from ._lib import EB_PREC_FP64, EB_PREC_MIXED, EasyBemError, SolveOptions, SolveStats, check, lib

__all__ = ["Mesh", "Batch", "Solver", "Server", "solve", "EasyBemError", "init_gpu", "close_gpu", "apply_gpu_laplace3d_1layer",
           "apply_gpu_laplace3d_1layer_linears", "apply_gpu_laplace3d_2layer",
           "apply_gpu_laplace3d_hypersing", "version", "precision_code", "save_plans", "load_plans", "clear_plans"]


# far-field engines of the fused mixed SL+DL apply (EB_FAR_* in easybem_gpu.h)
FAR_ENGINES = {"cuda": 0, "tensor": 1, "sym": 2, "sym_all": 3}


def precision_code(precision) -> int:
    if precision in (None, "fp64", "double", EB_PREC_FP64):
        return EB_PREC_FP64
    if precision in ("mixed", "fp32", EB_PREC_MIXED):
        return EB_PREC_MIXED
    raise ValueError(f"unknown precision {precision!r}: use 'fp64' or 'mixed'")


def _vec(a, n, name):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if a.shape[0] != n:
        raise ValueError(f"{name} has {a.shape[0]} entries, expected {n}")
    return a


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class Mesh:
    """A surface mesh resident on the GPU with its FP64 near-field correction.

    ``nodes``: float [n, 3]; ``elems``: int [m, 3], 1-based (easybem's
    convention); ``order``: easybem quadrature index (default 4).
    """

    def __init__(self, nodes, elems, order: int = 4):
        L = lib()
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        elems = np.ascontiguousarray(elems, dtype=np.int32)
        if nodes.ndim != 2 or nodes.shape[1] != 3 or elems.ndim != 2 or elems.shape[1] != 3:
            raise ValueError("nodes must be [n, 3] and elements [m, 3]")
        h = ctypes.c_void_p()
        check(L.eb_mesh_create(nodes.shape[0], _ptr(nodes), elems.shape[0], _ptr(elems), int(order),
                               ctypes.byref(h)))
        self._h = h
        self.nnodes = nodes.shape[0]
        self.nelems = elems.shape[0]
        self.order = order
        nv, ne, npairs, nquad = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong(), ctypes.c_longlong()
        check(L.eb_mesh_info(h, ctypes.byref(nv), ctypes.byref(ne), ctypes.byref(npairs), ctypes.byref(nquad)))
        self.near_pairs = npairs.value
        self.far_quad_pairs = nquad.value

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().eb_mesh_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # host-buffer applies -------------------------------------------------
    def apply_sl(self, t, precision="fp64"):
        """v = V t (P0 single layer), t and v of length nelems."""
        t = _vec(t, self.nelems, "t")
        v = np.empty(self.nelems)
        check(lib().eb_apply_sl_p0(self._h, precision_code(precision), _ptr(t), _ptr(v)))
        return v

    def apply_dl(self, u, precision="fp64"):
        """q = K u (double layer, P0 test x P1 trial), u of length nnodes."""
        u = _vec(u, self.nnodes, "u")
        q = np.empty(self.nelems)
        check(lib().eb_apply_dl_p1(self._h, precision_code(precision), _ptr(u), _ptr(q)))
        return q

    def apply_sl_dl(self, t, u, precision="fp64"):
        """(V t, K u) in one pass over the pairs."""
        t = _vec(t, self.nelems, "t")
        u = _vec(u, self.nnodes, "u")
        v = np.empty(self.nelems)
        q = np.empty(self.nelems)
        check(lib().eb_apply_sl_dl(self._h, precision_code(precision), _ptr(t), _ptr(u), _ptr(v), _ptr(q)))
        return v, q

    def apply_sl_p1(self, t, precision="fp64"):
        """v = V1 t (P1 x P1 single layer), t and v of length nnodes."""
        t = _vec(t, self.nnodes, "t")
        v = np.empty(self.nnodes)
        check(lib().eb_apply_sl_p1(self._h, precision_code(precision), _ptr(t), _ptr(v)))
        return v

    def apply_hypersingular(self, u, precision="fp64"):
        """q = D u (hypersingular operator, curl form), u and q of length nnodes."""
        u = _vec(u, self.nnodes, "u")
        q = np.empty(self.nnodes)
        check(lib().eb_apply_hypersingular(self._h, precision_code(precision), _ptr(u), _ptr(q)))
        return q

    # device-pointer apply ------------------------------------------------
    def apply_device(self, d_t, d_u, d_v, d_q, precision="fp64", stream=0):
        """Asynchronous apply on device pointers (ints); 0 skips an operator."""
        check(lib().eb_apply_sl_dl_device(self._h, precision_code(precision), ctypes.c_void_p(d_t or None),
                                          ctypes.c_void_p(d_u or None), ctypes.c_void_p(d_v or None),
                                          ctypes.c_void_p(d_q or None), ctypes.c_void_p(stream or None)))

    def evaluate(self, points, t, u, precision="fp64"):
        """u(x) = V t - W u at points [n, 3] off the surface (representation formula)."""
        pts = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
        t = _vec(t, self.nelems, "t")
        u = _vec(u, self.nnodes, "u")
        out = np.empty(pts.shape[0])
        check(lib().eb_evaluate_potential(self._h, precision_code(precision), pts.shape[0], _ptr(pts), _ptr(t),
                                          _ptr(u), _ptr(out)))
        return out

    def dirichlet_rhs(self, g, precision: str = "fp64"):
        """b = (1/2) M g + K g for vertex data g ([nnodes] or [nrhs, nnodes]);
        K g in FP64 (default) or mixed precision (FP32 far field)."""
        g = np.ascontiguousarray(g, dtype=np.float64)
        one = g.ndim == 1
        g2 = g.reshape(-1, self.nnodes)
        b = np.empty((g2.shape[0], self.nelems))
        check(lib().eb_dirichlet_rhs_prec(self._h, precision_code(precision), g2.shape[0], _ptr(g2), _ptr(b)))
        return b[0] if one else b

    def apply_near_precond(self, x):
        """y = M x with the solver's preconditioner (sparse approximate inverse of the near field)."""
        x = _vec(x, self.nelems, "x")
        y = np.empty(self.nelems)
        check(lib().eb_apply_near_precond(self._h, _ptr(x), _ptr(y)))
        return y

    @property
    def topology_on_device(self) -> bool:
        """True when the near-pair lists were built on the GPU (large meshes)."""
        v = ctypes.c_int()
        check(lib().eb_mesh_topology_on_device(self._h, ctypes.byref(v)))
        return bool(v.value)

    def near_field_bytes(self):
        """(near-field SpMV bytes, far partial-sum fold bytes) of one fused apply."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().eb_mesh_near_field_bytes(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def cell_pairs(self):
        """(triangle pairs in well-separated source cells, in the other cells)."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().eb_mesh_cell_pairs(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_far_engine(self, engine: str = "tensor"):
        """Far-field engine of the fused mixed SL+DL apply: "tensor" (tcgen05
        GEMMs for the pair distances), "cuda" (FP32 pipes only, every ordered
        pair) or "sym" (FP32 pipes, every unordered pair once, added to both
        rows; the default); "sym_all" takes the symmetric kernel for the FP64
        apply too."""
        check(lib().eb_mesh_set_far_engine(self._h, FAR_ENGINES[engine]))

    def far_engine(self, precision="mixed"):
        e = ctypes.c_int()
        check(lib().eb_mesh_get_far_engine(self._h, precision_code(precision), ctypes.byref(e)))
        return {v: k for k, v in FAR_ENGINES.items() if k != "sym_all"}[e.value]

    def set_profiling(self, on: bool = True):
        check(lib().eb_set_profiling(self._h, 1 if on else 0))

    def last_kernel_ms(self):
        a, b = ctypes.c_double(), ctypes.c_double()
        check(lib().eb_last_kernel_ms(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    # launch plan -----------------------------------------------------------
    def plan(self):
        """The far-field launch plan: dict(items_per_sm, src_tile, nsplit, work_items)."""
        a, b, c, d = (ctypes.c_int() for _ in range(4))
        check(lib().eb_mesh_get_plan(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d)))
        return {"items_per_sm": a.value, "src_tile": b.value, "nsplit": c.value, "work_items": d.value}

    def set_plan(self, items_per_sm: int = 32, src_tile: int = 0):
        check(lib().eb_mesh_set_plan(self._h, int(items_per_sm), int(src_tile)))

    def autotune(self, precision="mixed", operators="sl+dl", reps: int = 3):
        """Times the candidate plans on this mesh and keeps the fastest.

        Returns dict(items_per_sm, src_tile, ms, start_ms)."""
        ops = {"sl": 1, "dl": 2, "sl+dl": 3}[operators]
        a, b = ctypes.c_int(), ctypes.c_int()
        ms, ms0 = ctypes.c_double(), ctypes.c_double()
        check(lib().eb_autotune(self._h, precision_code(precision), ops, int(reps), ctypes.byref(a), ctypes.byref(b),
                                ctypes.byref(ms), ctypes.byref(ms0)))
        return {"items_per_sm": a.value, "src_tile": b.value, "ms": ms.value, "start_ms": ms0.value}


def set_device_topology_min(nelems: int):
    """Meshes created from now on with at least nelems triangles build their
    near-pair lists on the GPU (default 65,536; 0: every mesh; 2**31 - 1: none)."""
    check(lib().eb_set_device_topology_min(int(nelems)))


def device_topology_min() -> int:
    v = ctypes.c_int()
    check(lib().eb_get_device_topology_min(ctypes.byref(v)))
    return v.value


def save_plans(path: str):
    """Writes the process-wide table of tuned plans to a text file."""
    check(lib().eb_plan_table_save(os.fsencode(path)))


def load_plans(path: str) -> int:
    """Merges a saved plan table; meshes created afterwards start from it."""
    n = ctypes.c_int()
    check(lib().eb_plan_table_load(os.fsencode(path), ctypes.byref(n)))
    return n.value


def clear_plans():
    check(lib().eb_plan_table_clear())


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def read_surface(path: str):
    """Reads a mesh file through the C ABI: easybem's plain-text surface
    (``.txt``) or the surface triangles of a Netgen ``.vol`` file. Returns
    (nodes [n,3] float64, elems [m,3] int32 1-based, labels [m] int32)."""
    fn = lib().eb_read_netgen_vol if str(path).lower().endswith(".vol") else lib().eb_read_surface_txt
    n, m = ctypes.c_int(), ctypes.c_int()
    p = os.fsencode(str(path))
    check(fn(p, ctypes.byref(n), None, ctypes.byref(m), None, None))
    nodes = np.empty((n.value, 3))
    elems = np.empty((m.value, 3), dtype=np.int32)
    labels = np.empty(m.value, dtype=np.int32)
    check(fn(p, ctypes.byref(n), _ptr(nodes), ctypes.byref(m), _ptr(elems), _ptr(labels)))
    return nodes, elems, labels


def refine_mesh(nodes, elems, labels=None):
    """Uniform 1->4 refinement through the C ABI (1-based elements in and
    out); returns (nodes, elems, labels or None)."""
    nodes = np.ascontiguousarray(nodes, dtype=np.float64)
    elems = np.ascontiguousarray(elems, dtype=np.int32)
    lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.int32)
    n2, m2 = ctypes.c_int(), ctypes.c_int()
    args = (nodes.shape[0], _ptr(nodes), elems.shape[0], _ptr(elems), _ptr(lab))
    check(lib().eb_mesh_refine(*args, ctypes.byref(n2), None, ctypes.byref(m2), None, None))
    P2 = np.empty((n2.value, 3))
    T2 = np.empty((m2.value, 3), dtype=np.int32)
    L2 = None if lab is None else np.empty(m2.value, dtype=np.int32)
    check(lib().eb_mesh_refine(*args, ctypes.byref(n2), _ptr(P2), ctypes.byref(m2), _ptr(T2), _ptr(L2)))
    return P2, T2, L2


class Batch:
    """Applies of many meshes in one launch.

    ``Batch(meshes, ncols)``: P0 single layer with ncols right-hand sides;
    ``apply_device(d_t, d_v, stream)`` takes lists of device pointers (one
    [ncols][nelems] array per mesh). ``Batch(meshes, sl_dl=True)``: single
    and double layer of one density pair per mesh in the same pass;
    ``apply_sl_dl_device(d_t, d_u, d_v, d_q, stream)`` (t, v, q: [nelems],
    u: [nnodes]) or ``apply_sl_dl(ts, us)`` with host arrays.
    """

    def __init__(self, meshes, ncols: int = 1, precision="mixed", sl_dl: bool = False):
        arr = (ctypes.c_void_p * len(meshes))(*[m.handle.value for m in meshes])
        h = ctypes.c_void_p()
        if sl_dl:
            check(lib().eb_batch_create_sl_dl(len(meshes), arr, precision_code(precision), ctypes.byref(h)))
        else:
            check(lib().eb_batch_create(len(meshes), arr, int(ncols), precision_code(precision), ctypes.byref(h)))
        self._h = h
        self.meshes = list(meshes)
        self.ncols = ncols
        self.sl_dl = sl_dl
        q = ctypes.c_longlong()
        check(lib().eb_batch_info(h, ctypes.byref(q)))
        self.quad_pairs = q.value

    def apply_device(self, d_t, d_v, stream=0):
        n = len(self.meshes)
        check(lib().eb_batch_apply(self._h, (ctypes.c_void_p * n)(*d_t), (ctypes.c_void_p * n)(*d_v),
                                   ctypes.c_void_p(stream or None)))

    def apply_sl_dl_device(self, d_t, d_u, d_v, d_q, stream=0):
        n = len(self.meshes)
        arr = [(ctypes.c_void_p * n)(*x) for x in (d_t, d_u, d_v, d_q)]
        check(lib().eb_batch_apply_sl_dl(self._h, *arr, ctypes.c_void_p(stream or None)))

    def apply_sl_dl(self, ts, us):
        """Host arrays in and out (through device copies made with torch)."""
        import torch
        dt = [torch.from_numpy(np.ascontiguousarray(t, dtype=np.float64)).cuda() for t in ts]
        du = [torch.from_numpy(np.ascontiguousarray(u, dtype=np.float64)).cuda() for u in us]
        dv = [torch.empty_like(t) for t in dt]
        dq = [torch.empty_like(t) for t in dt]
        torch.cuda.synchronize()
        self.apply_sl_dl_device([x.data_ptr() for x in dt], [x.data_ptr() for x in du], [x.data_ptr() for x in dv],
                                [x.data_ptr() for x in dq])
        return [x.cpu().numpy() for x in dv], [x.cpu().numpy() for x in dq]

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().eb_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Solver:
    """Batched GMRES with iterative refinement for V x = b (see include/easybem_gpu.h).

    Systems (mesh, right-hand side) join with ``add`` and advance together with
    ``step``; ``result`` returns (x, stats) once ``done``.
    """

    def __init__(self, tol=1e-8, inner_tol=1e-6, restart=50, max_cycles=40, max_iterations=4000,
                 inner_precision="mixed", precond=True):
        o = SolveOptions(tol, inner_tol, restart, max_cycles, max_iterations, precision_code(inner_precision),
                         1 if precond else 0, precision_code("fp64"))
        h = ctypes.c_void_p()
        check(lib().eb_solver_create(ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._ne = {}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().eb_solver_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, mesh: "Mesh", b):
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1, mesh.nelems)
        ids = (ctypes.c_int * b.shape[0])()
        check(lib().eb_solver_add(self._h, mesh.handle, b.shape[0], _ptr(b), ids))
        for i in ids:
            self._ne[i] = mesh.nelems
        return list(ids)

    def step(self) -> int:
        n = ctypes.c_int()
        check(lib().eb_solver_step(self._h, ctypes.byref(n)))
        return n.value

    def done(self, sid: int) -> bool:
        d = ctypes.c_int()
        check(lib().eb_solver_done(self._h, int(sid), ctypes.byref(d)))
        return bool(d.value)

    def result(self, sid: int):
        x = np.empty(self._ne[sid])
        st = SolveStats()
        check(lib().eb_solver_result(self._h, int(sid), _ptr(x), ctypes.byref(st)))
        return x, {"converged": bool(st.converged), "cycles": st.cycles, "iterations": st.iterations,
                   "rel_residual": st.rel_residual}

    def remove(self, sid: int):
        check(lib().eb_solver_remove(self._h, int(sid)))
        self._ne.pop(sid, None)

    def bytes_per_system(self, mesh: "Mesh") -> int:
        n = ctypes.c_longlong()
        check(lib().eb_solver_bytes_per_system(self._h, mesh.handle, ctypes.byref(n)))
        return n.value


class Server:
    """Continuous-batching BEM solve server (see include/easybem_gpu.h).

    ``submit(nodes, elems, g)`` queues a request (g: [nrhs, nnodes] Dirichlet
    vertex data) and returns its id; ``step()`` advances every running
    request by one iteration; ``result(id)`` returns (t, stats, times) once
    ``state(id) == 4``. ``rhs_precision`` is the precision of the right-hand
    sides (1/2 M + K) g the server computes: "fp64" (default) or "mixed" (FP32
    far field of K g; 1/2 M g and K g cancel for data harmonic inside the
    surface, so b and the solution then carry errors of a few 1e-6).
    """

    STATES = {0: "queued", 1: "preparing", 2: "prepared", 3: "solving", 4: "done", 5: "failed"}

    def __init__(self, budget_bytes: int, max_systems: int = 4096, tol=1e-8, inner_tol=1e-6, restart=50,
                 max_cycles=40, max_iterations=4000, inner_precision="mixed", precond=True, rhs_precision="fp64"):
        o = SolveOptions(tol, inner_tol, restart, max_cycles, max_iterations, precision_code(inner_precision),
                         1 if precond else 0, precision_code(rhs_precision))
        h = ctypes.c_void_p()
        check(lib().eb_server_create(int(budget_bytes), int(max_systems), ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self._shape = {}

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().eb_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, nodes, elems, g, order: int = 4) -> int:
        nodes = np.ascontiguousarray(nodes, dtype=np.float64)
        elems = np.ascontiguousarray(elems, dtype=np.int32)
        g = np.ascontiguousarray(g, dtype=np.float64).reshape(-1, nodes.shape[0])
        rid = ctypes.c_longlong()
        check(lib().eb_server_submit(self._h, nodes.shape[0], _ptr(nodes), elems.shape[0], _ptr(elems), int(order),
                                     g.shape[0], _ptr(g), ctypes.byref(rid)))
        self._shape[rid.value] = (g.shape[0], elems.shape[0])
        return rid.value

    def step(self):
        a, w = ctypes.c_int(), ctypes.c_int()
        check(lib().eb_server_step(self._h, ctypes.byref(a), ctypes.byref(w)))
        return a.value, w.value

    def state(self, rid: int) -> int:
        st = ctypes.c_int()
        check(lib().eb_server_poll(self._h, ctypes.c_longlong(rid), ctypes.byref(st)))
        return st.value

    def result(self, rid: int):
        nrhs, ne = self._shape[rid]
        t = np.empty((nrhs, ne))
        stats = (SolveStats * nrhs)()
        times = np.zeros(4)
        check(lib().eb_server_result(self._h, ctypes.c_longlong(rid), _ptr(t), stats, _ptr(times)))
        st = [{"converged": bool(s.converged), "cycles": s.cycles, "iterations": s.iterations,
               "rel_residual": s.rel_residual} for s in stats]
        return t, st, {"latency_ms": times[0], "queue_ms": times[1], "prepare_ms": times[2], "solve_ms": times[3]}

    def release(self, rid: int):
        check(lib().eb_server_release(self._h, ctypes.c_longlong(rid)))
        self._shape.pop(rid, None)

    def usage(self):
        u, b = ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().eb_server_usage(self._h, ctypes.byref(u), ctypes.byref(b)))
        return u.value, b.value

    STAT_NAMES = ("steps", "step_s", "rebuilds", "rebuild_s", "prepared", "prepare_s", "mesh_s", "rhs_s",
                  "precond_s", "mesh_topology_s", "mesh_tables_s", "mesh_near_s", "tables_alloc_s", "tables_copy_s")

    def stats(self):
        """Operating counters: steps and time in step(), solver batch rebuilds,
        and the preparation worker's time (mesh, right-hand sides, preconditioner)."""
        v = np.zeros(len(self.STAT_NAMES))
        check(lib().eb_server_stats(self._h, _ptr(v), len(v)))
        return dict(zip(self.STAT_NAMES, v.tolist()))


def solve(problems, **options):
    """Solves V x = b for a list of (mesh, b) with b [ne] or [nrhs, ne], all in lockstep.

    Returns a list (per problem) of (x, stats) where x has b's shape and stats
    is a list of per-right-hand-side dicts.
    """
    s = Solver(**options)
    try:
        ids = [s.add(m, b) for m, b in problems]
        while s.step() > 0:
            pass
        out = []
        for (m, b), idl in zip(problems, ids):
            res = [s.result(i) for i in idl]
            x = np.stack([r[0] for r in res])
            out.append((x.reshape(np.shape(b)), [r[1] for r in res]))
        return out
    finally:
        s.close()


# ---------------------------------------------------------------------------
# easybem's module-level GPU API (python/bindings.cpp:186-253).

_global_mesh: Mesh | None = None


def _legacy_precision():
    return "mixed" if os.environ.get("EASYBEM_PRECISION", "fp64") in ("mixed", "fp32") else "fp64"


def init_gpu(nodes, elements, order: int = 4, nblocks: int = 0, nthreads: int = 0):
    """Uploads the process-global mesh (``nblocks``/``nthreads`` are ignored)."""
    global _global_mesh
    if _global_mesh is not None:
        _global_mesh.close()
    _global_mesh = Mesh(nodes, elements, order)


def close_gpu():
    global _global_mesh
    if _global_mesh is not None:
        _global_mesh.close()
    _global_mesh = None


def _mesh() -> Mesh:
    if _global_mesh is None:
        raise RuntimeError("init_gpu must be called first")
    return _global_mesh


def apply_gpu_laplace3d_1layer(vec):
    return _mesh().apply_sl(vec, _legacy_precision())


def apply_gpu_laplace3d_1layer_linears(vec):
    return _mesh().apply_sl_p1(vec, _legacy_precision())


def apply_gpu_laplace3d_2layer(vec):
    return _mesh().apply_dl(vec, _legacy_precision())


def apply_gpu_laplace3d_hypersing(vec):
    return _mesh().apply_hypersingular(vec, _legacy_precision())


def version():
    return "1.0"
