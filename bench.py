"""Benchmark: matrix-free Galerkin SL (P0) + DL (P0 x P1) apply on one B200.

Workload: the single-mesh matvec of a radius-perturbed icosphere refined 6
times (81,920 triangles, 40,962 vertices; r = 1 + 0.1 sum_{l<=4} a_lm Y_lm,
a_lm ~ N(0, 0.2^2), seed 1), quadrature index 4 (7-point triangle rule),
densities t ~ N(0,1) per triangle and u ~ N(0,1) per vertex. One step is one
fused SL+DL apply: v = V t and q = K u (far field + FP64 near field).

Metric: quadrature-pair evaluations per second (Gpairs/s); one pair is one
(x_a, y_b) kernel evaluation of both operators between triangles that share
no vertex, 49 per triangle pair at index 4. The headline ``value`` is the
mixed-precision apply (FP32 far field with compensated row sums, FP64 near
field) with inputs resident in HBM; the plain FP64 apply is reported beside
it, with the relative L2 error of both against the CPU oracle on sampled
rows. ``e2e`` repeats the mixed apply through the host-buffer C ABI
(eb_apply_sl_dl) with pinned host vectors: H2D of t, u and D2H of v, q in
every step.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
For N > 1 it runs under torch.distributed.run: every rank applies the same
operator on its own GPU (replicas, no data-path collective; weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SL+DL Galerkin apply Gpairs/s, mixed vs FP64 at 1e-6 rel err; p99 solve ms"
LEVEL = 6
SEED = 1
ORDER = 4
WORKLOAD = ("single-mesh SL(P0)+DL(P1) matvec, radius-perturbed icosphere L{level} "
            "({ne:,} triangles, {nv:,} vertices), quadrature index 4 (Q=7)")
# DRAM bytes (read + write) of one CUDA-core far-field launch on the L6 workload under the
# plan of 512 work items per SM (the autotuner's choice there), from an ncu capture of that
# launch: 46.94 MB read (records, target tables) + 107.84 MB written (the partial sums of
# the 117-way source split).
FAR_TRAFFIC_L6 = 46.94e6 + 107.84e6
FAR_TRAFFIC_PLAN = 512
# The same for the symmetric kernel on the L6 workload (independent of the plan): 81.45 MB
# read + 597.83 MB written (the FP64 partial slots, one per 128-triangle tile, row and output).
FAR_SYM_TRAFFIC_L6 = 81.45e6 + 597.83e6
# Far-field engines of the fused mixed apply and their kernels.
ENGINES = ("cuda", "sym", "tensor")
ENGINE_KERNELS = {"cuda": "far_kernel<float,7,7,1,1,false>", "sym": "far_sym_kernel",
                  "tensor": "far_tc_kernel"}
ENGINE_BOUNDS = {"cuda": "FMA pipe and MUFU together",
                 "sym": "FMA pipe (one MUFU rsqrt per two ordered pairs)",
                 "tensor": "MUFU reciprocal square root (tensor cores carry the distance GEMMs)"}


def parse_args(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--level", type=int, default=LEVEL)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-autotune", action="store_true",
                   help="matvec: keep the default launch plan instead of tuning it on the mesh first")
    p.add_argument("--workload", default="matvec", choices=["matvec", "batch", "serve", "large", "small"],
                   help="matvec: the headline single-mesh SL+DL apply (default); batch: 256 uneven "
                        "ellipsoids x 4 RHS, batched apply and GMRES-IR solves; serve: Poisson stream of "
                        "torus solves, p50/p99 latency; large: icosphere L7 apply and solve; small: "
                        "icosphere L3 Dirichlet solve")
    p.add_argument("--requests", type=int, default=2000, help="serve: number of requests in the stream")
    p.add_argument("--serve-sample", type=int, default=300,
                   help="matvec: requests of the serving stream replayed for the p50/p99 sample (0: skip)")
    p.add_argument("--far-engine", default="sym", choices=list(ENGINES),
                   help="matvec: far field of the mixed apply on the FP32 pipes over every ordered pair (cuda), "
                        "over every unordered pair once, added to both rows (sym), or with tcgen05 distance "
                        "GEMMs (tensor); the other engines are timed beside it")
    p.add_argument("--no-extras", action="store_true",
                   help="matvec: skip the batch (256 ellipsoids), large (L7) and small (L3 solve) records "
                        "that a one-GPU run adds to its line")
    p.add_argument("--rhs-precision", default="fp64", choices=["mixed", "fp64"],
                   help="serve: precision of the served right-hand sides (1/2 M + K) g")
    return p.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x, dist=None, device="cpu"):
    """The largest value of x over all ranks (the slowest replica's time)."""
    if dist is None:
        return x
    import torch
    tt = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def replica_throughput(world, pairs_per_replica, step_ms):
    """Whole-job Gpairs/s of `world` independent replicas, each applying
    `pairs_per_replica` pairs per step, timed by the slowest rank's step."""
    return world * pairs_per_replica / (step_ms * 1e-3) / 1e9


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, flag in zip(names, parts[4:8]):
                if flag.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        loaded = [x for x in sm if mx is None or x > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_problem(level):
    from easybem_b200 import meshes
    nodes, elems = meshes.perturbed_icosphere(level, seed=SEED)
    rng = np.random.default_rng(2024)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    return nodes, elems, t, u


def cpu_reference_sample(nodes, elems, t, u, target_s=15.0, nthreads=0):
    """The reference's own FP64 pair routines (oracle/_ref) on sampled rows,
    all host threads; falls back to the oracle port when _ref is absent."""
    from oracle import oracle as O
    ne = elems.shape[0]
    rng = np.random.default_rng(99)
    kind = "reference" if O.ref_available() else "port"
    run = (lambda rows: O.ref_apply_rows(nodes, elems, t, u, rows, nthreads=nthreads, order=ORDER)) \
        if kind == "reference" else (lambda rows: O.Oracle(ORDER).apply_rows(nodes, elems, t, u, rows, nthreads))
    ncores = nthreads or os.cpu_count()
    nrows = max(ncores, 8)
    rows = np.sort(rng.choice(ne, nrows, replace=False)).astype(np.int32)
    a = time.perf_counter(); run(rows); dt = time.perf_counter() - a
    nrows = int(min(ne, max(nrows, nrows * target_s / max(dt, 1e-3))))
    rows = np.sort(rng.choice(ne, nrows, replace=False)).astype(np.int32)
    a = time.perf_counter(); v, q = run(rows); dt = time.perf_counter() - a
    pairs = nrows * (ne - 13) * 49  # disjoint triangle pairs per row (~13 near) x Q^2
    return {"value": pairs / dt / 1e9, "unit": "Gpairs/s", "cores": ncores, "kind": kind,
            "sample": f"{nrows} of {ne} rows of the same SL+DL apply (FP64, {dt:.1f} s)", "seconds": dt}


def run_reference(args):
    """--impl reference: the reference's CPU implementation of the path."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    nodes, elems, t, u = make_problem(args.level)
    from oracle import oracle as O
    kind = "reference" if O.ref_available() else "port"
    ne = elems.shape[0]
    ncores = os.cpu_count()
    rng = np.random.default_rng(7)
    # size one step to a few seconds of work
    probe = cpu_reference_sample(nodes, elems, t, u, target_s=2.0)
    rows_per_step = max(ncores, int(probe["value"] * 1e9 * 4.0 / ((ne - 13) * 49)))
    times = []
    for k in range(args.warmup + args.steps):
        rows = np.sort(rng.choice(ne, min(ne, rows_per_step), replace=False)).astype(np.int32)
        a = time.perf_counter()
        if kind == "reference":
            O.ref_apply_rows(nodes, elems, t, u, rows, order=ORDER)
        else:
            O.Oracle(ORDER).apply_rows(nodes, elems, t, u, rows)
        if k >= args.warmup:
            times.append(time.perf_counter() - a)
    pairs = len(rows) * (ne - 13) * 49
    value = pairs * len(times) / sum(times) / 1e9
    line = {"metric": METRIC, "value": value, "unit": "Gpairs/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD.format(level=args.level, ne=ne, nv=nodes.shape[0]),
                                            "sample_rows_per_step": len(rows)},
            "cpu_baseline": {"value": value, "unit": "Gpairs/s", "cores": ncores, "kind": kind,
                             "sample": f"{len(rows)} of {ne} rows per step, reference FP64 pair routines "
                                       f"(src/BEM3dLaplace.cpp:22-437) with OpenMP"},
            "e2e": {"value": value, "unit": "Gpairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def serve_stream(n, seed=0):
    from easybem_b200 import meshes
    return list(meshes.serving_stream(n, rate=200.0, seed=seed))


def run_serve(args):
    """Serving: 2,000 torus solve requests, Poisson arrivals at 200/s, 120 GB budget."""
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    from easybem_b200.serving import run_stream
    reqs = serve_stream(args.requests, seed=rank)
    res = run_stream(reqs, budget_bytes=120 * 10 ** 9, tol=1e-8, rhs_precision=args.rhs_precision)
    res.pop("results", None)
    if rank == 0:
        line = {"metric": METRIC, "workload": "serve", "value": res["p99_ms"], "unit": "ms (p99 request latency)",
                "higher_is_better": False, "n_gpus": world, "data": "synthetic",
                "config": {"workload": "2,000 torus Dirichlet solves (512-32,768 triangles, 1-8 RHS), Poisson "
                                       "arrivals at 200/s, 120 GB admission budget, tol 1e-8",
                           "requests": args.requests, "rhs_precision": args.rhs_precision},
                **{k: v for k, v in res.items()}}
        print(json.dumps(line), flush=True)


def batch_record(local, solves=True):
    """256 closed surfaces (icosphere L2-L5 ellipsoids): batched SL+DL applies in
    both precisions (one density pair per mesh, one persistent launch), the
    4-RHS batched SL apply, and the GMRES-IR solves of all 1,024 systems."""
    import torch
    import easybem_b200 as eb
    from easybem_b200 import meshes
    items = meshes.ellipsoid_batch(256, seed=3, levels=(2, 3, 4, 5), nrhs=4)
    t0 = time.perf_counter()
    ms = [eb.Mesh(it["nodes"], it["elems"]) for it in items]
    t_create = time.perf_counter() - t0
    dev = torch.device("cuda", local)
    st = torch.cuda.current_stream()
    rng = np.random.default_rng(41)
    d_t = [torch.from_numpy(rng.normal(size=m.nelems)).to(dev) for m in ms]
    d_u = [torch.from_numpy(rng.normal(size=it["nodes"].shape[0])).to(dev) for it in items]
    d_v = [torch.empty_like(x) for x in d_t]
    d_q = [torch.empty_like(x) for x in d_t]
    ptrs = lambda xs: [x.data_ptr() for x in xs]

    def time_batch(bt, run, k):
        for _ in range(2):  # the first call captures the graph
            run(bt)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        for _ in range(k):
            run(bt)
        b.record(st)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / k

    out = {}
    for key, prec, engine in (("mixed", "mixed", "sym"), ("mixed_cuda", "mixed", "cuda"),
                              ("mixed_tensor", "mixed", "tensor"), ("fp64", "fp64", "cuda"),
                              ("fp64_sym", "fp64", "sym_all")):
        for m in ms:
            m.set_far_engine(engine)
        bt = eb.Batch(ms, precision=prec, sl_dl=True)
        ms_apply = time_batch(bt, lambda b: b.apply_sl_dl_device(ptrs(d_t), ptrs(d_u), ptrs(d_v), ptrs(d_q),
                                                                  st.cuda_stream), 3 if prec == "mixed" else 2)
        out[key] = {"engine": engine, "ms_per_apply": ms_apply, "Gpairs_per_s": bt.quad_pairs / (ms_apply * 1e-3) / 1e9}
        out[key + "_vq"] = (torch.cat(d_v).cpu().numpy(), torch.cat(d_q).cpu().numpy())
        bt.close()
    for m in ms:
        m.set_far_engine("sym")
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    mixed_vs_fp64 = {"sl": rel(out["mixed_vq"][0], out["fp64_vq"][0]), "dl": rel(out["mixed_vq"][1], out["fp64_vq"][1])}
    # sampled rows of 8 meshes against the CPU oracle
    from oracle.oracle import Oracle
    orc = Oracle(ORDER)
    offs = np.cumsum([0] + [m.nelems for m in ms])
    ev, eq = [], []
    for i in range(0, 256, 32):
        rows = np.sort(rng.choice(ms[i].nelems, 8, replace=False)).astype(np.int32)
        vo, qo = orc.apply_rows(items[i]["nodes"], items[i]["elems"], d_t[i].cpu().numpy(), d_u[i].cpu().numpy(), rows)
        ev.append((out["fp64_vq"][0][offs[i] + rows], out["mixed_vq"][0][offs[i] + rows], vo))
        eq.append((out["fp64_vq"][1][offs[i] + rows], out["mixed_vq"][1][offs[i] + rows], qo))
    cat = lambda L, k: np.concatenate([x[k] for x in L])
    err = {"fp64_sl": rel(cat(ev, 0), cat(ev, 2)), "mixed_sl": rel(cat(ev, 1), cat(ev, 2)),
           "fp64_dl": rel(cat(eq, 0), cat(eq, 2)), "mixed_dl": rel(cat(eq, 1), cat(eq, 2)), "oracle_rows": 64,
           "mixed_vs_fp64_full": mixed_vs_fp64,
           "mixed_cuda_cores_vs_fp64_full": {"sl": rel(out["mixed_cuda_vq"][0], out["fp64_vq"][0]),
                                             "dl": rel(out["mixed_cuda_vq"][1], out["fp64_vq"][1])}}
    # 4 SL right-hand sides per mesh (the Dirichlet data of the solves)
    rhs = [m.dirichlet_rhs(np.stack([1.0 / np.linalg.norm(it["nodes"] - p, axis=1) for p in it["sources"]]))
           for m, it in zip(ms, items)]
    d_b = [torch.from_numpy(np.ascontiguousarray(b)).to(dev) for b in rhs]
    d_w = [torch.empty_like(x) for x in d_b]
    bt = eb.Batch(ms, 4, "mixed")
    ms4 = time_batch(bt, lambda b: b.apply_device(ptrs(d_b), ptrs(d_w), st.cuda_stream), 3)
    pairs = bt.quad_pairs
    bt.close()
    rec = {"workload": "256 ellipsoids (icosphere L2-L5, 320-20,480 triangles), SL+DL batched apply "
                       "(one density pair per mesh), 4-RHS SL batched apply, GMRES(50)-IR to 1e-8",
           "quad_pairs_per_apply": int(pairs), "mesh_setup_s": t_create,
           "sl_dl_mixed": out["mixed"], "sl_dl_mixed_cuda_cores": out["mixed_cuda"],
           "sl_dl_mixed_tensor_cores": out["mixed_tensor"], "sl_dl_fp64": out["fp64"],
           "sl_dl_fp64_symmetric": out["fp64_sym"],
           "mixed_over_fp64_symmetric": out["mixed"]["Gpairs_per_s"] / out["fp64_sym"]["Gpairs_per_s"],
           "mixed_over_fp64": out["mixed"]["Gpairs_per_s"] / out["fp64"]["Gpairs_per_s"],
           "mixed_cuda_cores_over_fp64": out["mixed_cuda"]["Gpairs_per_s"] / out["fp64"]["Gpairs_per_s"],
           "mixed_tensor_cores_over_fp64": out["mixed_tensor"]["Gpairs_per_s"] / out["fp64"]["Gpairs_per_s"],
           "rel_err_vs_oracle": err,
           "sl_4rhs_mixed": {"ms_per_apply": ms4, "Gpairs_per_s": pairs / (ms4 * 1e-3) / 1e9,
                             "rhs_evals_per_s_G": 4 * pairs / (ms4 * 1e-3) / 1e9}}
    if solves:
        t0 = time.perf_counter()
        res = eb.solve(list(zip(ms, rhs)), tol=1e-8)
        t_solve = time.perf_counter() - t0
        stats = [x for _, sl in res for x in sl]
        rec["solves"] = {"systems": len(stats), "seconds": t_solve, "solves_per_s": len(stats) / t_solve,
                         "converged": sum(x["converged"] for x in stats),
                         "max_rel_residual": max(x["rel_residual"] for x in stats),
                         "iterations_mean": float(np.mean([x["iterations"] for x in stats])),
                         "cycles_mean": float(np.mean([x["cycles"] for x in stats]))}
    for m in ms:
        m.close()
    return rec


def run_batch(args):
    import torch
    _, _, local = dist_env()
    torch.cuda.set_device(local)
    rec = batch_record(local)
    line = {"metric": METRIC, "workload": "batch", "value": rec["sl_dl_mixed"]["Gpairs_per_s"], "unit": "Gpairs/s",
            "higher_is_better": True, "data": "synthetic", "config": {"workload": rec.pop("workload")}, **rec}
    print(json.dumps(line), flush=True)


def large_record(local, solve=False):
    """Icosphere L7 (327,680 triangles): SL+DL apply in both precisions, error on
    16 oracle rows, optionally the GMRES-IR solve."""
    import easybem_b200 as eb
    from oracle.oracle import Oracle
    nodes, elems, t, u = make_problem(7)
    t0 = time.perf_counter()
    m = eb.Mesh(nodes, elems)
    t_create = time.perf_counter() - t0
    m.set_profiling(True)
    res = {}
    for key, engine in (("mixed", "sym"), ("mixed_cuda", "cuda"), ("mixed_tensor", "tensor"), ("fp64", "cuda"),
                        ("fp64_sym", "sym_all")):
        m.set_far_engine(engine)
        p = "fp64" if key.startswith("fp64") else "mixed"
        m.apply_sl_dl(t, u, precision=p)
        v, q = m.apply_sl_dl(t, u, precision=p)
        far, fin = m.last_kernel_ms()
        res[key] = (v, q, far, fin)
    m.set_far_engine("sym")
    rng = np.random.default_rng(5)
    rows = np.sort(rng.choice(elems.shape[0], 16, replace=False)).astype(np.int32)
    vo, qo = Oracle(ORDER).apply_rows(nodes, elems, t, u, rows)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    pairs = m.far_quad_pairs
    peak_tflops, peak_rsqrt = _measure_peak()

    def engine_rec(key, engine):
        mufu_pp, fma_pp, _ = _engine_costs(engine)
        rate = pairs / (res[key][2] * 1e-3)
        bound = min(peak_tflops * 1e12 / (2 * fma_pp), peak_rsqrt * 1e12 / mufu_pp)
        return {"engine": engine, "kernel": ENGINE_KERNELS[engine], "far_ms": res[key][2],
                "finalize_ms": res[key][3], "Gpairs_per_s": rate / 1e9,
                "fma_pipe_frac": rate * 2 * fma_pp / (peak_tflops * 1e12),
                "mufu_frac": rate * mufu_pp / (peak_rsqrt * 1e12), "frac_of_pair_bound": rate / bound,
                "rel_err_sl": rel(res[key][0][rows], vo), "rel_err_dl": rel(res[key][1][rows], qo)}

    cf, cn = m.cell_pairs()
    rec = {"workload": "radius-perturbed icosphere L7 (327,680 triangles, 163,842 vertices)",
           "quad_pairs_per_step": pairs, "near_pairs": m.near_pairs, "mesh_setup_s": t_create,
           "near_cell_share": cn / (cf + cn),
           "mixed": engine_rec("mixed", "sym"),
           "mixed_cuda_cores": engine_rec("mixed_cuda", "cuda"),
           "mixed_tensor_cores": engine_rec("mixed_tensor", "tensor"),
           "fp64": {"far_ms": res["fp64"][2], "finalize_ms": res["fp64"][3],
                    "Gpairs_per_s": pairs / (res["fp64"][2] * 1e-3) / 1e9},
           "fp64_symmetric": {"far_ms": res["fp64_sym"][2], "finalize_ms": res["fp64_sym"][3],
                              "Gpairs_per_s": pairs / (res["fp64_sym"][2] * 1e-3) / 1e9,
                              "rel_err_sl": rel(res["fp64_sym"][0][rows], vo),
                              "rel_err_dl": rel(res["fp64_sym"][1][rows], qo)},
           "rel_err_vs_oracle": {"mixed_sl": rel(res["mixed"][0][rows], vo),
                                 "mixed_dl": rel(res["mixed"][1][rows], qo),
                                 "fp64_sl": rel(res["fp64"][0][rows], vo), "fp64_dl": rel(res["fp64"][1][rows], qo),
                                 "oracle_rows": len(rows)}}
    rec["mixed_over_fp64"] = rec["mixed"]["Gpairs_per_s"] / rec["fp64"]["Gpairs_per_s"]
    rec["mixed_cuda_cores_over_fp64"] = rec["mixed_cuda_cores"]["Gpairs_per_s"] / rec["fp64"]["Gpairs_per_s"]
    rec["mixed_over_fp64_symmetric"] = rec["mixed"]["Gpairs_per_s"] / rec["fp64_symmetric"]["Gpairs_per_s"]
    if solve:
        g = 1.0 / np.linalg.norm(nodes - np.array([0.0, 0.0, 3.0]), axis=1)
        b = m.dirichlet_rhs(g)
        t0 = time.perf_counter()
        [(x, st)] = eb.solve([(m, b)], tol=1e-8)
        rec["solve"] = {"seconds": time.perf_counter() - t0, **st[0]}
    m.close()
    return rec


def run_large(args):
    import torch
    _, _, local = dist_env()
    torch.cuda.set_device(local)
    rec = large_record(local, solve=True)
    line = {"metric": METRIC, "workload": "large", "value": rec["mixed"]["Gpairs_per_s"], "unit": "Gpairs/s",
            "higher_is_better": True, "data": "synthetic", "config": {"workload": rec.pop("workload")}, **rec}
    print(json.dumps(line), flush=True)


def small_record(local):
    """Icosphere L3 (1,280 triangles): Dirichlet solve, g = 1/|x - (0,0,3)|, checked against the reference."""
    import easybem_b200 as eb
    from easybem_b200 import meshes
    from oracle import oracle as O
    nodes, elems = meshes.icosphere(3)
    g = 1.0 / np.linalg.norm(nodes - np.array([0.0, 0.0, 3.0]), axis=1)

    def once():
        t0 = time.perf_counter()
        m = eb.Mesh(nodes, elems)
        b = m.dirichlet_rhs(g)
        [(x, st)] = eb.solve([(m, b)], tol=1e-8)
        return time.perf_counter() - t0, m, x, st

    t_cold, m, x, st = once()  # includes the process's first kernel loads and memory-pool set-up
    m.close()
    t_gpu, m, x, st = once()
    rel = lambda a, c: float(np.linalg.norm(a - c) / np.linalg.norm(c))
    rec = {"workload": "unit icosphere L3 (1,280 triangles, 642 vertices), Dirichlet g = 1/|x-(0,0,3)|, "
                       "mesh + right-hand side + GMRES-IR solve to 1e-8",
           "ms": 1e3 * t_gpu, "cold_ms": 1e3 * t_cold, "solve": st[0]}
    rng = np.random.default_rng(0)
    dens = rng.normal(size=elems.shape[0])
    if O.ref_available():
        t0 = time.perf_counter()
        V, K, D, M = O.ref_dense(nodes, elems, ORDER)
        x_ref = np.linalg.solve(V, (0.5 * M + K) @ g)
        rec["reference_cpu_dense_s"] = time.perf_counter() - t0
        rec["rel_err_solution_vs_reference"] = rel(x, x_ref)
        rec["rel_err_matvec_vs_reference"] = rel(m.apply_sl(dens), V @ dens)
    m.close()
    return rec


def run_small(args):
    import torch
    _, _, local = dist_env()
    torch.cuda.set_device(local)
    rec = small_record(local)
    line = {"metric": METRIC, "workload": "small", "value": rec["ms"], "unit": "ms (mesh + RHS + solve)",
            "higher_is_better": False, "data": "synthetic", "config": {"workload": rec.pop("workload")}, **rec}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "matvec":
        {"batch": run_batch, "serve": run_serve, "large": run_large, "small": run_small}[args.workload](args)
        return
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    import easybem_b200 as eb
    from easybem_b200 import _lib

    nodes, elems, t, u = make_problem(args.level)
    ne, nv = elems.shape[0], nodes.shape[0]
    mesh = eb.Mesh(nodes, elems, ORDER)
    pairs = mesh.far_quad_pairs
    dev = torch.device("cuda", local)
    st = torch.cuda.current_stream()
    d_t = torch.from_numpy(t).to(dev)
    d_u = torch.from_numpy(u).to(dev)
    d_v = torch.empty(ne, dtype=torch.float64, device=dev)
    d_q = torch.empty(ne, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def apply(prec):
        mesh.apply_device(d_t.data_ptr(), d_u.data_ptr(), d_v.data_ptr(), d_q.data_ptr(), precision=prec,
                          stream=st.cuda_stream)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(prec, steps, warmup, sampler=None):
        for _ in range(warmup):
            apply(prec)
        mesh.set_profiling(True)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        far_ms = []
        barrier()
        ctx = sampler if sampler is not None else _Null()
        with ctx:
            for k in range(steps):
                flush.zero_()  # L2 flush between timed steps (outside the events)
                starts[k].record(st)
                apply(prec)
                ends[k].record(st)
                far_ms.append(mesh.last_kernel_ms())  # syncs on this step's events
            barrier()
        mesh.set_profiling(False)
        ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
        return ms, far_ms

    # launch plan: tuned on this mesh before any timing (untimed setup). The plan is the work split
    # of the ordered-pair kernels (the FP64 apply and the CUDA-core engine); the symmetric engine's
    # work list does not depend on it, so the tuning times the CUDA-core engine.
    mesh.set_far_engine("cuda")
    plan = None if args.no_autotune else mesh.autotune(precision="mixed", operators="sl+dl", reps=2)
    mesh.set_far_engine(args.far_engine)
    plan_info = dict(mesh.plan(), tuned=plan is not None)
    if plan is not None:
        plan_info.update(tuned_ms=plan["ms"], default_ms=plan["start_ms"])

    # headline: mixed precision, device-resident inputs
    sampler = ClockSampler(local)
    ms_mixed, far_mixed = timed("mixed", args.steps, args.warmup, sampler)
    v_mixed = d_v.cpu().numpy()
    q_mixed = d_q.cpu().numpy()
    # plain FP64 beside it (fewer steps: it is ~3x slower)
    k64 = max(2, args.steps // 3)
    ms_fp64, far_fp64 = timed("fp64", k64, 1)
    v_64 = d_v.cpu().numpy()
    q_64 = d_q.cpu().numpy()
    # FP64 on the symmetric kernel too (opt-in engine): the same formulation in both precisions
    mesh.set_far_engine("sym_all")
    ms_fp64s, far_fp64s = timed("fp64", k64, 1)
    v_64s = d_v.cpu().numpy()
    q_64s = d_q.cpu().numpy()
    mesh.set_far_engine(args.far_engine)
    # the other far-field engines of the mixed apply, same plan
    others = {}
    for other in ENGINES:
        if other == args.far_engine:
            continue
        mesh.set_far_engine(other)
        ms_o, far_o = timed("mixed", max(2, args.steps // 3), 1)
        others[other] = (ms_o, far_o, d_v.cpu().numpy(), d_q.cpu().numpy())
    mesh.set_far_engine(args.far_engine)

    step_ms = max_over_ranks(sum(ms_mixed) / len(ms_mixed), dist, dev)
    step_ms64 = max_over_ranks(sum(ms_fp64) / len(ms_fp64), dist, dev)
    step_ms64s = max_over_ranks(sum(ms_fp64s) / len(ms_fp64s), dist, dev)
    value = replica_throughput(world, pairs, step_ms)
    value64 = replica_throughput(world, pairs, step_ms64)
    value64s = replica_throughput(world, pairs, step_ms64s)

    # e2e through the host-buffer C ABI with pinned host memory
    h_t = torch.from_numpy(t).pin_memory()
    h_u = torch.from_numpy(u).pin_memory()
    h_v = torch.empty(ne, dtype=torch.float64).pin_memory()
    h_q = torch.empty(ne, dtype=torch.float64).pin_memory()
    import ctypes
    L = _lib.lib()
    P = lambda x: ctypes.c_void_p(x.data_ptr())
    for _ in range(max(1, args.warmup)):
        _lib.check(L.eb_apply_sl_dl(mesh.handle, 1, P(h_t), P(h_u), P(h_v), P(h_q)))
    barrier()
    e2e_times = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        a = time.perf_counter()
        _lib.check(L.eb_apply_sl_dl(mesh.handle, 1, P(h_t), P(h_u), P(h_v), P(h_q)))
        e2e_times.append(time.perf_counter() - a)
    barrier()
    e2e_s = max_over_ranks(sum(e2e_times) / len(e2e_times), dist, dev)
    e2e_value = replica_throughput(world, pairs, 1e3 * e2e_s)

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # accuracy against the CPU oracle on sampled rows (same inputs)
    from oracle.oracle import Oracle
    rng = np.random.default_rng(5)
    rows = np.sort(rng.choice(ne, 24, replace=False)).astype(np.int32)
    vo, qo = Oracle(ORDER).apply_rows(nodes, elems, t, u, rows)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    err = {"mixed_sl": rel(v_mixed[rows], vo), "mixed_dl": rel(q_mixed[rows], qo),
           "fp64_sl": rel(v_64[rows], vo), "fp64_dl": rel(q_64[rows], qo),
           "mixed_vs_fp64_full_sl": rel(v_mixed, v_64), "mixed_vs_fp64_full_dl": rel(q_mixed, q_64),
           "oracle_rows": len(rows)}

    # roofline of the dominant kernel (far field), event-timed on its stream
    far_avg = sum(f for f, _ in far_mixed) / len(far_mixed)
    fin_avg = sum(g for _, g in far_mixed) / len(far_mixed)
    peak_tflops, peak_rsqrt = _measure_peak()
    costs = {e: _engine_costs(e) for e in ENGINES}
    mufu_pp, fma_pp, tc_pp = costs[args.far_engine]
    pair_rate = pairs / (far_avg * 1e-3)
    # pipe rates at this pair rate, and the pair rate the measured pipe peaks allow
    fma_tflops = pair_rate * 2 * fma_pp / 1e12
    mufu = pair_rate * mufu_pp / 1e12
    pair_bound = min(peak_tflops * 1e12 / (2 * fma_pp), peak_rsqrt * 1e12 / mufu_pp)
    cell_far, cell_near = mesh.cell_pairs()
    nb = ctypes.c_longlong()
    _lib.check(L.eb_mesh_finalize_bytes(mesh.handle, ctypes.byref(nb)))
    near_bytes = nb.value  # near-field CSR + gathered densities + far partial sums + outputs
    nb_spmv, nb_fold = ctypes.c_longlong(), ctypes.c_longlong()
    _lib.check(L.eb_mesh_near_field_bytes(mesh.handle, ctypes.byref(nb_spmv), ctypes.byref(nb_fold)))
    cpu = None if args.no_cpu_baseline else cpu_reference_sample(nodes, elems, t, u)
    clocks = sampler.summary()
    extras = {}
    if world == 1 and not args.no_extras:
        torch.cuda.synchronize()
        for name, fn in (("small", small_record), ("batch", batch_record), ("large", large_record)):
            a = time.perf_counter()
            extras[name] = fn(local)
            extras[name]["record_wall_s"] = time.perf_counter() - a
    serve = None
    if args.serve_sample > 0 and world == 1:
        from easybem_b200.serving import run_stream
        serve = run_stream(serve_stream(args.serve_sample), budget_bytes=120 * 10 ** 9, tol=1e-8,
                           rhs_precision=args.rhs_precision)
        serve.pop("results", None)
    line = {
        "metric": METRIC, "value": value, "unit": "Gpairs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 far field / f64 near field", "data": "synthetic",
        "config": {"workload": WORKLOAD.format(level=args.level, ne=ne, nv=nv), "triangles": ne, "vertices": nv, "quad_pairs_per_step": pairs,
                   "near_pairs": mesh.near_pairs, "parallelism": f"replicas x{world}", "plan": plan_info,
                   "l2": "flushed between timed steps (256 MB write)"},
        "fp64": {"value": value64, "unit": "Gpairs/s", "ms_per_step": step_ms64, "steps": len(ms_fp64),
                 "far_ms": sum(f for f, _ in far_fp64) / len(far_fp64)},
        "mixed_over_fp64": value / value64,
        "fp64_symmetric": {"value": value64s, "unit": "Gpairs/s", "ms_per_step": step_ms64s,
                           "far_ms": sum(f for f, _ in far_fp64s) / len(far_fp64s),
                           "rel_err_vs_oracle": {"sl": rel(v_64s[rows], vo), "dl": rel(q_64s[rows], qo)},
                           "note": "the FP64 apply on the symmetric kernel (opt-in EB_FAR_SYMMETRIC_ALL); the "
                                   "'fp64' record is the plain ordered-pair FP64 kernel, the FP64 default"},
        "mixed_over_fp64_symmetric": value / value64s,
        "far_engine": args.far_engine,
        "pair_count_note": ("value counts the apply's ordered quadrature-point pairs (quad_pairs_per_step) per "
                            "second; the symmetric engine evaluates each unordered pair of two different "
                            "128-triangle tiles once and adds it to both rows, so it runs about half as many "
                            "kernel evaluations (the FP64 default and the CUDA-core engine evaluate every "
                            "ordered pair)"),
        "other_engines": {e: {"ms_per_step": sum(o[0]) / len(o[0]),
                              "far_ms": sum(f for f, _ in o[1]) / len(o[1]),
                              "Gpairs_per_s": pairs / (sum(f for f, _ in o[1]) / len(o[1]) * 1e-3) / 1e9,
                              "mixed_over_fp64": (pairs / (sum(o[0]) / len(o[0]) * 1e-3) / 1e9) / value64
                              if value64 else None,
                              "rel_err_vs_oracle": {"sl": rel(o[2][rows], vo), "dl": rel(o[3][rows], qo)},
                              "kernel": ENGINE_KERNELS[e]}
                          for e, o in others.items()},
        "near_cell_share": cell_near / (cell_far + cell_near),
        "rel_err_vs_oracle": err,
        "e2e": {"value": e2e_value, "unit": "Gpairs/s", "h2d_bytes_per_step": 8 * (ne + nv),
                "d2h_bytes_per_step": 16 * ne, "ms_per_step": 1e3 * e2e_s},
        "gpu_launches": (4 if args.far_engine == "tensor" else 3) * args.steps,
        "roofline": {"bound": ENGINE_BOUNDS[args.far_engine],
                     "achieved": pair_rate / 1e9, "peak": pair_bound / 1e9, "unit": "Gpairs/s",
                     "frac": pair_rate / pair_bound,
                     "traffic": (FAR_SYM_TRAFFIC_L6 if args.level == LEVEL and args.far_engine == "sym" else
                                 FAR_TRAFFIC_L6 if (args.level == LEVEL and args.far_engine == "cuda"
                                                    and plan_info.get("items_per_sm") == FAR_TRAFFIC_PLAN) else None),
                     "traffic_unit": "bytes per launch",
                     "kernel": ENGINE_KERNELS[args.far_engine],
                     "far_ms": far_avg,
                     "per_pair": {"mufu_rsqrt": mufu_pp, "fma_pipe_ops": fma_pp, "tensor_flops": tc_pp},
                     "fma": {"achieved": fma_tflops, "peak": peak_tflops, "unit": "TFLOP/s",
                             "frac": fma_tflops / peak_tflops if peak_tflops else None},
                     "mufu": {"achieved": mufu, "peak": peak_rsqrt, "unit": "Trsqrt/s",
                              "frac": mufu / peak_rsqrt if peak_rsqrt else None},
                     "tensor_tflops_tf32": pair_rate * tc_pp / 1e12,
                     "peak_source": "FFMA-chain and MUFU rsqrt-chain calibration kernels measured in this run; "
                                    "peak = the pair rate those two measured pipe peaks allow at the kernel's "
                                    "per-pair pipe work (eb_far_engine_costs)"},
        "near_field": {"kernel": "finalize_kernel<1,1> (near-field SpMV + partial-sum fold)",
                       "finalize_ms": fin_avg, "algorithmic_bytes": near_bytes,
                       "spmv_bytes": nb_spmv.value, "fold_bytes": nb_fold.value,
                       "note": "one launch does both the SL+DL near-field SpMV (spmv_bytes: CSR row pointers, "
                               "columns, values, gathered densities, outputs) and the fold of the far-field "
                               "partial sums (fold_bytes); GB/s counts both over the launch's event time",
                       "GB/s": near_bytes / (fin_avg * 1e-3) / 1e9 if fin_avg > 0 else None,
                       "hbm_peak_GB/s": _hbm_peak(), "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
        "clocks": clocks,
    }
    if cpu is not None:
        line["cpu_baseline"] = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if serve is not None:
        line["serve_sample"] = {"requests": serve["requests"], "p50_ms": serve["p50_ms"], "p99_ms": serve["p99_ms"],
                                "p50_solve_ms": serve["p50_solve_ms"], "p99_solve_ms": serve["p99_solve_ms"],
                                "p99_queue_ms": serve["p99_queue_ms"], "wall_s": serve["wall_s"],
                                "solves_per_s": serve["solves_per_s"], "rhs_per_s": serve["rhs_per_s"],
                                "converged": serve["converged"], "right_hand_sides": serve["right_hand_sides"],
                                "max_rel_residual": serve["max_rel_residual"], "iterations_mean": serve["iterations_mean"],
                                "rhs_precision": args.rhs_precision, "server": serve["server"],
                                "note": "first requests of the 2,000-request Poisson stream (200/s, 120 GB budget); "
                                        "full stream: bench.py --workload serve"}
    for name, rec in extras.items():
        line[name] = rec
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def _hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh).get("hbm_gbs")
    except (OSError, ValueError):
        return None


def _engine_costs(engine):
    import ctypes
    from easybem_b200 import _lib
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.lib().eb_far_engine_costs({"cuda": 0, "tensor": 1, "sym": 2}[engine], ctypes.byref(a), ctypes.byref(b),
                                              ctypes.byref(c)))
    return a.value, b.value, c.value


def _measure_peak():
    import ctypes
    from easybem_b200 import _lib
    tf, rs, s = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    _lib.check(_lib.lib().eb_measure_fp32_peak(ctypes.byref(tf), ctypes.byref(s)))
    _lib.check(_lib.lib().eb_measure_rsqrt_peak(ctypes.byref(rs), ctypes.byref(s)))
    return tf.value, rs.value


if __name__ == "__main__":
    main()
