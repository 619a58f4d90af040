"""Request loop over the continuous-batching server (``easybem_b200.Server``).

``run_stream`` replays a list of requests (dicts with ``t_arrival`` in
seconds, ``nodes``, ``elems``, ``g``) in real time: each request is submitted
when the wall clock reaches its arrival time, the server advances every
running request by one step in between, and finished requests are collected
as they complete. Latency is measured by the server from submission to
completion.
"""
from __future__ import annotations

import time

import numpy as np

from . import Server


def percentile(x, p):
    return float(np.percentile(np.asarray(x, dtype=np.float64), p)) if len(x) else float("nan")


def run_stream(requests, budget_bytes=120 * 10 ** 9, max_systems=4096, keep_results=False, **solve_options):
    srv = Server(budget_bytes=budget_bytes, max_systems=max_systems, **solve_options)
    pending = sorted(requests, key=lambda r: r["t_arrival"])
    ids = []
    done = {}
    t0 = time.perf_counter()
    k = 0
    steps = 0
    while len(done) < len(pending):
        now = time.perf_counter() - t0
        while k < len(pending) and pending[k]["t_arrival"] <= now:
            r = pending[k]
            ids.append(srv.submit(r["nodes"], r["elems"], r["g"]))
            k += 1
        active, waiting = srv.step()
        steps += 1
        for rid in ids:
            if rid in done:
                continue
            st = srv.state(rid)
            if st >= 4:
                if st == 4:
                    t, stats, times = srv.result(rid)
                    done[rid] = dict(stats=stats, times=times, t=t if keep_results else None)
                else:
                    done[rid] = dict(stats=None, times=None, failed=True)
                srv.release(rid)
        if active == 0 and waiting == 0 and k < len(pending):
            time.sleep(max(0.0, min(0.01, pending[k]["t_arrival"] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    counters = srv.stats()
    srv.close()
    ok = [d for d in done.values() if d.get("stats")]
    lat = [d["times"]["latency_ms"] for d in ok]
    nrhs = sum(len(d["stats"]) for d in ok)
    conv = sum(all(s["converged"] and s["rel_residual"] <= solve_options.get("tol", 1e-8) for s in d["stats"])
               for d in ok)
    return {
        "requests": len(pending), "completed": len(ok), "failed": len(pending) - len(ok),
        "converged": conv, "right_hand_sides": nrhs, "wall_s": wall, "steps": steps,
        "solves_per_s": len(ok) / wall, "rhs_per_s": nrhs / wall,
        "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99), "mean_ms": float(np.mean(lat)) if lat else None,
        "p50_solve_ms": percentile([d["times"]["solve_ms"] for d in ok], 50),
        "p99_solve_ms": percentile([d["times"]["solve_ms"] for d in ok], 99),
        "p99_queue_ms": percentile([d["times"]["queue_ms"] for d in ok], 99),
        "max_rel_residual": max((s["rel_residual"] for d in ok for s in d["stats"]), default=None),
        "iterations_mean": float(np.mean([s["iterations"] for d in ok for s in d["stats"]])) if ok else None,
        "server": counters,
        "results": done if keep_results else None,
    }
