"""A short, fixed workload for kernel profilers (ncu -k ... -s 1 -c 1).

    python -m easybem_b200.profile_apply LEVEL ENGINE ITEMS_PER_SM [PRECISION] [OPERATORS]

Creates the radius-perturbed icosphere of the given level (seed 1, the bench's
mesh family), sets the far-field launch plan (ITEMS_PER_SM work items per SM)
and engine ("cuda", "sym", "sym_all" or "tensor"), and runs two applies
(PRECISION "mixed" by default, or "fp64") on seeded densities: the fused SL+DL
apply (OPERATORS "sl+dl", the default) or the single layer alone ("sl").
Each kernel of the apply launches twice: skip the first launch (-s 1) to
capture a warm one.
"""
from __future__ import annotations

import sys

import numpy as np


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    level, engine, ips = int(argv[0]), argv[1], int(argv[2])
    precision = argv[3] if len(argv) > 3 else "mixed"
    operators = argv[4] if len(argv) > 4 else "sl+dl"
    import easybem_b200 as eb
    from easybem_b200 import meshes
    nodes, elems = meshes.perturbed_icosphere(level, seed=1)
    rng = np.random.default_rng(2024)
    t = rng.normal(size=elems.shape[0])
    u = rng.normal(size=nodes.shape[0])
    with eb.Mesh(nodes, elems) as m:
        m.set_plan(ips)
        m.set_far_engine(engine)
        for _ in range(2):
            if operators == "sl":
                v = m.apply_sl(t, precision=precision)
                q = np.zeros(1)
            else:
                v, q = m.apply_sl_dl(t, u, precision=precision)
    print(f"applied: L{level} {engine} {precision} {operators}, |V t|_1 = {np.abs(v).sum():.6e}, "
          f"|K u|_1 = {np.abs(q).sum():.6e}")


if __name__ == "__main__":
    main()
