"""Configuration-3 run: many independent small lattices in one persistent
launch against one solve per lattice.

  python -m qex_b200.batched_bench [--n 64] [--r2req 1e-20]

64 naive staggered problems with dims drawn (seeded) from {8^4, 12^4, 16^4,
8^3 x 16}, each with its own SU(3) field U = warmSU(eps), eps ~ U[0.1, 0.5],
mass ~ U[0.02, 0.2] and Gaussian even source; every problem solved to a
true FP64 relative residual of 1e-10.  Reports the device time of one
qexstag_solve_batched call (graph launch, after the autotuning call) and of
the same solves one problem at a time with qexstag_solveEE.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import fields as F
from . import stag as S

SHAPES = [(8, 8, 8, 8), (12, 12, 12, 12), (16, 16, 16, 16), (8, 8, 8, 16)]


def problem_set(n=64, seed=2024):
    """The seeded problem set: per problem (dims, phased links (4, V, 3, 3),
    mass, even source), host arrays in QEX's V=1 order."""
    rng = np.random.default_rng(seed)
    probs = []
    for i in range(n):
        dims = SHAPES[int(rng.integers(0, len(SHAPES)))]
        eps = float(rng.uniform(0.1, 0.5))
        m = float(rng.uniform(0.02, 0.2))
        g = F.apply_phases(dims, F.gauge_warm(dims, eps, 1000 + i))
        probs.append((dims, g, m, F.even_source(dims, 2000 + i)))
    return probs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--r2req", type=float, default=1e-20)
    a = ap.parse_args()
    import torch
    S.init(0)
    t0 = time.perf_counter()
    stags, bs, ms, dims_list = [], [], [], []
    for dims, g, m, b in problem_set(a.n):
        stags.append(S.Staggered(S.Layout(dims), S.to_device_links(g)))
        bs.append(S.to_device_vector(b))
        ms.append(m)
        dims_list.append(dims)
    setup = time.perf_counter() - t0
    xs = [torch.zeros_like(b) for b in bs]
    res = {}
    for rep in ("tune", "warm", "timed"):
        sp = S.SolverParams(r2req=a.r2req)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = S.solve_batched(stags, xs, bs, ms, sp)
        torch.cuda.synchronize()
        res[rep] = {"wall": time.perf_counter() - t0, "device": sp.seconds}
    seq = {}
    for rep in ("warm", "timed"):
        tot_dev, tot_its = 0.0, 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s, b, m in zip(stags, bs, ms):
            y = torch.zeros_like(b)
            sp = S.SolverParams(r2req=a.r2req)
            s.solveEE(y, b, m, sp)
            tot_dev += sp.seconds
            tot_its += sp.iterations
        torch.cuda.synchronize()
        seq[rep] = {"wall": time.perf_counter() - t0, "device": tot_dev, "iterations": tot_its}
    sites = sum(F.volume(d) for d in dims_list)
    print(json.dumps({
        "n": a.n, "total_sites": sites, "setup_seconds": setup,
        "batched": {"seconds": res["timed"]["device"], "wall": res["timed"]["wall"],
                    "first_call_with_tuning": res["tune"]["wall"],
                    "block": out["block"], "blocks_per_sm": out["blocks_per_sm"], "graph": out["graph"],
                    "iterations_total": int(sum(out["iterations"])),
                    "iterations_max": int(max(out["iterations"])), "max_true_r2": float(out["r2"].max())},
        "one_at_a_time": {"seconds": seq["timed"]["device"], "wall": seq["timed"]["wall"],
                          "iterations_total": seq["timed"]["iterations"]},
        "speedup": seq["timed"]["wall"] / res["timed"]["wall"]}))


if __name__ == "__main__":
    main()
