"""Configuration-2 run: multi-shift solves for a rational term.

  python -m qex_b200.multishift_bench [--dims 24,24,24,48] [--nrhs 8] [--nshift 12]
                                      [--mass 0.01] [--r2req 1e-18] [--sloppy 0,1,2]

(A + sigma_k) y_jk = b_j on even sites, A = stagD2ee(m^2), fat+Naik fields of
the 32^4 workload's recipe, sigma_k = 10^(-4 + 4k/(nshift-1)), Gaussian b_j,
per-shift tolerance r2req (1e-18 = relative residual 1e-9).  Reports, per
inner precision, the device time of qexstag_cgm_ee (multi-shift phase with
the multi-right-hand-side Dslash, FP64 true residuals, refinement), the
iterations and the worst FP64 true residual over all (j, k).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import fields as F
from . import stag as S


def shifts(nshift=12):
    """sigma_k = 10^(-4 + 4k/(nshift-1)): log-spaced from 1e-4 to 1."""
    return [10.0 ** (-4 + 4 * k / (nshift - 1)) for k in range(nshift)]


def run(dims, nrhs, nshift, mass, r2req, sloppies):
    import torch
    S.init(0)
    V = F.volume(dims)
    t0 = time.perf_counter()
    g = F.fat_naik_links(dims, 21)
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    del g
    sig = shifts(nshift)
    bs = [S.to_device_vector(F.even_source(dims, 100 + j)) for j in range(nrhs)]
    ys = [[torch.zeros((3, V), dtype=torch.complex128, device="cuda") for _ in sig] for _ in bs]
    out = {"dims": dims, "nrhs": nrhs, "nshift": nshift, "mass": mass, "r2req": r2req,
           "setup_seconds": time.perf_counter() - t0, "runs": {}}
    for sl in sloppies:
        for rep in ("warm", "timed"):
            sp = S.SolverParams(r2req=r2req, sloppySolve=sl)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r2 = s.cgm_ee(mass, sig, bs, ys, sp)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
        out["runs"][{0: "fp64", 1: "fp32", 2: "16bit"}[sl]] = {
            "seconds": sp.seconds, "wall": wall, "iterations": sp.iterations,
            "refinement_passes": sp.outer_iterations - 1, "reliable_updates": sp.reliable_updates,
            "max_true_r2": float(r2.max()), "launches": sp.kernel_launches}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="24,24,24,48")
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--nshift", type=int, default=12)
    ap.add_argument("--mass", type=float, default=0.01)
    ap.add_argument("--r2req", type=float, default=1e-18)
    ap.add_argument("--sloppy", default="1,2,0")
    a = ap.parse_args()
    dims = tuple(int(v) for v in a.dims.split(","))
    print(json.dumps(run(dims, a.nrhs, a.nshift, a.mass, a.r2req, [int(v) for v in a.sloppy.split(",")])))


if __name__ == "__main__":
    main()
