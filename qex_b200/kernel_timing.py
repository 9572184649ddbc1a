"""Time the even-parity Schur operator (two Dslash half sweeps) per precision
and report HBM throughput against its compulsory bytes.

  python -m qex_b200.kernel_timing [--dims 32,32,32,32] [--naive]
                                   [--prec 0,1,2] [--nrep 20]
  python -m qex_b200.kernel_timing --solve 2 [--delta 0.1]   (whole solves)

Compulsory bytes per even site of one Schur application (each link read
once per half sweep, each vector once; 12-real long links):
  FP64 fat+Naik  2400 + 2448 = 4848     naive 1248 + 1296 = 2544
  FP32 fat+Naik  1008 + 1032 = 2040     naive  624 +  648 = 1272
  FP16 fat+Naik   512 +  536 = 1048     naive  320 +  344 =  664
(second half sweep: + same-site input and an FP32 output for the sloppy
precisions).
"""
from __future__ import annotations

import argparse
import json

BYTES = {  # (nlinks, prec) -> bytes per even site per Schur call
    (8, 0): 4848, (8, 1): 2040, (8, 2): 1048,
    (4, 0): 2544, (4, 1): 1272, (4, 2): 664,
}
NAMES = {0: "fp64", 1: "fp32", 2: "fp16"}
VEC_BYTES = {0: 48, 1: 24, 2: 16}  # one site of the input vector per precision


def no_reuse_bytes_per_site(nlinks: int, prec: int, recon12: bool = True) -> int:
    """The same count with every neighbour's input vector charged (8 naive or
    16 fat+Naik per output site and half sweep, no cache reuse), the figure
    other staggered codes quote: FP64 fat+Naik 3120 B per half sweep."""
    hops = 16 if nlinks == 8 else 8
    return bytes_per_site(nlinks, prec, recon12) + 2 * (hops - 1) * VEC_BYTES[prec]


def bytes_per_site(nlinks: int, prec: int, recon12: bool = True) -> int:
    b = BYTES[(nlinks, prec)]
    if nlinks == 8 and prec > 0 and not recon12:
        b += 2 * 4 * (2 * 24 if prec == 1 else 2 * 12)  # long links with 18 reals
    return b


def time_schur(stag, nh: int, precs=(0, 1, 2), nrep: int = 20, m2: float = 1e-4):
    out = {}
    for p in precs:
        sec = stag.bench_schur(p, nrep, m2)
        bps = bytes_per_site(stag.nlinks, p, stag.recon12)
        nrb = no_reuse_bytes_per_site(stag.nlinks, p, stag.recon12)
        out[NAMES[p]] = {"seconds": sec, "bytes_per_even_site": bps,
                         "GBps": bps * nh / sec / 1e9,
                         "no_reuse_bytes_per_even_site": nrb, "GBps_no_reuse": nrb * nh / sec / 1e9,
                         "GFLOPs": (2 * (1146 if stag.nlinks == 8 else 570)) * nh / sec / 1e9}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="32,32,32,32")
    ap.add_argument("--naive", action="store_true")
    ap.add_argument("--prec", default="0,1,2")
    ap.add_argument("--nrep", type=int, default=20)
    ap.add_argument("--solve", type=int, default=-1,
                    help="instead: one warm-up and one timed solveEE (m=0.01, r2req 1e-20) "
                         "with this inner precision (0 FP64, 1 FP32, 2 16-bit)")
    ap.add_argument("--delta", type=float, default=0.0,
                    help="reliable-update threshold of the --solve runs (0: the library's default)")
    a = ap.parse_args()
    from . import fields as F
    from . import stag as S
    dims = tuple(int(v) for v in a.dims.split(","))
    S.init(0)
    g = F.naive_links(dims) if a.naive else F.fat_naik_links(dims)
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    del g
    if a.solve >= 0:
        import time

        import torch
        b = S.to_device_vector(F.even_source(dims))
        y = torch.zeros_like(b)
        out = {}
        for rep in ("warm", "timed"):
            sp = S.SolverParams(r2req=1e-20, sloppySolve=a.solve, delta=a.delta)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.solveEE(y, b, 0.01, sp)
            torch.cuda.synchronize()
            out[rep] = {"seconds": time.perf_counter() - t0, "iterations": sp.iterations,
                        "launches": sp.kernel_launches, "reliable_updates": sp.reliable_updates}
        print(json.dumps({"dims": dims, "solve": a.solve, "delta": a.delta, **out}))
        return
    res = time_schur(s, F.volume(dims) // 2, [int(v) for v in a.prec.split(",")], a.nrep)
    print(json.dumps({"dims": dims, "nlinks": s.nlinks, "recon12": s.recon12, "schur": res}))


if __name__ == "__main__":
    main()
