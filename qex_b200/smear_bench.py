"""HISQ link smearing on one GPU: device time of each stage and of the whole
HisqCoefs.smear on a thin SU(3) field with staggered phases.

  python -m qex_b200.smear_bench [--dims 32,32,32,32] [--reps 5]

Stages (one call each through the C ABI on device fields, CUDA events on the
library's stream): fat7 with the first-level coefficients (one-link, 3-, 5-,
7-staple), projectU, fat7 with the second-level coefficients (adds Lepage)
plus the Naik product, and the whole smear.  Reported per stage: ms,
algorithmic HBM bytes per site (each link or staple field read and written
once: sweep 1 reads U and writes 12 3-staple fields and fl, sweep 2 reads U,
the 3-staples and fl and writes 24 5-staple fields and fl, sweep 3 reads U,
the 5-staples and fl and writes fl; 144 B per FP64 link) and the achieved
GB/s, plus QEX's flop count (61632 per site per makeImpLinks,
src/gauge/fat7l.nim:106) as GF/s.
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import fields as F
from . import smear as SM
from . import stag as S

LINK = 144
# bytes per site of each stage, all four directions
FAT7_FULL = 4 * LINK * (1 + 3 + 1) + 4 * LINK * (1 + 3 + 1 + 6 + 1) + 4 * LINK * (1 + 6 + 2)
PROJECT = 2 * 4 * LINK
NAIK = 2 * 4 * LINK
QEX_FLOPS_FAT7 = 61632
# adjoint of one fat7 level: sweep A reads M and U, writes 12 T7 fields;
# sweep B reads M, U, T7, writes 12 M3 fields; sweep C reads M, U, M3, T7,
# the 12 S3 and 24 S5 forward fields and writes the derivative
ADJ_FULL = 4 * LINK * (2 + 3) + 4 * LINK * (2 + 3 + 3) + 4 * LINK * (2 + 3 + 3 + 3 + 6 + 1)
ADJ_NAIK = 4 * LINK  # the long-link chain, read once more by sweep C
PROJECT_DERIV = 4 * LINK * 4  # reads v, w, the chain; writes the result


def timed(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ts = []
    for _ in range(reps):
        ev[0].record()
        fn()
        ev[1].record()
        torch.cuda.synchronize()
        ts.append(ev[0].elapsed_time(ev[1]) * 1e-3)
    return float(np.median(ts))


def run(dims, reps):
    import torch
    S.init(0)
    # the library issues on the legacy default stream; torch's events record
    # there too
    V = F.volume(dims)
    lay = S.Layout(dims)
    g = S.to_device_links(F.apply_phases(dims, F.gauge_warm(dims, 0.3, 17)))
    sm = SM.Smear(lay)
    coef = SM.newHISQ()
    t1, w, fl, ll = (torch.empty_like(g) for _ in range(4))
    out = {"dims": dims, "V": V, "stages": {}}

    def stage(name, fn, bytes_site, flops_site):
        t = timed(fn, reps)
        out["stages"][name] = {"ms": t * 1e3, "bytes_per_site": bytes_site, "GBps": bytes_site * V / t * 1e-9,
                               "qex_GFps": flops_site * V / t * 1e-9 if flops_site else None}

    stage("fat7_first", lambda: sm.makeImpLinks(t1, g, coef.fat7first), FAT7_FULL, QEX_FLOPS_FAT7)
    stage("projectU", lambda: sm.projectU(w, t1), PROJECT, 4 * 646)
    stage("fat7_second_naik", lambda: sm.makeImpLinks(fl, w, coef.fat7second, ll, w, coef.naik),
          FAT7_FULL + NAIK, QEX_FLOPS_FAT7)
    stage("hisq_smear", lambda: sm.smear(coef, g, fl, ll), 2 * FAT7_FULL + PROJECT + NAIK, 2 * QEX_FLOPS_FAT7)
    # chain rule (smearGetForce's smearedForce) for Gaussian chains on the fat
    # and long links: forward smear with the second level's staples, the
    # second level's adjoint (+ Naik), projectU's, the first level's staples
    # again and its adjoint
    gen = torch.Generator(device="cuda").manual_seed(5)
    cf = torch.complex(torch.randn(g.shape, dtype=torch.float64, device="cuda", generator=gen),
                       torch.randn(g.shape, dtype=torch.float64, device="cuda", generator=gen))
    cl = cf.flip(0).contiguous()
    d = torch.empty_like(g)
    deriv_bytes = 3 * FAT7_FULL + PROJECT + 2 * ADJ_FULL + ADJ_NAIK + PROJECT_DERIV
    stage("hisq_deriv", lambda: sm.smearDeriv(coef, g, cf, cl, d), deriv_bytes, None)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="32,32,32,32")
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    print(json.dumps(run(tuple(int(v) for v in a.dims.split(",")), a.reps)))


if __name__ == "__main__":
    main()
