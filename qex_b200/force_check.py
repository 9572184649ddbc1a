"""Configuration-4 check of the fermion force (the adjoint of the solve).

  python -m qex_b200.force_check [--dims 16,16,16,16] [--mass 0.05] [--entries 64]

On the fat+Naik fields of the 32^4 workload's recipe (fat = 0.8 SU(3) + noise,
long = SU(3), phases folded) and a Gaussian even-site phi, S = phi_e^dagger
A^-1 phi_e with A = stagD2ee(m^2).  For a seeded sample of (site, direction,
fat/long) links and each of the 8 generators T_a = i lambda_a (Gell-Mann),
the central difference of S under W -> exp(+-eps T_a) W (eps = 1e-5, FP64)
is compared with Re Tr[T_a f^dagger]/8, f = qexstag_force (QEX's fermForce
output, whose psi carries QEX's factor 4).  The difference is formed as
<y+, (A- - A+) y->, y+- = A(+-eps)^-1 phi, which avoids cancelling two large
actions.  The whole force is also compared with the oracle's (the C
restatement of QEX's stagForceSolve + fermForce), when --oracle is given.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import fields as F
from . import stag as S


def gell_mann():
    l = np.zeros((8, 3, 3), dtype=np.complex128)
    l[0][0, 1] = l[0][1, 0] = 1
    l[1][0, 1], l[1][1, 0] = -1j, 1j
    l[2][0, 0], l[2][1, 1] = 1, -1
    l[3][0, 2] = l[3][2, 0] = 1
    l[4][0, 2], l[4][2, 0] = -1j, 1j
    l[5][1, 2] = l[5][2, 1] = 1
    l[6][1, 2], l[6][2, 1] = -1j, 1j
    l[7][0, 0] = l[7][1, 1] = 1 / np.sqrt(3)
    l[7][2, 2] = -2 / np.sqrt(3)
    return 1j * l  # anti-Hermitian traceless generators


def run(dims, mass=0.05, entries=64, seed=5, eps=1e-5, oracle=False):
    import torch
    S.init(0)
    V = F.volume(dims)
    h = V // 2
    g = F.fat_naik_links(dims, 21)
    phi = F.even_source(dims, 33)
    gd = S.to_device_links(g)
    s = S.Staggered(S.Layout(dims), gd)
    phid = S.to_device_vector(phi)
    f = torch.zeros_like(gd)
    t0 = time.perf_counter()
    s.force(f, phid, mass, S.SolverParams(r2req=1e-26))
    fh = S.to_host_links(f)
    t_force = time.perf_counter() - t0
    T = gell_mann()
    rng = np.random.default_rng(seed)
    errs, rows = [], []
    t0 = time.perf_counter()
    for _ in range(entries):
        k = int(rng.integers(0, 8))
        x = int(rng.integers(0, V))
        for a in range(8):
            ys = []
            links = []
            for e in (eps, -eps):
                gp = gd.clone()
                u = torch.from_numpy(F.exp_ah(T[a][None], e)[0] @ g[k, x]).to("cuda")
                gp[k, :, :, x] = u
                links.append(gp)
                s.update_links(gp)
                y = torch.zeros_like(phid)
                s.solveEE(y, phid, mass, S.SolverParams(r2req=1e-26))
                ys.append(y)
            s.update_links(links[1])
            am = torch.zeros_like(phid)
            s.stagD2ee(am, ys[1], mass * mass)
            s.update_links(links[0])
            ap = torch.zeros_like(phid)
            s.stagD2ee(ap, ys[1], mass * mass)
            dS = torch.vdot(ys[0][:, :h].reshape(-1), (am - ap)[:, :h].reshape(-1)).real.item()
            fd = dS / (2 * eps)
            an = np.trace(T[a] @ np.conj(fh[k, x]).T).real / 8
            errs.append(abs(fd - an))
            rows.append((k, x, a, fd, an))
    t_fd = time.perf_counter() - t0
    s.update_links(gd)
    scale = max(abs(r[4]) for r in rows)
    out = {"dims": dims, "mass": mass, "entries": entries, "directions": len(rows),
           "max_abs_err": max(errs), "max_abs_derivative": scale,
           "max_rel_err_vs_largest": max(errs) / scale,
           "median_abs_err": float(np.median(errs)), "seconds_force": t_force, "seconds_fd": t_fd}
    if oracle:
        from oracle import oracle as O
        o = O.Oracle(dims, g)
        fo = np.zeros_like(g)
        t0 = time.perf_counter()
        o.force(fo, phi, mass, 1e-26)
        out["oracle_seconds"] = time.perf_counter() - t0
        out["max_rel_diff_vs_oracle"] = float(np.abs(fh - fo).max() / np.abs(fo).max())
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="16,16,16,16")
    ap.add_argument("--mass", type=float, default=0.05)
    ap.add_argument("--entries", type=int, default=64)
    ap.add_argument("--oracle", action="store_true")
    a = ap.parse_args()
    dims = tuple(int(v) for v in a.dims.split(","))
    print(json.dumps(run(dims, a.mass, a.entries, oracle=a.oracle)))


if __name__ == "__main__":
    main()
