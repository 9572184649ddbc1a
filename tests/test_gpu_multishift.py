"""GPU parity of the multi-shift solvers against the oracle (cgm.nim and the
multi-mass solve of stagSolve.nim)."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("naik", [False, True])
def test_solve_multi_mass_matches_oracle(cuda, naik):
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 3) if naik else F.naive_links(dims, 0.3, 3)
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    b = F.even_source(dims, 71)
    ms = [0.05, 0.1, 0.2, 0.5]
    xo = [o.vec() for _ in ms]
    its_o, _ = o.solve_multishift(xo, b, ms, 1e-20)
    xg = [o.vec() for _ in ms]
    sp = S.SolverParams(r2req=1e-20)
    s.solve_multi(xg, b, ms, sp)
    assert abs(sp.iterations - its_o) <= 1
    for m, a, e in zip(ms, xg, xo):
        assert rel(a, e) < 1e-8
        dx = o.vec()
        o.D(dx, a, m)
        assert np.linalg.norm(dx - b) ** 2 / np.linalg.norm(b) ** 2 < 1e-14


@pytest.mark.parametrize("nrhs", [1, 3])
@pytest.mark.parametrize("sloppy", [L.SLOPPY_NONE, L.SLOPPY_SINGLE, L.SLOPPY_HALF])
def test_cgm_shifts_and_rhs(cuda, sloppy, nrhs):
    """(A + sigma_k) y_jk = b_j for 1 or 3 right-hand sides and 6
    log-spaced shifts, each to the requested FP64 true residual (one
    right-hand side runs the single-vector sloppy Schur and refines with the
    reliable-update CG)."""
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 5)
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    m = 0.01
    sig = list(np.logspace(-4, 0, 6))
    bs = [F.even_source(dims, 80 + j) for j in range(nrhs)]
    ys = [[o.vec() for _ in sig] for _ in bs]
    sp = S.SolverParams(r2req=1e-18, sloppySolve=sloppy)
    r2 = s.cgm_ee(m, sig, bs, ys, sp)
    assert sp.status == L.OK
    assert (r2 <= 1e-18).all()
    for j, b in enumerate(bs):
        for k, sg in enumerate(sig):
            ay = o.vec()
            o.stagD2ee(ay, ys[j][k], m * m)
            ay += sg * ys[j][k]
            h = V // 2
            res = np.linalg.norm(ay[:h] - b[:h]) ** 2 / np.linalg.norm(b[:h]) ** 2
            assert res <= 1e-18, (j, k, res)
            assert not np.any(ys[j][k][h:])
    # against the oracle's multi-shift CG for one right-hand side
    xo = [o.vec() for _ in sig]
    sg0 = [x - sig[0] for x in sig]
    o.cgm(0, xo, sg0, bs[-1], m * m + 0.25 * sig[0], 1e-22)
    for k in range(len(sig)):
        assert rel(ys[-1][k], xo[k]) < 1e-7
