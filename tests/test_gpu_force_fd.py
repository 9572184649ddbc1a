"""The staggered fermion force at the size of the force workload: 16^4,
fat+Naik fields of the solver workload's recipe (fat = 0.8 SU(3) + Gaussian
noise of std 0.2, long = SU(3), phases folded in), m = 0.05, Gaussian phi on
even sites.

S = phi_e^dagger A^-1 phi_e with A = stagD2ee(m^2) (QEX's action up to its
factor 2; stagForceSolve + fermForce, src/hmc/hmcAction.nim:669-790).  For
64 seeded (site, direction, fat/long) links and each of the 8 generators
T_a = i lambda_a, the central difference of S under W -> exp(+-eps T_a) W
(eps = 1e-5, FP64) equals Re Tr[T_a f^dagger]/8, f = qexstag_force (whose psi
carries QEX's factor 4).  The difference is formed as <y+, (A- - A+) y->,
y+- = A(+-eps)^-1 phi, which avoids cancelling two large actions.  The whole
force is also compared with the oracle's (the C restatement of QEX's
stagForceSolve + fermForce).
"""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu

DIMS = (16, 16, 16, 16)
MASS = 0.05
ENTRIES = 64
EPS = 1e-5
FD_TOL = 1e-8       # |FD - force| relative to the largest derivative sampled
ORACLE_TOL = 1e-10  # force against the oracle's, relative to its largest entry
R2REQ = 1e-26


@pytest.fixture(scope="module")
def force16(cuda):
    torch = cuda
    g = F.fat_naik_links(DIMS, 21)
    phi = F.even_source(DIMS, 33)
    gd = S.to_device_links(g)
    s = S.Staggered(S.Layout(DIMS), gd)
    phid = S.to_device_vector(phi)
    f = torch.zeros_like(gd)
    s.force(f, phid, MASS, S.SolverParams(r2req=R2REQ))
    return {"g": g, "phi": phi, "gd": gd, "s": s, "phid": phid, "f": S.to_host_links(f)}


def test_force_matches_oracle_16x16x16x16(force16):
    o = O.Oracle(DIMS, force16["g"])
    fo = np.zeros_like(force16["g"])
    o.force(fo, force16["phi"], MASS, R2REQ)
    assert np.abs(force16["f"] - fo).max() / np.abs(fo).max() < ORACLE_TOL


def test_force_finite_differences_16x16x16x16(cuda, force16):
    torch = cuda
    g, gd, s, phid, fh = force16["g"], force16["gd"], force16["s"], force16["phid"], force16["f"]
    V = F.volume(DIMS)
    h = V // 2
    T = F.su3_generators()
    rng = np.random.default_rng(5)
    errs, ans = [], []
    kinds = set()
    for _ in range(ENTRIES):
        k = int(rng.integers(0, 8))  # link 2 mu: fat, 2 mu + 1: long
        x = int(rng.integers(0, V))
        kinds.add(k & 1)
        for a in range(8):
            ys, links = [], []
            for e in (EPS, -EPS):
                gp = gd.clone()
                gp[k, :, :, x] = torch.from_numpy(F.exp_ah(T[a][None], e)[0] @ g[k, x]).to("cuda")
                links.append(gp)
                s.update_links(gp)
                y = torch.zeros_like(phid)
                s.solveEE(y, phid, MASS, S.SolverParams(r2req=R2REQ))
                ys.append(y)
            s.update_links(links[1])
            am = torch.zeros_like(phid)
            s.stagD2ee(am, ys[1], MASS * MASS)
            s.update_links(links[0])
            ap = torch.zeros_like(phid)
            s.stagD2ee(ap, ys[1], MASS * MASS)
            dS = torch.vdot(ys[0][:, :h].reshape(-1), (am - ap)[:, :h].reshape(-1)).real.item()
            fd = dS / (2 * EPS)
            an = np.trace(T[a] @ np.conj(fh[k, x]).T).real / 8
            errs.append(abs(fd - an))
            ans.append(abs(an))
    s.update_links(gd)
    assert kinds == {0, 1}  # fat and long links both sampled
    assert len(errs) == 8 * ENTRIES
    assert max(errs) <= FD_TOL * max(ans)
