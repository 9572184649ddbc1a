"""GPU checks of the force path and the HMC glue (configuration 4 shapes):
fermForce outer products against the oracle, the adjoint against finite
differences through a torch.autograd harness and along su(3) generators,
and an HMC trajectory's energy conservation and reversibility."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_ferm_outer_and_force_solve_match_oracle(cuda):
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 9)
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    psi = F.gaussian_vector(V, 3)
    fo, fg = np.zeros_like(g), np.zeros_like(g)
    o.ferm_outer(fo, psi)
    s.ferm_outer(fg, psi)
    assert rel(fg, fo) < 1e-14
    phi = F.even_source(dims, 4)
    po, pg = o.vec(), o.vec()
    o.force_solve(po, phi, 0.05, 1e-24)
    s.force_solve(pg, phi, 0.05, S.SolverParams(r2req=1e-24))
    assert rel(pg, po) < 1e-9


def test_links_update_matches_new_handle(cuda):
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g1, g2 = F.fat_naik_links(dims, 1), F.fat_naik_links(dims, 2)
    s = S.Staggered(S.Layout(dims), g1)
    s.update_links(g2)
    t = S.Staggered(S.Layout(dims), g2)
    x = F.gaussian_vector(V, 5)
    a, b = np.zeros_like(x), np.zeros_like(x)
    s.D(a, x, 0.1)
    t.D(b, x, 0.1)
    assert np.array_equal(a, b)
    for sp in (S.L.SLOPPY_SINGLE, S.L.SLOPPY_HALF):  # rebuilt reduced copies
        ya, yb = np.zeros_like(x), np.zeros_like(x)
        s.solveEE(ya, F.even_source(dims, 6), 0.1, S.SolverParams(r2req=1e-20, sloppySolve=sp))
        t.solveEE(yb, F.even_source(dims, 6), 0.1, S.SolverParams(r2req=1e-20, sloppySolve=sp))
        assert np.array_equal(ya, yb)


def test_autograd_harness_directional_derivative(cuda):
    """torch.autograd gradient of S = phi^dagger A^-1 phi (backward = the
    library's adjoint) against a central difference along a random complex
    direction, computed stably as <y+, (A- - A+) y->."""
    torch = cuda
    from qex_b200.autograd import StaggeredAction
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = S.to_device_links(F.fat_naik_links(dims, 11))
    s = S.Staggered(S.Layout(dims), g)
    phi = S.to_device_vector(F.even_source(dims, 12))
    m = 0.1
    W = g.clone().requires_grad_(True)
    Sval = StaggeredAction.apply(W, phi, s, m)
    Sval.backward()
    grad = W.grad
    gen = torch.Generator(device="cuda").manual_seed(3)
    D = torch.complex(torch.randn(g.shape, dtype=torch.float64, device="cuda", generator=gen),
                      torch.randn(g.shape, dtype=torch.float64, device="cuda", generator=gen))
    eps = 1e-5

    def solve(links):
        s.update_links(links.contiguous())
        y = torch.zeros_like(phi)
        s.solveEE(y, phi, m, S.SolverParams(r2req=1e-26))
        return y

    yp, ym = solve(g + eps * D), solve(g - eps * D)
    s.update_links((g - eps * D).contiguous())
    am = torch.zeros_like(phi)
    s.stagD2ee(am, ym, m * m)
    s.update_links((g + eps * D).contiguous())
    ap = torch.zeros_like(phi)
    s.stagD2ee(ap, ym, m * m)
    h = V // 2
    dS = torch.vdot(yp[:, :h].reshape(-1), (am - ap)[:, :h].reshape(-1)).real.item()
    fd = dS / (2 * eps)
    an = (torch.conj(grad) * D).real.sum().item()
    assert abs(fd - an) <= 1e-7 * abs(an), (fd, an)


def test_hmc_trajectory_reversible(cuda):
    """Config-4-shaped trajectories: Wilson beta 5.6 + fat/Naik staggered
    pseudofermion from thin links, leapfrog.  The energy violation falls as
    the square of the step (halving it divides dH by ~4) and the reversed
    trajectory returns to the start."""
    torch = cuda
    import hmc_harness as hmc
    dims = (8, 8, 8, 8)
    lat = hmc.Lattice(dims)
    U0 = torch.from_numpy(F.gauge_warm(dims, 0.3, 41)).to("cuda")
    outs = [hmc.trajectory_with_reversal(lat, U0, 5.6, 0.1, -1.0 / 24.0, 0.5, n, sloppy=S.L.SLOPPY_NONE,
                                         r2req_action=1e-24, r2req_force=1e-24) for n in (10, 20)]
    ratio = outs[0]["dH"] / outs[1]["dH"]
    assert 3.0 < ratio < 5.0, (ratio, outs)
    for out in outs:
        assert out["max_dU"] < 1e-7 and out["max_dp"] < 1e-7, out
        assert abs(out["dH_reversed"]) < 1e-5, out


def test_hmc_force_matches_finite_difference(cuda):
    """The MD force (Wilson + fermion through the Naik chain rule) against a
    central difference of the potential along su(3) generators."""
    torch = cuda
    import hmc_harness as hmc
    dims = (4, 4, 4, 8)
    lat = hmc.Lattice(dims)
    U = torch.from_numpy(F.gauge_warm(dims, 0.3, 5)).to("cuda")
    ferm = hmc.StaggeredFermion(lat, 0.2, -1.0 / 24.0, r2req_action=1e-26, r2req_force=1e-26,
                                sloppy=S.L.SLOPPY_NONE)
    ferm.heatbath(U, torch.Generator(device="cuda").manual_seed(1))
    h = hmc.HMC(lat, 5.6, ferm)
    Fo = h.force(U)
    rng = np.random.default_rng(2)
    eps = 1e-5
    for _ in range(6):
        mu, x = int(rng.integers(0, 4)), int(rng.integers(0, lat.V))
        T = torch.from_numpy(F.rand_tah(1, rng)[0]).to("cuda")
        vals = []
        for e in (eps, -eps):
            Up = U.clone()
            Up[mu, x] = hmc.exp_ah(e * T) @ U[mu, x]
            vals.append(h.potential(Up))
        fd = (vals[0] - vals[1]) / (2 * eps)
        an = torch.trace(T @ hmc.dagger(Fo[mu, x])).real.item()
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1.0), (mu, x, fd, an)


def test_hisq_hmc_force_matches_finite_difference(cuda):
    """HISQ molecular-dynamics force: Wilson plus the pseudofermion of the
    HISQ-smeared operator (qexstag_hisq_force: smearing chain rule through
    fat7, projectU, fat7 + Naik) against a central difference of the
    potential along su(3) generators on the thin links."""
    torch = cuda
    import hmc_harness as hmc
    dims = (4, 4, 4, 8)
    lat = hmc.Lattice(dims)
    U = torch.from_numpy(F.gauge_warm(dims, 0.3, 6)).to("cuda")
    ferm = hmc.StaggeredFermion(lat, 0.2, r2req_action=1e-26, r2req_force=1e-26, sloppy=S.L.SLOPPY_NONE,
                                hisq=True)
    ferm.heatbath(U, torch.Generator(device="cuda").manual_seed(3))
    h = hmc.HMC(lat, 5.6, ferm)
    Fo = h.force(U)
    rng = np.random.default_rng(4)
    eps = 1e-5
    for _ in range(6):
        mu, x = int(rng.integers(0, 4)), int(rng.integers(0, lat.V))
        T = torch.from_numpy(F.rand_tah(1, rng)[0]).to("cuda")
        vals = []
        for e in (eps, -eps):
            Up = U.clone()
            Up[mu, x] = hmc.exp_ah(e * T) @ U[mu, x]
            vals.append(h.potential(Up))
        fd = (vals[0] - vals[1]) / (2 * eps)
        an = torch.trace(T @ hmc.dagger(Fo[mu, x])).real.item()
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1.0), (mu, x, fd, an)


def test_hisq_hmc_trajectory_reversible(cuda):
    """HISQ trajectories (QEX's tgenerichmchisq shape): dH falls as the square
    of the step and the reversed trajectory returns to the start."""
    torch = cuda
    import hmc_harness as hmc
    dims = (8, 8, 8, 8)
    lat = hmc.Lattice(dims)
    U0 = torch.from_numpy(F.gauge_warm(dims, 0.3, 43)).to("cuda")
    outs = [hmc.trajectory_with_reversal(lat, U0, 5.6, 0.1, None, 0.5, n, sloppy=S.L.SLOPPY_NONE,
                                         r2req_action=1e-24, r2req_force=1e-24, hisq=True) for n in (10, 20)]
    ratio = outs[0]["dH"] / outs[1]["dH"]
    assert 3.0 < ratio < 5.0, (ratio, outs)
    for out in outs:
        assert out["max_dU"] < 1e-7 and out["max_dp"] < 1e-7, out
        assert abs(out["dH_reversed"]) < 1e-5, out
