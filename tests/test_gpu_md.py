"""GPU parity of the molecular-dynamics kernels (gauge action and force,
link update, momenta) against the oracle, and of the device-side MD driver
(qex_b200/md.py) against the torch-glue HMC of tests/hmc_harness.py on the same
fields and momenta."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu
DIMS = [(4, 6, 4, 8), (8, 8, 8, 8)]


def dev(g):
    return S.to_device_links(g)


def host(t):
    return S.to_host_links(t)


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("dims", DIMS)
def test_gauge_kernels_match_oracle(cuda, dims):
    torch = cuda
    from qex_b200 import md
    lay = S.Layout(dims)
    u = F.gauge_warm(dims, 0.5, 11)
    ud = dev(u)
    for beta, c1 in ((5.6, 0.0), (4.8, -1.0 / 12)):
        ga = md.GaugeAction(lay, beta, c1)
        plaq, rect = ga.c.plaq, ga.c.rect
        a = ga.action(ud)
        ao = O.gauge_action(dims, u, plaq, rect)
        assert abs(a - ao) < 1e-12 * abs(ao)
        f = torch.empty_like(ud)
        ga.force(ud, f)
        assert rel(host(f), O.gauge_force(dims, u, plaq, rect)) < 1e-12
    rng = np.random.default_rng(3)
    p = F.rand_tah(4 * lay.V, rng).reshape(4, lay.V, 3, 3)
    pd = dev(p)
    u2 = ud.clone()
    md.link_update(lay, u2, pd, 0.37)
    assert rel(host(u2), O.link_update(u, p, 0.37)) < 1e-13
    t = md.kinetic_action(lay, pd)
    assert abs(t - (0.5 * np.sum(np.abs(p) ** 2) - 16 * lay.V)) < 1e-9 * lay.V
    q = pd.clone()
    md.momenta_update(lay, q, pd, -0.25)
    assert rel(host(q), 0.75 * p) < 1e-15


def test_momenta_heatbath(cuda):
    torch = cuda
    from qex_b200 import md
    dims = (16, 16, 16, 16)
    lay = S.Layout(dims)
    p = torch.empty((4, 3, 3, lay.V), dtype=torch.complex128, device="cuda")
    md.momenta_heatbath(lay, p, 1234, 0)
    h = host(p)
    assert np.abs(h + np.conj(np.swapaxes(h, -1, -2))).max() == 0.0
    assert np.abs(np.trace(h, axis1=-2, axis2=-1)).max() < 1e-15
    n2 = np.sum(np.abs(h) ** 2, axis=(-1, -2))
    # randTah3: E|p|^2 = 8 per link, variance of the sum of 8 chi^2(1)/... terms
    assert abs(n2.mean() - 8.0) < 0.02
    off = h[..., 0, 1]
    assert abs(off.real.var() - 0.5) < 0.01 and abs(off.real.mean()) < 0.005
    q = torch.empty_like(p)
    md.momenta_heatbath(lay, q, 1234, 0)
    assert torch.equal(p, q)
    md.momenta_heatbath(lay, q, 1234, 1)
    assert not torch.equal(p, q)
    assert abs(md.kinetic_action(lay, p)) < 5 * np.sqrt(4 * lay.V * 16)


def test_pure_gauge_md_matches_torch_hmc(cuda):
    torch = cuda
    import hmc_harness as hmc
    from qex_b200 import md
    dims = (8, 8, 8, 8)
    lay = S.Layout(dims)
    lat = hmc.Lattice(dims)
    U0 = torch.from_numpy(F.gauge_warm(dims, 0.3, 41)).to("cuda")
    p0 = hmc.random_momenta(lat, np.random.default_rng(7))
    h = hmc.HMC(lat, 5.6, None)
    H0 = h.hamiltonian(U0, p0)
    U1, p1 = h.leapfrog(U0, p0, 0.5, 10)
    H1 = h.hamiltonian(U1, p1)
    m = md.MD(lay, md.GaugeAction(lay, 5.6))
    U = U0.permute(0, 2, 3, 1).contiguous()
    P = p0.permute(0, 2, 3, 1).contiguous()
    assert abs(m.hamiltonian(U, P) - H0) < 1e-9 * abs(H0)
    m.leapfrog(U, P, 0.5, 10)
    assert abs(m.hamiltonian(U, P) - H1) < 1e-9 * abs(H1)
    assert (U.permute(0, 3, 1, 2) - U1).abs().max().item() < 1e-11


@pytest.mark.parametrize("hisq", [True, False])
def test_md_with_fermion_matches_torch_hmc(cuda, hisq):
    """One pseudofermion: the HISQ operator, or the thin-link fat + Naik
    operator written as one-link-only smearing.  Same U, p and phi as
    qex_b200/hmc.py's trajectory; dH agrees and the trajectory reverses."""
    torch = cuda
    import hmc_harness as hmc
    from qex_b200 import md
    dims = (8, 8, 8, 8)
    lay = S.Layout(dims)
    lat = hmc.Lattice(dims)
    U0 = torch.from_numpy(F.gauge_warm(dims, 0.3, 43)).to("cuda")
    ref = hmc.trajectory_with_reversal(lat, U0, 5.6, 0.1, -1.0 / 24.0, 0.5, 10, seed=7, sloppy=S.L.SLOPPY_NONE,
                                       r2req_action=1e-24, r2req_force=1e-24, hisq=hisq)
    ferm = md.StaggeredPseudofermion(lay, 0.1, hisq=hisq, r2req_action=1e-24, r2req_force=1e-24,
                                     sloppy=S.L.SLOPPY_NONE)
    Ud = U0.permute(0, 2, 3, 1).contiguous()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    ferm.heatbath(Ud, gen)
    p0 = hmc.random_momenta(lat, np.random.default_rng(7)).permute(0, 2, 3, 1).contiguous()
    out = md.trajectory_with_reversal(lay, Ud, 5.6, 0.5, 10, fermion=ferm, P0=p0)
    assert abs(out["H0"] - ref["H0"]) < 1e-9 * abs(ref["H0"])
    assert abs(out["dH"] - ref["dH"]) < 1e-6 * max(1.0, abs(ref["dH"])), (out, ref)
    assert abs(out["dH_reversed"]) < 1e-5 and out["max_dU"] < 1e-7, out


def test_omelyan_second_order_and_hmc_loop(cuda):
    """QEX's default integrator 2MN (Omelyan): dH falls as eps^2 (halving
    the step divides it by about 4), the trajectory reverses, and at equal
    force evaluations its error is below leapfrog's.  The HMC loop
    (momenta and pseudofermion heatbath, MD, Metropolis) runs and records
    every trajectory."""
    torch = cuda
    from qex_b200 import md
    dims = (8, 8, 8, 8)
    lay = S.Layout(dims)
    U0 = dev(F.gauge_warm(dims, 0.2, 5))
    P0 = torch.empty_like(U0)
    md.momenta_heatbath(lay, P0, 21, 0)
    m = md.MD(lay, md.GaugeAction(lay, 5.6))
    h0 = m.hamiltonian(U0, P0)
    dh = {}
    for integ, n in (("omelyan", 4), ("omelyan", 8), ("leapfrog", 8)):
        U, P = U0.clone(), P0.clone()
        m.integrate(U, P, 1.0, n, integ)
        dh[(integ, n)] = m.hamiltonian(U, P) - h0
        if (integ, n) == ("omelyan", 8):
            P.neg_()
            m.integrate(U, P, 1.0, n, integ)
            assert abs(m.hamiltonian(U, P) - h0) < 1e-8 * abs(h0)
            assert float((U - U0).abs().max()) < 1e-10
    ratio = dh[("omelyan", 4)] / dh[("omelyan", 8)]
    assert 3.0 < ratio < 5.5, dh
    assert abs(dh[("omelyan", 4)]) < abs(dh[("leapfrog", 8)]), dh
    ferm = md.StaggeredPseudofermion(lay, 0.2, hisq=False)
    U, rec = md.hmc(lay, U0, 5.6, ferm, 2, nsteps=6, integrator="omelyan")
    assert len(rec) == 2 and all(np.isfinite(r["dH"]) for r in rec)
    assert all(0.0 < r["plaquette"] < 1.0 for r in rec)
