"""GPU parity of the HISQ smearing kernels (qexstag_fat7, qexstag_project_u,
qexstag_hisq_smear, qexstag_links_hisq) against the oracle's restatement of
QEX's makeImpLinks / projectU / smear, through the C ABI.  FP64 with a
different order of accumulation: tolerance 1e-12 relative (max-norm)."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import smear as SM
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu
TOL = 1e-12
SHAPES = [(4, 4, 4, 4), (6, 4, 8, 4), (8, 8, 8, 8)]
GENERIC = [0.3, 0.2, -0.1, 0.05, 0.07]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def thin(dims, seed=3, eps=0.5):
    return O.apply_phases(dims, F.gauge_warm(dims, eps, seed))


@pytest.mark.parametrize("dims", SHAPES)
def test_fat7_all_terms_host(cuda, dims):
    g = thin(dims)
    sm = SM.Smear(S.Layout(dims))
    for c in (GENERIC, O.hisq_coefs()[0], O.hisq_coefs()[1], [0.5, 0.0, 0.0, 0.0, 0.0], [0.1, 0.3, 0.0, 0.0, 0.0]):
        fl = np.empty_like(g)
        sm.makeImpLinks(fl, g, SM.Fat7lCoefs(*c))
        assert rel(fl, O.fat7(dims, c, g)) < TOL, c


@pytest.mark.parametrize("dims", SHAPES[:2])
def test_fat7_with_naik_host_and_device(cuda, dims):
    torch = cuda
    g = thin(dims, 4)
    gl = thin(dims, 5, 0.3)
    ofl, oll = O.fat7(dims, GENERIC, g, gl, -1 / 24)
    sm = SM.Smear(S.Layout(dims))
    fl, ll = np.empty_like(g), np.empty_like(g)
    sm.makeImpLinks(fl, g, SM.Fat7lCoefs(*GENERIC), ll, gl, -1 / 24)
    assert rel(fl, ofl) < TOL and rel(ll, oll) < TOL
    gd, gld = S.to_device_links(g), S.to_device_links(gl)
    fd, ld = torch.empty_like(gd), torch.empty_like(gd)
    sm.makeImpLinks(fd, gd, SM.Fat7lCoefs(*GENERIC), ld, gld, -1 / 24)
    assert np.array_equal(S.to_host_links(fd), fl)
    assert np.array_equal(S.to_host_links(ld), ll)


def test_project_u(cuda):
    dims = (4, 4, 4, 6)
    g = thin(dims)
    x = O.fat7(dims, O.hisq_coefs()[0], g)
    sm = SM.Smear(S.Layout(dims))
    w = np.empty_like(x)
    sm.projectU(w, x)
    assert rel(w, O.project_u(x)) < TOL
    eye = np.conj(np.swapaxes(w, -1, -2)) @ w - np.eye(3)
    assert np.abs(eye).max() < 1e-12


@pytest.mark.parametrize("dims", SHAPES)
def test_hisq_smear_matches_oracle(cuda, dims):
    g = thin(dims, 6)
    ofl, oll = O.hisq_smear(dims, g)
    fl, ll = SM.hisq_smear(S.Layout(dims), g)
    assert rel(fl, ofl) < TOL
    assert rel(ll, oll) < TOL


def test_hisq_free_field(cuda):
    dims = (4, 4, 4, 8)
    V = F.volume(dims)
    ph = O.apply_phases(dims, np.broadcast_to(np.eye(3, dtype=complex), (4, V, 3, 3)).copy())
    fl, ll = SM.hisq_smear(S.Layout(dims), ph)
    assert np.abs(fl - 9 / 8 * ph).max() < 1e-14
    _, oll = O.hisq_smear(dims, ph)
    assert np.abs(ll - oll).max() < 1e-15


def test_links_hisq_operator(cuda):
    """Smearing into a fat+Naik handle gives the Dslash of the oracle's
    smeared links; a second smear of new thin links replaces them."""
    torch = cuda
    dims = (8, 4, 4, 8)
    V = F.volume(dims)
    lay = S.Layout(dims)
    sm = SM.Smear(lay)
    coef = SM.newHISQ()
    x = F.gaussian_vector(V, 12)
    stag = S.Staggered(lay, np.zeros((8, V, 3, 3), complex) + np.eye(3), long_coeff=-1 / 24)
    for seed in (7, 8):
        g = thin(dims, seed)
        sm.smear_into(stag, coef, S.to_device_links(g) if seed == 8 else g)
        ofl, oll = O.hisq_smear(dims, g)
        o = O.Oracle(dims, F.interleave(ofl, oll))
        a, b = np.zeros_like(x), np.zeros_like(x)
        stag.D(a, x, 0.05)
        o.D(b, x, 0.05)
        assert rel(a, b) < TOL
        # mixed solves still converge on the smeared (non-SU(3)) long links
        y = np.zeros_like(x)
        stag.solve(y, x, 0.05, S.SolverParams(r2req=1e-20, sloppySolve=L.SLOPPY_HALF))
        o.D(b, y, 0.05)
        assert np.linalg.norm(b - x) ** 2 / np.linalg.norm(x) ** 2 <= 1e-20
    assert not stag.recon12


def test_smear_errors(cuda):
    dims = (4, 4, 4, 4)
    lay = S.Layout(dims)
    sm = SM.Smear(lay)
    g = thin(dims)
    naive = S.Staggered(lay, g)
    with pytest.raises(L.QexStagError) as e:
        sm.smear_into(naive, SM.newHISQ(), g)
    assert e.value.code == L.ERR_ARG
    lib = L.load()
    assert lib.qexstag_hisq_smear(None, None, None, None, None, 0) == L.ERR_ARG
    with pytest.raises(ValueError):
        sm.projectU(np.empty((4, 10, 3, 3), complex), g)


# ---- chain rule ------------------------------------------------------------

def chains(g, seed):
    rng = np.random.default_rng(seed)
    return tuple(rng.normal(size=g.shape) + 1j * rng.normal(size=g.shape) for _ in range(2))


@pytest.mark.parametrize("dims", SHAPES[:2])
def test_fat7_deriv_matches_oracle(cuda, dims):
    g = thin(dims, 4)
    gl = thin(dims, 5, 0.3)
    ch, chl = chains(g, 6)
    sm = SM.Smear(S.Layout(dims))
    c = SM.Fat7lCoefs(*GENERIC)
    # without Naik; adds to what deriv holds
    pre = chains(g, 7)[0]
    d = pre.copy()
    sm.fat7Deriv(d, g, ch, c)
    od, _ = O.fat7_deriv(dims, GENERIC, g, ch)
    assert rel(d - pre, od) < TOL
    # Naik on a separate field
    d, dl = np.zeros_like(g), np.zeros_like(g)
    sm.fat7Deriv(d, g, ch, c, dl, gl, chl, -0.3)
    od, odl = O.fat7_deriv(dims, GENERIC, g, ch, gl, chl, -0.3)
    assert rel(d, od) < TOL and rel(dl, odl) < TOL
    # Naik on the same field (HISQ's second level)
    d = np.zeros_like(g)
    sm.fat7Deriv(d, g, ch, c, d, g, chl, -0.3)
    assert rel(d, od + O.fat7_deriv(dims, GENERIC, g, ch * 0, g, chl, -0.3)[1]) < TOL


def test_project_u_deriv_matches_oracle(cuda):
    dims = (4, 4, 4, 6)
    x = O.fat7(dims, O.hisq_coefs()[0], thin(dims, 3))
    u = O.project_u(x)
    ch, _ = chains(x, 9)
    sm = SM.Smear(S.Layout(dims))
    r = np.empty_like(x)
    sm.projectUderiv(r, u, x, ch)
    assert rel(r, O.project_u_deriv(u, x, ch)) < 1e-11


DERIV_CASES = {
    "hisq": (None, None),
    "fat7": ((0.0, 0.0), (0.0, 0.0)),
    "lepage+naik": (None, [0.5, -0.1, 0.2, -0.03, 0.04]),
}


@pytest.mark.parametrize("case", sorted(DERIV_CASES))
@pytest.mark.parametrize("dims", SHAPES)
def test_hisq_deriv_matches_oracle(cuda, dims, case):
    torch = cuda
    g = thin(dims, 6)
    cf, cl = chains(g, 11)
    coef = SM.newHISQ()
    first, second, cn = O.hisq_coefs()
    f2, s2 = DERIV_CASES[case]
    if f2 is not None:
        first, second, cn = O.hisq_fat7_coefs(*f2), O.hisq_fat7_coefs(*s2), 0.0
        coef.fat7first, coef.fat7second, coef.naik = SM.Fat7lCoefs(*first), SM.Fat7lCoefs(*second), 0.0
    elif s2 is not None:
        second, cn = s2, -0.1
        coef.fat7second, coef.naik = SM.Fat7lCoefs(*second), cn
    od = O.hisq_deriv(dims, g, cf, cl, coefs=(first, second, cn))
    sm = SM.Smear(S.Layout(dims))
    d = np.empty_like(g)
    sm.smearDeriv(coef, g, cf, cl, d)
    assert rel(d, od) < 1e-11
    if dims == SHAPES[0]:
        dd = torch.empty_like(S.to_device_links(g))
        sm.smearDeriv(coef, S.to_device_links(g), S.to_device_links(cf), S.to_device_links(cl), dd)
        assert np.array_equal(S.to_host_links(dd), d)


# ---- HISQ fermion force ------------------------------------------------------

def oracle_hisq_force(dims, thin, phi, m):
    """QEX's force with HISQ smearing, composed from the oracle's pieces."""
    fl, ll = O.hisq_smear(dims, thin)
    o = O.Oracle(dims, F.interleave(fl, ll))
    psi = o.vec()
    o.force_solve(psi, phi, m, 1e-26)
    f8 = np.zeros((8,) + thin.shape[1:], complex)
    o.ferm_outer(f8, psi)
    ff = O.hisq_deriv(dims, thin, f8[0::2], f8[1::2])
    m = (ff @ np.conj(np.swapaxes(thin, -1, -2))).reshape(-1, 3, 3)
    return np.stack([O.project_tah(x) for x in m]).reshape(thin.shape)


def test_hisq_force_matches_oracle(cuda):
    dims = (4, 6, 4, 8)
    V = F.volume(dims)
    lay = S.Layout(dims)
    thin_links = thin(dims, 12, 0.4)
    phi = F.gaussian_vector(V, 13)
    phi[V // 2:] = 0
    stag = S.Staggered(lay, np.zeros((8, V, 3, 3), complex) + np.eye(3))
    sm = SM.Smear(lay)
    f = np.empty_like(thin_links)
    sp = S.SolverParams(r2req=1e-26)
    sm.force(stag, SM.newHISQ(), thin_links, f, phi, 0.2, sp)
    fo = oracle_hisq_force(dims, thin_links, phi, 0.2)
    assert rel(f, fo) < 1e-10
    # the operator now holds the smeared links
    ofl, oll = O.hisq_smear(dims, thin_links)
    o = O.Oracle(dims, F.interleave(ofl, oll))
    x = F.gaussian_vector(V, 14)
    a, b = np.zeros_like(x), np.zeros_like(x)
    stag.D(a, x, 0.2)
    o.D(b, x, 0.2)
    assert rel(a, b) < TOL


def test_hisq_force_finite_differences(cuda):
    """S = phi_e^dag A^-1 phi_e, A = stagD2ee(m^2) of the HISQ-smeared thin
    links; along W -> exp(t T_a) W on one thin link, dS/dt = Re Tr[T_a
    f^dag]/8 (f carries QEX's factor 4 in psi and S_QEX = 2 S)."""
    torch = cuda
    dims = (4, 4, 4, 6)
    V = F.volume(dims)
    h = V // 2
    m = 0.2
    lay = S.Layout(dims)
    g = thin(dims, 15, 0.4)
    phi = F.gaussian_vector(V, 16)
    phi[h:] = 0
    stag = S.Staggered(lay, np.zeros((8, V, 3, 3), complex) + np.eye(3))
    sm = SM.Smear(lay)
    coef = SM.newHISQ()
    f = np.empty_like(g)
    sm.force(stag, coef, g, f, phi, m, S.SolverParams(r2req=1e-26))
    T = F.su3_generators()
    rng = np.random.default_rng(17)
    eps = 1e-5
    worst, scale = 0.0, 0.0
    for _ in range(6):
        mu, x = int(rng.integers(0, 4)), int(rng.integers(0, V))
        for a in (0, 3, 7):
            ys, gs = [], []
            for e in (eps, -eps):
                gp = g.copy()
                gp[mu, x] = F.exp_ah(T[a][None], e)[0] @ g[mu, x]
                gs.append(gp)
                sm.smear_into(stag, coef, gp)
                y = np.zeros_like(phi)
                stag.solveEE(y, phi, m, S.SolverParams(r2req=1e-26))
                ys.append(y)
            am, ap = np.zeros_like(phi), np.zeros_like(phi)
            sm.smear_into(stag, coef, gs[1])
            stag.stagD2ee(am, ys[1], m * m)
            sm.smear_into(stag, coef, gs[0])
            stag.stagD2ee(ap, ys[1], m * m)
            fd = np.vdot(ys[0][:h], (am - ap)[:h]).real / (2 * eps)
            an = np.trace(T[a] @ np.conj(f[mu, x]).T).real / 8
            worst = max(worst, abs(fd - an))
            scale = max(scale, abs(an))
    assert worst < 1e-6 * scale
