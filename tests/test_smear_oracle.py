"""CPU tests that pin the oracle's HISQ smearing (smear_oracle.c, QEX's
makeImpLinks / projectU / HisqCoefs.smear).

QEX stores no smeared-link vectors, so the restatement is pinned by known
answers: the free-field values of fat7 on phased unit links (each staple of
a phased unit field is -2 times the phases, since every plaquette of
staggered phases is -1), the Naik product of phases, projectU against an
independent eigen-decomposition, and gauge covariance of every stage.
"""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import fields as F

SHAPES = [(4, 4, 4, 4), (4, 6, 4, 8)]


def phased_unit(dims):
    V = F.volume(dims)
    return O.apply_phases(dims, np.broadcast_to(np.eye(3, dtype=complex), (4, V, 3, 3)).copy())


def fwd(dims, mu, hop):
    c = F.coords(dims).copy()
    c[:, mu] = (c[:, mu] + hop) % dims[mu]
    return F.index_of(dims, c)


def gauge_transform(dims, u, gt, hop=1):
    """u_mu(x) -> g(x) u_mu(x) g(x + hop mu)^dagger"""
    out = np.empty_like(u)
    for mu in range(4):
        out[mu] = gt @ u[mu] @ np.conj(np.swapaxes(gt[fwd(dims, mu, hop)], -1, -2))
    return out


def test_hisq_coefficients_are_qex_values():
    first, second, naik = O.hisq_coefs()
    assert first == [1 / 8, -1 / 16, 1 / 64, -1 / 384, 0.0]
    assert second == [1.0, -1 / 16, 1 / 64, -1 / 384, -1 / 8]
    assert naik == -1 / 24


@pytest.mark.parametrize("dims", SHAPES)
def test_free_field_known_answers(dims):
    ph = phased_unit(dims)
    first, second, _ = O.hisq_coefs()
    # c1 + 6 cL - 6 c3 + 24 c5 - 48 c7 times the phases
    for c in (first, second, [0.3, 0.2, -0.1, 0.05, 0.07]):
        want = c[0] + 6 * c[4] - 6 * c[1] + 24 * c[2] - 48 * c[3]
        fl = O.fat7(dims, c, ph)
        assert np.abs(fl - want * ph).max() < 1e-14
    fl, ll = O.hisq_smear(dims, ph)
    assert np.abs(fl - 9 / 8 * ph).max() < 1e-14
    for mu in range(4):
        prod = ph[mu] @ ph[mu][fwd(dims, mu, 1)] @ ph[mu][fwd(dims, mu, 2)]
        assert np.abs(ll[mu] + prod / 24).max() < 1e-15


def test_project_u_matches_eigendecomposition():
    rng = np.random.default_rng(5)
    x = rng.normal(size=(500, 3, 3)) + 1j * rng.normal(size=(500, 3, 3))
    w = O.project_u(x)
    h = np.conj(np.swapaxes(x, -1, -2)) @ x
    e, v = np.linalg.eigh(h)
    want = x @ (v * e[:, None, :] ** -0.5) @ np.conj(np.swapaxes(v, -1, -2))
    assert np.abs(w - want).max() < 1e-11
    eye = np.conj(np.swapaxes(w, -1, -2)) @ w - np.eye(3)
    assert np.abs(eye).max() < 1e-12
    # a unitary matrix is its own projection
    u = F.warm_su3(50, 1.0, rng).reshape(50, 3, 3)
    assert np.abs(O.project_u(u) - u).max() < 1e-13


@pytest.mark.parametrize("dims", SHAPES)
def test_gauge_covariance(dims):
    V = F.volume(dims)
    rng = np.random.default_rng(7)
    g = O.apply_phases(dims, F.gauge_warm(dims, 0.5, 3))
    gt = F.warm_su3(V, 1.0, rng).reshape(V, 3, 3)
    coefs = [0.3, 0.2, -0.1, 0.05, 0.07]
    fl = O.fat7(dims, coefs, g)
    fl2 = O.fat7(dims, coefs, gauge_transform(dims, g, gt))
    assert np.abs(fl2 - gauge_transform(dims, fl, gt)).max() < 1e-13
    fl, ll = O.hisq_smear(dims, g)
    fl2, ll2 = O.hisq_smear(dims, gauge_transform(dims, g, gt))
    assert np.abs(fl2 - gauge_transform(dims, fl, gt)).max() < 1e-12
    assert np.abs(ll2 - gauge_transform(dims, ll, gt, 3)).max() < 1e-13


def test_terms_are_separable():
    """fat7 is linear in its coefficients: the sum of single-term smearings
    equals the smearing with all terms (Lepage's c1 shift included)."""
    dims = (4, 4, 4, 4)
    g = O.apply_phases(dims, F.gauge_warm(dims, 0.4, 9))
    c = [0.3, 0.2, -0.1, 0.05, 0.07]
    total = O.fat7(dims, c, g)
    parts = sum(O.fat7(dims, [c[i] if j == i else 0.0 for j in range(5)], g) for i in range(5))
    assert np.abs(total - parts).max() < 1e-14


# ---- chain rule (fat7lDeriv, projectUderiv, smearGetForce) ----------------

def rdot(a, b):
    return float(np.sum((np.conj(a) * b).real))


def test_sylsolve_solves_the_sylvester_equation():
    rng = np.random.default_rng(2)
    a = rng.normal(size=(50, 3, 3)) + 1j * rng.normal(size=(50, 3, 3))
    a = a @ np.conj(np.swapaxes(a, -1, -2)) + 0.1 * np.eye(3)
    c = rng.normal(size=(50, 3, 3)) + 1j * rng.normal(size=(50, 3, 3))
    x = O.sylsolve(a, c)
    assert np.abs(a @ x + x @ a - c).max() < 1e-12 * np.abs(c).max()


def test_project_u_deriv_finite_differences():
    rng = np.random.default_rng(4)
    x = rng.normal(size=(40, 3, 3)) + 1j * rng.normal(size=(40, 3, 3))
    ch = rng.normal(size=x.shape) + 1j * rng.normal(size=x.shape)
    dx = rng.normal(size=x.shape) + 1j * rng.normal(size=x.shape)
    r = O.project_u_deriv(O.project_u(x), x, ch)
    eps = 1e-6
    fd = (rdot(ch, O.project_u(x + eps * dx)) - rdot(ch, O.project_u(x - eps * dx))) / (2 * eps)
    assert abs(fd - rdot(dx, r)) < 1e-8 * abs(fd)


HISQ_CASES = {
    # QEX's own check (hisqsmear.nim:158-168): one-link only, fat7 without
    # Naik, full HISQ
    "oneLink": ([1.0, 0, 0, 0, 0], [1.0, 0, 0, 0, 0], 0.0),
    "fat7": (O.hisq_fat7_coefs(0, 0), O.hisq_fat7_coefs(0, 0), 0.0),
    "hisq": O.hisq_coefs(),
    "lepage+naik": (O.hisq_coefs()[0], [0.5, -0.1, 0.2, -0.03, 0.04], -0.1),
}


@pytest.mark.parametrize("case", sorted(HISQ_CASES))
def test_hisq_chain_rule_finite_differences(case):
    """d/dt S(g + t dg) at t = 0 by central differences (eps 1e-5) against
    sum Re Tr dg^dag deriv, S = sum Re Tr (C^dag fat + Cl^dag long)."""
    dims = (4, 4, 4, 4)
    rng = np.random.default_rng(3)
    g = O.apply_phases(dims, F.gauge_warm(dims, 0.5, 3))
    ch = rng.normal(size=g.shape) + 1j * rng.normal(size=g.shape)
    chl = rng.normal(size=g.shape) + 1j * rng.normal(size=g.shape)
    dg = rng.normal(size=g.shape) + 1j * rng.normal(size=g.shape)
    first, second, cn = coefs = HISQ_CASES[case]

    def S(u):
        w = O.project_u(O.fat7(dims, first, u))
        fl, ll = O.fat7(dims, second, w, w, cn)
        return rdot(ch, fl) + rdot(chl, ll)

    d = O.hisq_deriv(dims, g, ch, chl, coefs=coefs)
    eps = 1e-5
    fd = (S(g + eps * dg) - S(g - eps * dg)) / (2 * eps)
    assert abs(fd - rdot(dg, d)) < 1e-7 * abs(fd)


def test_fat7_deriv_finite_differences_with_naik():
    dims = (4, 4, 4, 6)
    rng = np.random.default_rng(8)
    g = O.apply_phases(dims, F.gauge_warm(dims, 0.5, 3))
    gl = O.apply_phases(dims, F.gauge_warm(dims, 0.4, 5))
    ch = rng.normal(size=g.shape) + 1j * rng.normal(size=g.shape)
    chl = rng.normal(size=g.shape) + 1j * rng.normal(size=g.shape)
    dg = rng.normal(size=g.shape) + 1j * rng.normal(size=g.shape)
    c = [0.3, 0.2, -0.1, 0.05, 0.07]

    def S(u, ul):
        fl, ll = O.fat7(dims, c, u, ul, -0.3)
        return rdot(ch, fl) + rdot(chl, ll)

    d, dl = O.fat7_deriv(dims, c, g, ch, gl, chl, -0.3)
    eps = 1e-5
    fd = (S(g + eps * dg, gl) - S(g - eps * dg, gl)) / (2 * eps)
    assert abs(fd - rdot(dg, d)) < 1e-8 * abs(fd)
    fd = (S(g, gl + eps * dg) - S(g, gl - eps * dg)) / (2 * eps)
    assert abs(fd - rdot(dg, dl)) < 1e-8 * abs(fd)
