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
