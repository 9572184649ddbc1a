"""CPU tests that pin the oracle's gauge action, gauge force and expAH
(oracle/hmc_oracle.c, QEX's gaugeAction1 / gaugeForce / expAH).

Pinned by: the free-field action -(6 plaq + 12 rect) V, finite differences
of the action along su(3) generators against the force
(dS/deps = Re Tr[T^dagger F] for U -> exp(eps T) U), expAH against scipy's
expm and its unitarity, and the group property of the link update."""
import numpy as np
import pytest
import scipy.linalg

from oracle import oracle as O
from qex_b200 import fields as F

DIMS = [(4, 4, 4, 4), (4, 6, 4, 8)]


@pytest.mark.parametrize("dims", DIMS)
def test_free_field_action(dims):
    V = F.volume(dims)
    u = np.broadcast_to(np.eye(3, dtype=complex), (4, V, 3, 3)).copy()
    assert abs(O.gauge_action(dims, u, 5.6) + 6 * 5.6 * V) < 1e-9
    assert abs(O.gauge_action(dims, u, 2.0, -0.3) + (6 * 2.0 - 12 * 0.3) * V) < 1e-9
    assert np.abs(O.gauge_force(dims, u, 5.6, 0.4)).max() < 1e-14


@pytest.mark.parametrize("rect", [0.0, -5.6 / 12])
@pytest.mark.parametrize("dims", DIMS)
def test_force_is_the_derivative_of_the_action(dims, rect):
    V = F.volume(dims)
    rng = np.random.default_rng(3)
    u = F.gauge_warm(dims, 0.5, 4)
    plaq = 5.6 * (1 - 8 * rect / 5.6) if rect else 5.6
    f = O.gauge_force(dims, u, plaq, rect)
    # the action is ~1e4: its rounding (~1e-11) over 2 eps bounds the
    # difference from below, the eps^2 truncation from above
    # along all 8 generators on 64 seeded (site, direction) entries
    eps = 1e-4
    entries = set()
    while len(entries) < 64:
        entries.add((int(rng.integers(0, 4)), int(rng.integers(0, V))))
    gens = F.su3_generators()
    for mu, x in sorted(entries):
        for a, T in enumerate(gens):
            vals = []
            for e in (eps, -eps):
                up = u.copy()
                up[mu, x] = scipy.linalg.expm(e * T) @ u[mu, x]
                vals.append(O.gauge_action(dims, up, plaq, rect))
            fd = (vals[0] - vals[1]) / (2 * eps)
            an = np.trace(np.conj(T).T @ f[mu, x]).real
            assert abs(fd - an) < 2e-6 * max(1.0, abs(an)), (mu, x, a, fd, an)
    # traceless anti-Hermitian
    assert np.abs(f + np.conj(np.swapaxes(f, -1, -2))).max() < 1e-13
    assert np.abs(np.trace(f, axis1=-2, axis2=-1)).max() < 1e-13


def test_exp_ah_matches_expm_and_is_unitary():
    rng = np.random.default_rng(5)
    t = F.rand_tah(200, rng)
    for eps in (0.01, 0.3, 2.5):
        e = O.exp_ah(t, eps)
        ref = np.stack([scipy.linalg.expm(eps * m) for m in t])
        assert np.abs(e - ref).max() < 1e-13
        assert np.abs(np.conj(np.swapaxes(e, -1, -2)) @ e - np.eye(3)).max() < 1e-13


def test_link_update_group_property():
    rng = np.random.default_rng(6)
    u = F.warm_su3(50, 0.7, rng).reshape(50, 3, 3)
    p = F.rand_tah(50, rng)
    a = O.link_update(O.link_update(u, p, 0.1), p, 0.2)
    b = O.link_update(u, p, 0.3)
    assert np.abs(a - b).max() < 1e-13


def test_action_against_explicit_loops():
    """sum_{x, mu>nu} Re Tr P and sum_{x, mu!=nu} Re Tr R (long side mu),
    formed loop by loop in numpy, give the oracle's action."""
    dims = (4, 4, 6, 4)
    u = F.gauge_warm(dims, 0.6, 9)
    c = F.coords(dims)

    def sh(f, steps):
        x = c.copy()
        for mu, n in steps:
            x[:, mu] = (x[:, mu] + n) % dims[mu]
        return f[F.index_of(dims, x)]

    def dag(m):
        return np.conj(np.swapaxes(m, -1, -2))

    sp = sr = 0.0
    for mu in range(4):
        for nu in range(4):
            if mu == nu:
                continue
            if mu > nu:
                p = u[mu] @ sh(u[nu], [(mu, 1)]) @ dag(sh(u[mu], [(nu, 1)])) @ dag(u[nu])
                sp += np.trace(p, axis1=-2, axis2=-1).real.sum()
            r = (u[mu] @ sh(u[mu], [(mu, 1)]) @ sh(u[nu], [(mu, 2)]) @ dag(sh(u[mu], [(mu, 1), (nu, 1)]))
                 @ dag(sh(u[mu], [(nu, 1)])) @ dag(u[nu]))
            sr += np.trace(r, axis1=-2, axis2=-1).real.sum()
    for plaq, rect in ((5.6, 0.0), (1.3, -0.4)):
        want = -(plaq * sp + rect * sr) / 3.0
        assert abs(O.gauge_action(dims, u, plaq, rect) - want) < 1e-10 * abs(want)
