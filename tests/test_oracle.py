"""CPU tests that pin the oracle (the C restatement of QEX's staggered path).

QEX cannot be built here (it is Nim) and stores no Dslash/CG/force golden
vectors, so the oracle is pinned by known answers: QEX's index formula and
shift semantics, the free-field spectrum, antihermiticity, gauge covariance,
the Schur identity, solver residuals and finite differences of the action.
"""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import fields as F

SHAPES = [(4, 4, 4, 4), (4, 6, 4, 8), (8, 4, 6, 4)]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("dims", SHAPES)
def test_index_is_qex_checkerboard(dims):
    V = F.volume(dims)
    c = F.coords(dims)
    seen = np.zeros(V, bool)
    for i in range(0, V, max(1, V // 97)):
        assert O.index(dims, c[i]) == i
    idx = F.index_of(dims, c)
    seen[idx] = True
    assert seen.all()
    # even sites first
    assert ((c[: V // 2].sum(1) & 1) == 0).all()
    assert ((c[V // 2:].sum(1) & 1) == 1).all()


def test_index_golden():
    """Known answers of idx = (lex + (sum x odd) V)/2 on 4^4 (V = 256)."""
    dims = (4, 4, 4, 4)
    assert O.index(dims, (0, 0, 0, 0)) == 0
    assert O.index(dims, (1, 0, 0, 0)) == (1 + 256) // 2
    assert O.index(dims, (2, 0, 0, 0)) == 1
    assert O.index(dims, (0, 1, 0, 0)) == (4 + 256) // 2
    assert O.index(dims, (1, 1, 0, 0)) == 5 // 2
    assert O.index(dims, (3, 3, 3, 3)) == 255 // 2


@pytest.mark.parametrize("dims", SHAPES)
def test_shift_tables(dims):
    V = F.volume(dims)
    c = F.coords(dims)
    for mu in range(4):
        for ln in (1, -1, 3, -3):
            for par in (0, 1, 2):
                t = O.shift_table(dims, mu, ln, par)
                i0 = V // 2 if par == 1 else 0
                i1 = V // 2 if par == 0 else V
                x = c[i0:i1].copy()
                x[:, mu] = (x[:, mu] + ln) % dims[mu]
                assert (F.index_of(dims, x) == t).all()
            # forward then backward is the identity (tests/base/tshift.nim)
            fa = O.shift_table(dims, mu, ln, 2)
            ba = O.shift_table(dims, mu, -ln, 2)
            assert (ba[fa] == np.arange(V)).all()


def test_phase_convention():
    """QEX phases [8,9,11,0]: eta0=(-1)^x3, eta1=(-1)^(x0+x3),
    eta2=(-1)^(x0+x1+x3), eta3=1; setBC negates U3 on the last time slice."""
    dims = (4, 4, 4, 4)
    V = F.volume(dims)
    c = F.coords(dims)
    one = np.zeros((4, V, 3, 3), complex)
    one[:] = np.eye(3)
    g = O.apply_phases(dims, one)
    x0, x1, x2, x3 = c.T
    exp = [(-1.0) ** x3, (-1.0) ** (x0 + x3), (-1.0) ** (x0 + x1 + x3), np.ones(V)]
    exp[3] = np.where(x3 == 3, -1.0, 1.0)
    for mu in range(4):
        assert np.allclose(g[mu][:, 0, 0].real, exp[mu])
    assert np.array_equal(g, F.apply_phases(dims, one))


def _unit_links(dims, naik: bool):
    V = F.volume(dims)
    one = np.zeros((8 if naik else 4, V, 3, 3), complex)
    one[:] = np.eye(3)
    return O.apply_phases(dims, one)


@pytest.mark.parametrize("naik", [False, True])
def test_free_field_spectrum(naik):
    """Unit gauge: A = 4 m^2 - (2D)^2 is diagonal on plane waves with
    eigenvalue 4 m^2 + 4 sum_mu (sin p + [Naik] sin 3p)^2, p_3 antiperiodic."""
    dims = (4, 6, 4, 8)
    V = F.volume(dims)
    c = F.coords(dims)
    o = O.Oracle(dims, _unit_links(dims, naik))
    m = 0.1
    rng = np.random.default_rng(0)
    for _ in range(4):
        n = rng.integers(0, 8, size=4)
        p = 2 * np.pi * n / np.array(dims)
        p[3] = (2 * n[3] + 1) * np.pi / dims[3]
        ph = np.exp(1j * (c @ p))
        col = rng.standard_normal(3) + 1j * rng.standard_normal(3)
        x = np.zeros((V, 3), complex)
        x[: V // 2] = ph[: V // 2, None] * col
        r = o.vec()
        o.stagD2ee(r, x, m * m)
        s = np.sin(p) + (np.sin(3 * p) if naik else 0.0)
        lam = 4 * m * m + 4 * np.sum(s ** 2)
        assert rel(r[: V // 2], lam * x[: V // 2]) < 1e-13
        # the free propagator: solveEE gives x / lam
        y = o.vec()
        its, r2 = o.solveXX(0, y, x, m, 1e-24)
        assert rel(y[: V // 2], x[: V // 2] / lam) < 1e-10


def _links(dims, naik, seed=5):
    return F.fat_naik_links(dims, seed) if naik else F.naive_links(dims, 0.3, seed)


@pytest.mark.parametrize("naik", [False, True])
def test_antihermitian(naik):
    dims = (4, 4, 4, 6)
    V = F.volume(dims)
    o = O.Oracle(dims, _links(dims, naik))
    x = F.gaussian_vector(V, 1)
    y = F.gaussian_vector(V, 2)
    dx, dy = o.vec(), o.vec()
    o.D(dx, x, 0.0)
    o.D(dy, y, 0.0)
    lhs = np.vdot(y, dx)
    rhs = -np.vdot(dy, x)
    assert abs(lhs - rhs) < 1e-13 * abs(lhs)
    # Ddag is the adjoint of D at nonzero mass
    m = 0.3
    o.D(dx, x, m)
    o.Ddag(dy, y, m)
    assert abs(np.vdot(y, dx) - np.vdot(dy, x)) < 1e-12 * abs(np.vdot(y, dx))


@pytest.mark.parametrize("naik", [False, True])
def test_gauge_covariance(naik):
    dims = (4, 4, 6, 4)
    V = F.volume(dims)
    c = F.coords(dims)
    g = _links(dims, naik)
    rng = np.random.default_rng(3)
    gt = F.warm_su3(V, 1.0, rng)
    nl = g.shape[0]
    gp = np.empty_like(g)
    for k in range(nl):
        mu = k // 2 if nl == 8 else k
        hop = (3 if k % 2 else 1) if nl == 8 else 1
        xs = c.copy()
        xs[:, mu] = (xs[:, mu] + hop) % dims[mu]
        j = F.index_of(dims, xs)
        gp[k] = gt @ g[k] @ np.conj(np.swapaxes(gt[j], 1, 2))
    x = F.gaussian_vector(V, 4)
    xp = np.einsum("sab,sb->sa", gt, x)
    o, op = O.Oracle(dims, g), O.Oracle(dims, gp)
    r, rp = o.vec(), op.vec()
    o.D(r, x, 0.2)
    op.D(rp, xp, 0.2)
    assert rel(rp, np.einsum("sab,sb->sa", gt, r)) < 1e-13


@pytest.mark.parametrize("naik", [False, True])
def test_schur_identity(naik):
    """stagD2ee(m2) = 4 m2 - (2D)_eo (2D)_oe, and D(m) Ddag(m) = A/4 on even."""
    dims = (4, 4, 4, 4)
    V = F.volume(dims)
    o = O.Oracle(dims, _links(dims, naik))
    x = F.gaussian_vector(V, 7)
    x[V // 2:] = 0
    m = 0.25
    r = o.vec()
    o.stagD2ee(r, x, m * m)
    t, u = o.vec(), o.vec()
    o.stagD2(1, t, x, 0.0, 0.0)
    o.stagD2(0, u, t, 0.0, 0.0)
    exp = 4 * m * m * x - u
    assert rel(r[: V // 2], exp[: V // 2]) < 1e-13
    a, b = o.vec(), o.vec()
    o.Ddag(a, x, m)
    o.D(b, a, m)
    assert rel(4 * b[: V // 2], r[: V // 2]) < 1e-13


@pytest.mark.parametrize("naik", [False, True])
def test_solvers_meet_residual(naik):
    dims = (4, 4, 4, 8)
    V = F.volume(dims)
    o = O.Oracle(dims, _links(dims, naik))
    m = 0.1
    b = F.gaussian_vector(V, 9)
    r2req = 1e-20
    # solveEE
    y = o.vec()
    its, r2 = o.solveXX(0, y, b, m, r2req)
    ay = o.vec()
    o.stagD2ee(ay, y, m * m)
    res = np.linalg.norm(ay[: V // 2] - b[: V // 2]) ** 2 / np.linalg.norm(b[: V // 2]) ** 2
    assert res <= r2req and abs(res - r2) <= 1e-3 * r2 + 1e-30
    assert not np.any(y[V // 2:])
    # full solve with reconstruction
    x = o.vec()
    its, r2 = o.solve(x, b, m, r2req)
    dx = o.vec()
    o.D(dx, x, m)
    res = np.linalg.norm(dx - b) ** 2 / np.linalg.norm(b) ** 2
    assert res <= r2req


def test_cg_in_steps_equals_one_call():
    """The CPU baseline runs one oracle CG in bounded pieces; the pieces
    give the iterations and solution of a single call (OpenMP sums are not
    bitwise reproducible from run to run, so the solution is compared to
    1e-8)."""
    dims = (4, 4, 4, 8)
    V = F.volume(dims)
    o = O.Oracle(dims, _links(dims, True))
    b = F.gaussian_vector(V, 11)
    m2 = 0.01
    x1 = o.vec()
    its1, r21 = o.cg(0, x1, b, m2, 1e-20)
    x2 = o.vec()
    run = o.cg_steps(0, x2, b, m2, 1e-20)
    steps = 0
    while not run.converged:
        run.run(7)
        steps += 1
    its2, r22 = run.end()
    assert abs(its2 - its1) <= 1 and steps == -(-its2 // 7)
    assert r22 <= 1e-20 and rel(x2, x1) < 1e-8


def test_multishift_matches_single():
    dims = (4, 4, 4, 4)
    V = F.volume(dims)
    o = O.Oracle(dims, _links(dims, True))
    m = 0.05
    b = F.gaussian_vector(V, 11)
    b[V // 2:] = 0
    sg = [0.0, 0.01, 0.1, 1.0]
    xs = [o.vec() for _ in sg]
    its, r2 = o.cgm(0, xs, sg, b, m * m, 1e-22)
    for s, x in zip(sg, xs):
        ax = o.vec()
        o.stagD2ee(ax, x, m * m)
        ax += s * x
        res = np.linalg.norm(ax[: V // 2] - b[: V // 2]) ** 2 / np.linalg.norm(b[: V // 2]) ** 2
        assert res < 1e-18
    # the mass-form driver: D(ms[k]) xs[k] = b
    ms = [0.05, 0.1, 0.4]
    xm = [o.vec() for _ in ms]
    o.solve_multishift(xm, b, ms, 1e-20)
    for mm, x in zip(ms, xm):
        dx = o.vec()
        o.D(dx, x, mm)
        assert np.linalg.norm(dx - b) ** 2 / np.linalg.norm(b) ** 2 < 1e-14


def _action(o, phi, m):
    """S = phi_e^dagger A^{-1} phi_e with A = stagD2ee(m^2)."""
    V = phi.shape[0]
    y = o.vec()
    o.solveXX(0, y, phi, m, 1e-28)
    return np.vdot(phi[: V // 2], y[: V // 2]).real


@pytest.mark.parametrize("naik", [False, True])
def test_force_finite_difference(naik):
    """dS/deps for U_k(x) -> exp(eps T_a) U_k(x) equals ReTr[T_a f_k(x)^dagger]/8
    with f the force fermForce returns (QEX's psi carries a factor 4): central
    differences at eps = 1e-5 along all 8 su(3) generators on 64 seeded
    (site, direction, link kind) entries (with Naik links, k runs over the
    interleaved fat and long fields)."""
    dims = (4, 4, 4, 4)
    V = F.volume(dims)
    g = _links(dims, naik, seed=13)
    o = O.Oracle(dims, g)
    m = 0.2
    phi = F.gaussian_vector(V, 17)
    phi[V // 2:] = 0
    f = np.zeros_like(g)
    o.force(f, phi, m, 1e-28)
    rng = np.random.default_rng(19)
    entries = set()
    while len(entries) < 64:
        entries.add((int(rng.integers(0, g.shape[0])), int(rng.integers(0, V))))
    gens = F.su3_generators()
    eps = 1e-5
    for k, s in sorted(entries):
        for a, T in enumerate(gens):
            vals = []
            for e in (eps, -eps):
                gp = g.copy()
                gp[k, s] = F.exp_ah(T[None], e)[0] @ g[k, s]
                vals.append(_action(O.Oracle(dims, gp), phi, m))
            fd = (vals[0] - vals[1]) / (2 * eps)
            an = np.trace(T @ np.conj(f[k, s]).T).real / 8
            assert abs(fd - an) <= 1e-7 * max(abs(an), 1.0), (k, s, a, fd, an)
