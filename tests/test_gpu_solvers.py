"""GPU parity of the FP64 solvers and the force against the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def links_for(dims, naik, seed=3):
    return F.fat_naik_links(dims, seed) if naik else F.naive_links(dims, 0.3, seed)


def true_r2_ee(o, y, b, m):
    V = b.shape[0]
    ay = o.vec()
    o.stagD2ee(ay, y, m * m)
    return np.linalg.norm(ay[: V // 2] - b[: V // 2]) ** 2 / np.linalg.norm(b[: V // 2]) ** 2


@pytest.mark.parametrize("naik", [False, True])
def test_solveEE_fp64_matches_oracle(cuda, naik):
    """Config-0-shaped check: 8^4, m = 0.1 (naive) / 0.05 (fat+Naik), r2req 1e-20."""
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, naik)
    m = 0.05 if naik else 0.1
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    b = F.even_source(dims, 31)
    yo = o.vec()
    its_o, r2_o = o.solveXX(0, yo, b, m, 1e-20)
    yg = o.vec()
    sp = S.SolverParams(r2req=1e-20)
    s.solveEE(yg, b, m, sp)
    assert sp.status == L.OK
    assert abs(sp.iterations - its_o) <= 1, (sp.iterations, its_o)
    assert true_r2_ee(o, yg, b, m) <= 1e-20
    assert rel(yg, yo) < 1e-8
    assert not np.any(yg[V // 2:])


@pytest.mark.parametrize("naik", [False, True])
def test_solve_full_matches_oracle(cuda, naik):
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, naik)
    m = 0.1
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    b = F.gaussian_vector(V, 41)
    xo = o.vec()
    its_o, _ = o.solve(xo, b, m, 1e-20)
    xg = o.vec()
    sp = S.SolverParams(r2req=1e-20)
    s.solve(xg, b, m, sp)
    dx = o.vec()
    o.D(dx, xg, m)
    assert np.linalg.norm(dx - b) ** 2 / np.linalg.norm(b) ** 2 <= 1e-20
    assert abs(sp.iterations - its_o) <= 2
    assert rel(xg, xo) < 1e-8


def test_solve_device_path(cuda):
    torch = cuda
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, False)
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), S.to_device_links(g))
    b = F.even_source(dims, 5)
    yd = torch.zeros((3, V), dtype=torch.complex128, device="cuda")
    sp = S.SolverParams(r2req=1e-20)
    s.solveEE(yd, S.to_device_vector(b), 0.1, sp)
    y = S.to_host_vector(yd)
    assert true_r2_ee(o, y, b, 0.1) <= 1e-20
    assert sp.r2 <= 1e-20 and sp.iterations > 0 and sp.seconds > 0


def test_solver_deterministic(cuda):
    dims = (8, 8, 8, 8)
    g = links_for(dims, True)
    s = S.Staggered(S.Layout(dims), g)
    b = F.even_source(dims, 7)
    out = []
    for _ in range(2):
        y = np.zeros_like(b)
        s.solveEE(y, b, 0.05, S.SolverParams(r2req=1e-18))
        out.append(y)
    assert np.array_equal(out[0], out[1])


def test_solver_maxits_reports_not_converged(cuda):
    dims = (8, 8, 8, 8)
    s = S.Staggered(S.Layout(dims), links_for(dims, False))
    b = F.even_source(dims, 7)
    y = np.zeros_like(b)
    sp = S.SolverParams(r2req=1e-20, maxits=5)
    s.solveEE(y, b, 0.1, sp)
    assert sp.status == L.NOT_CONVERGED and sp.iterations == 5


def test_solver_nan_source_is_an_error(cuda):
    dims = (4, 4, 4, 4)
    s = S.Staggered(S.Layout(dims), links_for(dims, False))
    b = F.even_source(dims, 7)
    b[3, 1] = np.nan
    y = np.zeros_like(b)
    with pytest.raises(L.QexStagError) as e:
        s.solveEE(y, b, 0.1, S.SolverParams(r2req=1e-20))
    assert e.value.code == L.ERR_NAN


def test_zero_source(cuda):
    dims = (4, 4, 4, 4)
    s = S.Staggered(S.Layout(dims), links_for(dims, True))
    b = np.zeros((256, 3), complex)
    y = np.ones_like(b)
    sp = S.SolverParams(r2req=1e-20)
    s.solveEE(y, b, 0.1, sp)
    assert not np.any(y) and sp.iterations == 0


@pytest.mark.parametrize("naik", [False, True])
def test_force_matches_oracle(cuda, naik):
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, naik)
    m = 0.05
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    phi = F.even_source(dims, 51)
    fo = np.zeros_like(g)
    o.force(fo, phi, m, 1e-24)
    fg = np.zeros_like(g)
    sp = S.SolverParams(r2req=1e-24)
    s.force(fg, phi, m, sp)
    assert rel(fg, fo) < 1e-9
    # fermForce alone on a given psi is exact to rounding
    psi = F.gaussian_vector(V, 52)
    fo2, fg2 = np.zeros_like(g), np.zeros_like(g)
    o.ferm_force(fo2, psi)
    s.ferm_force(fg2, psi)
    assert rel(fg2, fo2) < 1e-13


@pytest.mark.parametrize("sloppy", [L.SLOPPY_SINGLE, L.SLOPPY_HALF])
@pytest.mark.parametrize("naik", [False, True])
def test_mixed_precision_solveEE(cuda, naik, sloppy):
    """Reliable-update FP32/FP16 inner CG inside FP64 defect correction
    reaches the FP64 true residual and agrees with the FP64 oracle solve."""
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, naik)
    m = 0.05
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    if naik:
        assert s.recon12
    b = F.even_source(dims, 61)
    yo = o.vec()
    o.solveXX(0, yo, b, m, 1e-22)
    y = o.vec()
    sp = S.SolverParams(r2req=1e-20, sloppySolve=sloppy)
    s.solveEE(y, b, m, sp)
    assert sp.status == L.OK
    assert true_r2_ee(o, y, b, m) <= 1e-20
    assert rel(y, yo) < 1e-8
    assert sp.reliable_updates >= 1


def test_mixed_without_recon12(cuda):
    """Long links that are not a phase times SU(3) keep all 18 reals."""
    dims = (8, 8, 8, 8)
    g = links_for(dims, True)
    g[1::2] = g[0::2] * 0.5  # long := half the fat links (not unitary)
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    assert not s.recon12
    b = F.even_source(dims, 62)
    for sloppy in (L.SLOPPY_SINGLE, L.SLOPPY_HALF):
        y = o.vec()
        s.solveEE(y, b, 0.1, S.SolverParams(r2req=1e-20, sloppySolve=sloppy))
        assert true_r2_ee(o, y, b, 0.1) <= 1e-20


def test_mixed_long_coeff(cuda):
    """A long-link coefficient (QEX HISQ folds naik = -1/24 into the long
    links) is honoured by the 12-real reconstruction."""
    dims = (8, 8, 8, 8)
    g = links_for(dims, True)
    c = -1.0 / 24.0
    g[1::2] *= c
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g, long_coeff=c)
    assert s.recon12
    b = F.even_source(dims, 63)
    y = o.vec()
    s.solveEE(y, b, 0.05, S.SolverParams(r2req=1e-20, sloppySolve=L.SLOPPY_HALF))
    assert true_r2_ee(o, y, b, 0.05) <= 1e-20


def test_mixed_full_solve(cuda):
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, True)
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    b = F.gaussian_vector(V, 64)
    x = o.vec()
    s.solve(x, b, 0.1, S.SolverParams(r2req=1e-20, sloppySolve=L.SLOPPY_HALF))
    dx = o.vec()
    o.D(dx, x, 0.1)
    assert np.linalg.norm(dx - b) ** 2 / np.linalg.norm(b) ** 2 <= 1e-20


def test_solveXX_host_fields_read_the_solved_parity(cuda):
    """solveEE / solveOO with host fields copy in only the solved parity of
    the source: with the other parity nonzero the solution equals the one
    through device fields bit for bit, and the other parity of the result
    is zero."""
    import torch
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    s = S.Staggered(S.Layout(dims), links_for(dims, True))
    x = F.gaussian_vector(V, 5)
    for par, fn in ((0, s.solveEE), (1, s.solveOO)):
        yh = np.full_like(x, 7.0)
        fn(yh, x, 0.1, S.SolverParams(r2req=1e-18))
        yd = torch.zeros((3, V), dtype=torch.complex128, device="cuda")
        fn(yd, S.to_device_vector(x), 0.1, S.SolverParams(r2req=1e-18))
        yd = yd.cpu().numpy().T
        assert np.array_equal(yh, yd), par
        other = slice(V // 2, V) if par == 0 else slice(0, V // 2)
        assert not np.any(yh[other])
