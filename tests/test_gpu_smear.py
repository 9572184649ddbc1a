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
