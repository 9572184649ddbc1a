"""GPU checks at the benchmark's full size (32^4 fat+Naik) through
size-independent properties, where the oracle would take minutes:
antihermiticity of the hopping term, Hermiticity of the Schur operator, the
free-field spectrum, and the FP64 true residual of every solver precision."""
import numpy as np
import pytest

from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu
DIMS = (32, 32, 32, 32)


@pytest.fixture(scope="module")
def big(cuda):
    torch = cuda
    V = F.volume(DIMS)
    g = F.fat_naik_links(DIMS, 21)
    s = S.Staggered(S.Layout(DIMS), S.to_device_links(g))
    return torch, s, V


def _rand(torch, V, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    return torch.complex(torch.randn((3, V), dtype=torch.float64, device="cuda", generator=gen),
                         torch.randn((3, V), dtype=torch.float64, device="cuda", generator=gen))


def test_hopping_term_antihermitian(big):
    torch, s, V = big
    x, y = _rand(torch, V, 1), _rand(torch, V, 2)
    dx, dy = torch.zeros_like(x), torch.zeros_like(y)
    s.D(dx, x, 0.0)
    s.D(dy, y, 0.0)
    lhs = torch.vdot(y.reshape(-1), dx.reshape(-1))
    rhs = -torch.vdot(dy.reshape(-1), x.reshape(-1))
    assert abs(lhs - rhs).item() <= 1e-12 * abs(lhs).item()


def test_schur_hermitian_positive(big):
    torch, s, V = big
    h = V // 2
    x, y = _rand(torch, V, 3), _rand(torch, V, 4)
    x[:, h:] = 0
    y[:, h:] = 0
    ax, ay = torch.zeros_like(x), torch.zeros_like(y)
    s.stagD2ee(ax, x, 1e-4)
    s.stagD2ee(ay, y, 1e-4)
    a = torch.vdot(y[:, :h].reshape(-1), ax[:, :h].reshape(-1))
    b = torch.vdot(ay[:, :h].reshape(-1), x[:, :h].reshape(-1))
    assert abs(a - b).item() <= 1e-12 * abs(a).item()
    assert torch.vdot(x[:, :h].reshape(-1), ax[:, :h].reshape(-1)).real.item() > 0


def test_free_field_spectrum_full_size(cuda):
    """Unit links with phases: plane waves are eigenvectors of stagD2ee with
    eigenvalue 4 m^2 + 4 sum_mu (sin p + sin 3p)^2 (antiperiodic time)."""
    torch = cuda
    V = F.volume(DIMS)
    one = np.zeros((8, V, 3, 3), complex)
    one[:] = np.eye(3)
    s = S.Staggered(S.Layout(DIMS), S.to_device_links(F.apply_phases(DIMS, one)))
    c = F.coords(DIMS)
    n = np.array([3, 1, 7, 5])
    p = 2 * np.pi * n / np.array(DIMS)
    p[3] = (2 * n[3] + 1) * np.pi / DIMS[3]
    ph = np.exp(1j * (c @ p))
    x = np.zeros((V, 3), complex)
    x[: V // 2, 1] = ph[: V // 2]
    xd = S.to_device_vector(x)
    r = torch.zeros_like(xd)
    m = 0.01
    s.stagD2ee(r, xd, m * m)
    lam = 4 * m * m + 4 * np.sum((np.sin(p) + np.sin(3 * p)) ** 2)
    got = S.to_host_vector(r)[: V // 2]
    assert np.abs(got - lam * x[: V // 2]).max() <= 1e-13 * lam


@pytest.mark.parametrize("sloppy", [S.L.SLOPPY_NONE, S.L.SLOPPY_SINGLE, S.L.SLOPPY_HALF])
def test_solve_true_residual_full_size(big, sloppy):
    torch, s, V = big
    h = V // 2
    b = S.to_device_vector(F.even_source(DIMS, 31))
    y = torch.zeros_like(b)
    sp = S.SolverParams(r2req=1e-20, sloppySolve=sloppy)
    s.solveEE(y, b, 0.01, sp)
    ay = torch.zeros_like(y)
    s.stagD2ee(ay, y, 1e-4)
    r2 = ((ay[:, :h] - b[:, :h]).abs() ** 2).sum().item() / (b[:, :h].abs() ** 2).sum().item()
    assert r2 <= 1e-20 and sp.status == S.L.OK
    assert abs(sp.r2 - r2) <= 1e-3 * r2
    if sloppy == S.L.SLOPPY_NONE:
        assert sp.iterations == 2719  # the oracle's count for this system
