"""Seeded synthetic lattice fields in QEX's V=1 site order (host, numpy).

Restates what QEX uses to make test gauge fields and sources:
  - randTah3 / randomTAH (src/gauge/gaugeUtils.nim:1466-1493): a traceless
    anti-Hermitian 3x3 matrix from 8 Gaussian numbers, off-diagonal
    re/im with sqrt(1/2), diagonal from r3 = sqrt(1/2) g, r8 = sqrt(1/6) g;
  - warmSU (gaugeUtils.nim:1495-1499): U = exp(eps * T);
  - stagPhase with phases [8,9,11,0] (src/physics/stagD.nim:560-571) and
    setBC, antiperiodic time (src/gauge/gaugeUtils.nim:133-140).
The random numbers come from numpy's PCG64 with the seeds given here, not
from QEX's MILC generator, so fields are statistically but not bitwise like
QEX's.  The exponential of eps*T = i*eps*H is formed from the eigenvectors
of the Hermitian H, exactly up to rounding.
"""
from __future__ import annotations

import numpy as np

S2 = 0.70710678118654752440  # sqrt(1/2)
S3 = 0.57735026918962576450  # sqrt(1/3)
PHASES = (8, 9, 11, 0)


def volume(dims) -> int:
    return int(np.prod(dims))


def coords(dims) -> np.ndarray:
    """coords[idx] = (x0, x1, x2, x3) of QEX V=1 site index idx."""
    dims = tuple(int(d) for d in dims)
    V = volume(dims)
    lex = np.arange(V, dtype=np.int64)
    x = np.empty((V, 4), dtype=np.int64)
    t = lex.copy()
    for d in range(4):
        x[:, d] = t % dims[d]
        t //= dims[d]
    p = x.sum(axis=1) & 1
    idx = (lex + p * V) // 2
    out = np.empty_like(x)
    out[idx] = x
    return out


def index_of(dims, x) -> np.ndarray:
    """QEX V=1 index of coordinates x (..., 4) (qlayout.nim:108-136)."""
    x = np.asarray(x, dtype=np.int64)
    V = volume(dims)
    lex = x[..., 0] + dims[0] * (x[..., 1] + dims[1] * (x[..., 2] + dims[2] * x[..., 3]))
    p = x.sum(axis=-1) & 1
    return (lex + p * V) // 2


def rand_tah(n: int, rng: np.random.Generator) -> np.ndarray:
    """n traceless anti-Hermitian matrices as randTah3 draws them."""
    g = rng.standard_normal((n, 8))
    r3 = S2 * g[:, 0]
    r8 = S2 * S3 * g[:, 1]
    m = np.zeros((n, 3, 3), dtype=np.complex128)
    m[:, 0, 0] = 1j * (r8 + r3)
    m[:, 1, 1] = 1j * (r8 - r3)
    m[:, 2, 2] = -2j * r8
    r01, r02, r12 = S2 * g[:, 2], S2 * g[:, 3], S2 * g[:, 4]
    i01, i02, i12 = S2 * g[:, 5], S2 * g[:, 6], S2 * g[:, 7]
    m[:, 0, 1] = r01 + 1j * i01
    m[:, 1, 0] = -r01 + 1j * i01
    m[:, 0, 2] = r02 + 1j * i02
    m[:, 2, 0] = -r02 + 1j * i02
    m[:, 1, 2] = r12 + 1j * i12
    m[:, 2, 1] = -r12 + 1j * i12
    return m


def su3_generators() -> np.ndarray:
    """The 8 traceless anti-Hermitian generators i lambda_a (Gell-Mann
    matrices lambda_a), shape (8, 3, 3)."""
    lam = np.zeros((8, 3, 3), dtype=np.complex128)
    lam[0][0, 1] = lam[0][1, 0] = 1
    lam[1][0, 1], lam[1][1, 0] = -1j, 1j
    lam[2][0, 0], lam[2][1, 1] = 1, -1
    lam[3][0, 2] = lam[3][2, 0] = 1
    lam[4][0, 2], lam[4][2, 0] = -1j, 1j
    lam[5][1, 2] = lam[5][2, 1] = 1
    lam[6][1, 2], lam[6][2, 1] = -1j, 1j
    lam[7] = np.diag([1, 1, -2]) / np.sqrt(3)
    return 1j * lam


def exp_ah(t: np.ndarray, eps: float | np.ndarray = 1.0) -> np.ndarray:
    """exp(eps * t) for anti-Hermitian t (..., 3, 3)."""
    h = -1j * t  # Hermitian
    h = 0.5 * (h + np.conj(np.swapaxes(h, -1, -2)))
    w, v = np.linalg.eigh(h)
    e = np.exp(1j * np.asarray(eps)[..., None] * w) if np.ndim(eps) else np.exp(1j * eps * w)
    return (v * e[..., None, :]) @ np.conj(np.swapaxes(v, -1, -2))


def warm_su3(n: int, eps, rng: np.random.Generator) -> np.ndarray:
    """warmSU: exp(eps * randTah3) for n links."""
    return exp_ah(rand_tah(n, rng), eps)


def gauge_warm(dims, eps: float, seed: int) -> np.ndarray:
    """Four SU(3) link fields, shape (4, V, 3, 3), unphased."""
    rng = np.random.default_rng(seed)
    V = volume(dims)
    return warm_su3(4 * V, eps, rng).reshape(4, V, 3, 3)


def fat_from_su3(u: np.ndarray, rng: np.random.Generator, scale=0.8, noise=0.2) -> np.ndarray:
    """General complex links scale*U + N(0, noise^2) on every re and im entry."""
    z = rng.standard_normal(u.shape) + 1j * rng.standard_normal(u.shape)
    return scale * u + noise * z


def eta(mu: int, x: np.ndarray) -> np.ndarray:
    """Staggered phase of direction mu at coordinates x (..., 4)."""
    s = np.zeros(x.shape[:-1], dtype=np.int64)
    for k in range(4):
        if (PHASES[mu] >> k) & 1:
            s += x[..., k]
    return np.where(s & 1, -1.0, 1.0)


def link_signs(dims, mu: int, hop: int) -> np.ndarray:
    """Sign folded into a link of direction mu spanning `hop` sites: eta_mu(x),
    and -1 where the hop crosses the antiperiodic time boundary."""
    x = coords(dims)
    s = eta(mu, x)
    if mu == 3:
        s = np.where(x[:, 3] + hop >= dims[3], -s, s)
    return s


def apply_phases(dims, links: np.ndarray) -> np.ndarray:
    """Fold phases and boundary signs into a link list (4 naive or 8
    interleaved fat/long, shape (n, V, 3, 3)); returns a new array."""
    n = links.shape[0]
    out = links.copy()
    for k in range(n):
        mu = k // 2 if n == 8 else k
        hop = (3 if k % 2 else 1) if n == 8 else 1
        out[k] *= link_signs(dims, mu, hop)[:, None, None]
    return out


def interleave(fat: np.ndarray, lng: np.ndarray) -> np.ndarray:
    """newStag3's link list [fat0, long0, fat1, long1, ...]."""
    out = np.empty((8,) + fat.shape[1:], dtype=fat.dtype)
    out[0::2] = fat
    out[1::2] = lng
    return out


def gaussian_vector(V: int, seed: int) -> np.ndarray:
    """Complex Gaussian colour vector field, N(0,1) on re and im, (V, 3)."""
    rng = np.random.default_rng(seed)
    return rng.standard_normal((V, 3)) + 1j * rng.standard_normal((V, 3))


# ---------------------------------------------------------------------------
# the workloads of the path
# ---------------------------------------------------------------------------

def naive_links(dims, eps: float = 0.3, seed: int = 11) -> np.ndarray:
    """Naive staggered links: warmSU(eps) per link, phased, shape (4, V, 3, 3)."""
    return apply_phases(dims, gauge_warm(dims, eps, seed))


def fat_naik_links(dims, seed: int = 21) -> np.ndarray:
    """Fat+Naik list (8, V, 3, 3), phased: fat = 0.8*SU(3) + N(0, 0.2^2)
    entries, long = SU(3) (warmSU(0.3)), long coefficient 1."""
    rng = np.random.default_rng(seed)
    V = volume(dims)
    fat = fat_from_su3(warm_su3(4 * V, 0.3, rng), rng).reshape(4, V, 3, 3)
    lng = warm_su3(4 * V, 0.3, rng).reshape(4, V, 3, 3)
    return apply_phases(dims, interleave(fat, lng))


def fat_naik_slab(global_dims, local_dims, offset, seed: int) -> np.ndarray:
    """A rank's part of a fat+Naik field of the fat_naik_links recipe: links
    of the local lattice local_dims, whose site at local coordinates x is the
    global site x + offset, drawn with this rank's seed and phased with the
    global coordinates (the antiperiodic boundary at the global last time
    slice); (8, Vloc, 3, 3) in the local V=1 order.  With local_dims =
    global_dims and offset 0 it is fat_naik_links(global_dims, seed)."""
    rng = np.random.default_rng(seed)
    V = volume(local_dims)
    fat = fat_from_su3(warm_su3(4 * V, 0.3, rng), rng).reshape(4, V, 3, 3)
    lng = warm_su3(4 * V, 0.3, rng).reshape(4, V, 3, 3)
    g = interleave(fat, lng)
    xg = coords(local_dims) + np.asarray(offset, dtype=np.int64)
    for k in range(8):
        mu, hop = k // 2, (3 if k % 2 else 1)
        s = eta(mu, xg)
        if mu == 3:
            s = np.where(xg[:, 3] + hop >= global_dims[3], -s, s)
        g[k] *= s[:, None, None]
    return g


def even_source(dims, seed: int = 31) -> np.ndarray:
    """Gaussian source on even sites, zero on odd sites, (V, 3)."""
    V = volume(dims)
    b = gaussian_vector(V, seed)
    b[V // 2:] = 0
    return b
