"""GPU parity of the layout tables and the FP64 Dslash family against the
oracle, through the C ABI (host and device paths).  Tolerance 1e-13
relative (max-norm), bit-exact for index tables."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu
TOL = 1e-13
SHAPES = [(8, 8, 8, 8), (4, 6, 8, 4), (6, 4, 4, 10)]


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def links_for(dims, naik, seed=3):
    return F.fat_naik_links(dims, seed) if naik else F.naive_links(dims, 0.3, seed)


@pytest.mark.parametrize("dims", SHAPES)
def test_shift_tables_bit_exact(cuda, dims):
    lay = S.Layout(dims)
    V = F.volume(dims)
    for mu in range(4):
        for ln in (1, -1, 3, -3):
            for sub in (0, 1, 2):
                got = lay.shift_table(mu, ln, sub)
                exp = O.shift_table(dims, mu, ln, sub)
                assert np.array_equal(got, exp), (mu, ln, sub)
    c = F.coords(dims)
    for i in range(0, V, max(1, V // 50)):
        assert lay.index(c[i]) == i


@pytest.mark.parametrize("naik", [False, True])
@pytest.mark.parametrize("dims", SHAPES)
def test_dslash_family_host_path(cuda, dims, naik):
    V = F.volume(dims)
    g = links_for(dims, naik)
    o = O.Oracle(dims, g)
    lay = S.Layout(dims)
    s = S.Staggered(lay, g)
    x = F.gaussian_vector(V, 5)
    r0 = F.gaussian_vector(V, 6)
    for sub in (0, 1):
        for a, b in [(0.0, 0.0), (0.0, 0.7), (0.3, -1.2)]:
            rg, ro = r0.copy(), r0.copy()
            s.stagD2(sub, rg, x, a, b)
            o.stagD2(sub, ro, x, a, b)
            assert rel(rg, ro) < TOL, (sub, a, b)
        for m, sc, a in [(0.1, 1.0, 0.0), (0.2, -1.0, 0.0), (0.05, 1.0, 0.4)]:
            rg, ro = r0.copy(), r0.copy()
            s.stagD(sub, rg, x, m, sc, a)
            o.stagD(sub, ro, x, m, sc, a)
            assert rel(rg, ro) < TOL
    for fn in ("D", "Ddag"):
        rg, ro = o.vec(), o.vec()
        getattr(s, fn)(rg, x, 0.1)
        getattr(o, fn)(ro, x, 0.1)
        assert rel(rg, ro) < TOL
    for fn in ("stagD2ee", "stagD2oo"):
        rg, ro = r0.copy(), r0.copy()
        getattr(s, fn)(rg, x, 0.01)
        getattr(o, fn)(ro, x, 0.01)
        par = 0 if fn == "stagD2ee" else 1
        sl = slice(0, V // 2) if par == 0 else slice(V // 2, V)
        assert rel(rg[sl], ro[sl]) < TOL
        other = slice(V // 2, V) if par == 0 else slice(0, V // 2)
        assert np.array_equal(rg[other], r0[other])


@pytest.mark.parametrize("naik", [False, True])
def test_dslash_device_path_matches_host(cuda, naik):
    torch = cuda
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, naik)
    lay = S.Layout(dims)
    sh = S.Staggered(lay, g)
    sd = S.Staggered(lay, S.to_device_links(g))
    x = F.gaussian_vector(V, 8)
    rh = np.zeros((V, 3), complex)
    sh.D(rh, x, 0.3)
    xd = S.to_device_vector(x)
    rd = torch.zeros((3, V), dtype=torch.complex128, device="cuda")
    sd.D(rd, xd, 0.3)
    assert np.array_equal(S.to_host_vector(rd), rh)
    sd.stagD2ee(rd, xd, 0.09)
    o = O.Oracle(dims, g)
    ro = o.vec()
    o.stagD2ee(ro, x, 0.09)
    assert rel(S.to_host_vector(rd)[: V // 2], ro[: V // 2]) < TOL


def test_dslash_deterministic(cuda):
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = links_for(dims, True)
    s = S.Staggered(S.Layout(dims), g)
    x = F.gaussian_vector(V, 9)
    a, b = np.zeros((V, 3), complex), np.zeros((V, 3), complex)
    s.D(a, x, 0.1)
    s.D(b, x, 0.1)
    assert np.array_equal(a, b)


def test_argument_errors(cuda):
    dims = (4, 4, 4, 4)
    lay = S.Layout(dims)
    with pytest.raises(L.QexStagError) as e:
        S.Layout((4, 4, 5, 4))
    assert e.value.code == L.ERR_ARG
    g = links_for(dims, False)
    s = S.Staggered(lay, g)
    V = lay.V
    x = np.zeros((V, 3), complex)
    with pytest.raises(L.QexStagError) as e:
        s.stagD2(2, x.copy(), x, 0.0, 1.0)
    assert e.value.code == L.ERR_ARG
    lib = L.load()
    assert lib.qexstag_links_create(lay.handle, 5, None, 0, 1.0, None) == L.ERR_ARG


@pytest.mark.parametrize("naik", [False, True])
def test_rephase_on_device(cuda, naik):
    """Phasing every field of unphased links gives the operator of the
    phased links (oracle's setBC + stagPhase per direction and hop); a
    second call restores them.  For naive links this is QEX's rephase."""
    dims = (8, 4, 6, 8)
    V = F.volume(dims)
    if naik:
        rng = np.random.default_rng(4)
        raw = F.interleave(F.fat_from_su3(F.warm_su3(4 * V, 0.3, rng), rng).reshape(4, V, 3, 3),
                           F.warm_su3(4 * V, 0.3, rng).reshape(4, V, 3, 3))
    else:
        raw = F.gauge_warm(dims, 0.3, 4)
    s = S.Staggered(S.Layout(dims), raw)
    flip = s.rephase_all if naik else s.rephase
    flip()
    o = O.Oracle(dims, O.apply_phases(dims, raw))
    x = F.gaussian_vector(V, 9)
    a, b = np.zeros_like(x), np.zeros_like(x)
    s.D(a, x, 0.1)
    o.D(b, x, 0.1)
    assert rel(a, b) < TOL
    if naik:
        assert s.recon12
    flip()
    o2 = O.Oracle(dims, raw)
    o2.D(b, x, 0.1)
    s.D(a, x, 0.1)
    assert rel(a, b) < TOL


def test_rephase_fat_naik_is_qex_literal(cuda):
    """QEX's rephase(s) on newStag3's list acts on its first four fields
    only (setBC on field 3, stagPhase eta_k on field k, stagD.nim:106-114):
    fat_0, long_0, fat_1, long_1 change, the rest do not."""
    dims = (8, 4, 6, 8)
    V = F.volume(dims)
    rng = np.random.default_rng(6)
    raw = F.interleave(F.fat_from_su3(F.warm_su3(4 * V, 0.3, rng), rng).reshape(4, V, 3, 3),
                       F.warm_su3(4 * V, 0.3, rng).reshape(4, V, 3, 3))
    want = raw.copy()
    want[:4] = O.apply_phases(dims, np.ascontiguousarray(raw[:4]))  # fields 0-3 as directions 0-3
    s = S.Staggered(S.Layout(dims), raw)
    s.rephase()
    t = S.Staggered(S.Layout(dims), want)
    x = F.gaussian_vector(V, 10)
    a, b = np.zeros_like(x), np.zeros_like(x)
    s.D(a, x, 0.1)
    t.D(b, x, 0.1)
    assert np.array_equal(a, b)
    fat, lng = s.links_milc()
    assert np.array_equal(fat, np.ascontiguousarray(np.moveaxis(want[0::2], 0, 1)))
    assert np.array_equal(lng, np.ascontiguousarray(np.moveaxis(want[1::2], 0, 1)))


@pytest.mark.parametrize("naik", [False, True])
def test_links_milc_order(cuda, naik):
    """Links in MILC order (QUDA's MILC gauge order, qudaWrapperImpl.nim:
    205-245) give the operator of QEX's list bit for bit, and come back out
    unchanged."""
    dims = (8, 4, 6, 8)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 12) if naik else F.naive_links(dims, 0.3, 12)
    fat = np.ascontiguousarray(np.moveaxis(g[0::2] if naik else g, 0, 1))
    lng = np.ascontiguousarray(np.moveaxis(g[1::2], 0, 1)) if naik else None
    lay = S.Layout(dims)
    s = S.Staggered(lay, g)
    m = S.Staggered.from_milc(lay, fat, lng)
    assert m.nlinks == s.nlinks and m.recon12 == s.recon12
    x = F.gaussian_vector(V, 13)
    a, b = np.zeros_like(x), np.zeros_like(x)
    s.D(a, x, 0.07)
    m.D(b, x, 0.07)
    assert np.array_equal(a, b)
    f2, l2 = m.links_milc()
    assert np.array_equal(f2, fat) and (l2 is None or np.array_equal(l2, lng))
    f3, l3 = s.links_milc()  # QEX-ordered upload, MILC-ordered download
    assert np.array_equal(f3, fat) and (l3 is None or np.array_equal(l3, lng))
    g2 = F.fat_naik_links(dims, 14) if naik else F.naive_links(dims, 0.3, 14)
    m.update_links_milc(np.ascontiguousarray(np.moveaxis(g2[0::2] if naik else g2, 0, 1)),
                        np.ascontiguousarray(np.moveaxis(g2[1::2], 0, 1)) if naik else None)
    s.update_links(g2)
    s.D(a, x, 0.07)
    m.D(b, x, 0.07)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("naik", [False, True])
@pytest.mark.parametrize("n", [1, 3, 11])
def test_stagDN_matches_oracle(cuda, naik, n):
    """stagDN (stagD.nim:451-455): r_i = m x_i + (2D) x_i on one subset for
    n fields at once equals the oracle's stagD2(subset, r_i, x_i, 0, m) for
    every i, host and device paths; the other parity of r_i is unchanged.
    n = 11 spans two launches of the 8-field kernel."""
    torch = cuda
    dims = (8, 4, 6, 8)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 17) if naik else F.naive_links(dims, 0.3, 17)
    o = O.Oracle(dims, g)
    s = S.Staggered(S.Layout(dims), g)
    m = 0.37
    xs = [F.gaussian_vector(V, 100 + i) for i in range(n)]
    for subset in (L.EVEN, L.ODD):
        other = slice(V // 2, V) if subset == L.EVEN else slice(0, V // 2)
        mine = slice(0, V // 2) if subset == L.EVEN else slice(V // 2, V)
        rs = [np.full((V, 3), 3.0 + 1j) for _ in range(n)]
        s.stagDN(subset, rs, xs, m)
        rd = [torch.full((3, V), 2.0 - 1j, dtype=torch.complex128, device="cuda") for _ in range(n)]
        s.stagDN(subset, rd, [S.to_device_vector(x) for x in xs], m)
        for i in range(n):
            ro = o.vec()
            o.stagD2(subset, ro, xs[i], 0.0, m)
            assert rel(rs[i][mine], ro[mine]) < TOL, (subset, i)
            assert np.all(rs[i][other] == 3.0 + 1j)
            rh = S.to_host_vector(rd[i])
            assert np.array_equal(rh[mine], rs[i][mine])
            assert np.all(rh[other] == 2.0 - 1j)
