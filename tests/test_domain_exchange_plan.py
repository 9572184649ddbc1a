"""The ghost-exchange plan of the t-then-z domain decomposition (CPU only):
the copy ranges domain.cu issues, replayed on numpy parity blocks, leave
every site of every rank's extended lattice, corners included, equal to
the global field, and the row mask the CG sums use picks exactly the
interior z rows.  Index order: V=1 checkerboard order of the extended
lattice {L0, L1, Z + 2h, T + 2h}; a parity block's t slice holds
sh = P (Z + 2h) sites in rows of P = L0 L1 / 2."""
import numpy as np
import pytest

from qex_b200 import fields as F


def _plan(gdims, Rz, Rt, h):
    L0, L1, L2, L3 = gdims
    Z, T = L2 // Rz, L3 // Rt
    Ze, Te = Z + 2 * h, T + 2 * h
    edims = (L0, L1, Ze, Te)
    Ve = L0 * L1 * Ze * Te
    nh, P = Ve // 2, L0 * L1 // 2
    sh = P * Ze
    glob = np.arange(F.volume(gdims)) + 1.0
    ec = F.coords(edims)
    R = Rz * Rt

    def rank_of(rz, rt):
        return rz % Rz + Rz * (rt % Rt)

    def ideal(r):
        g = ec.copy()
        g[:, 2] = (g[:, 2] - h + (r % Rz) * Z) % L2
        g[:, 3] = (g[:, 3] - h + (r // Rz) * T) % L3
        return glob[F.index_of(gdims, g)]

    inter = (ec[:, 2] >= h) & (ec[:, 2] < h + Z) & (ec[:, 3] >= h) & (ec[:, 3] < h + T)
    fields = []
    for r in range(R):
        f = np.zeros(Ve)
        f[inter] = ideal(r)[inter]
        fields.append(f)
    # t phase: whole slices from the t neighbours' interior edge slices
    new = [f.copy() for f in fields]
    for r in range(R):
        up, dn = rank_of(r % Rz, r // Rz + 1), rank_of(r % Rz, r // Rz - 1)
        for o in (0, nh):
            new[r][o:o + h * sh] = fields[dn][o + T * sh:o + (T + h) * sh]
            new[r][o + (h + T) * sh:o + (T + 2 * h) * sh] = fields[up][o + h * sh:o + 2 * h * sh]
    fields = new
    # z phase: rows of every slice (t ghosts included), pitch sh
    new = [f.copy() for f in fields]
    for r in range(R):
        zu, zd = rank_of(r % Rz + 1, r // Rz), rank_of(r % Rz - 1, r // Rz)
        for o in (0, nh):
            for s in range(Te):
                b = o + s * sh
                new[r][b:b + h * P] = fields[zd][b + Z * P:b + (Z + h) * P]
                new[r][b + (h + Z) * P:b + (Z + 2 * h) * P] = fields[zu][b + h * P:b + 2 * h * P]
    complete = all(np.array_equal(new[r], ideal(r)) for r in range(R))
    i = np.arange(T * sh)
    mask = ((i // P) % Ze >= h) & ((i // P) % Ze < h + Z)
    blk = np.arange(h * sh, (h + T) * sh)
    rows_ok = np.array_equal(mask, inter[blk])
    return complete, rows_ok


@pytest.mark.parametrize("gdims,Rz,Rt,h", [((4, 4, 12, 12), 2, 2, 6), ((4, 4, 12, 12), 1, 1, 6),
                                          ((4, 4, 8, 8), 2, 2, 2), ((4, 4, 8, 12), 2, 1, 2),
                                          ((4, 4, 12, 24), 2, 2, 6), ((4, 4, 16, 8), 4, 2, 2)])
def test_two_phase_exchange_fills_every_ghost(gdims, Rz, Rt, h):
    complete, rows_ok = _plan(gdims, Rz, Rt, h)
    assert complete
    assert rows_ok


@pytest.mark.parametrize("gdims,grid", [((4, 4, 8, 8), (1, 2)), ((4, 4, 12, 12), (2, 2)), ((4, 4, 16, 8), (4, 2)),
                                        ((8, 4, 6, 16), (1, 4))])
def test_rank_sites_partition_the_lattice(gdims, grid):
    """The ranks' sites (DomainSet's split of global fields) cover every
    global site once, and a local site's parity is its global parity."""
    from qex_b200.domain import rank_sites
    ldims = (gdims[0], gdims[1], gdims[2] // grid[0], gdims[3] // grid[1])
    V, Vl = F.volume(gdims), F.volume(ldims)
    owned = np.concatenate([rank_sites(gdims, ldims, grid, r) for r in range(grid[0] * grid[1])])
    assert np.array_equal(np.sort(owned), np.arange(V))
    for r in range(grid[0] * grid[1]):
        gi = rank_sites(gdims, ldims, grid, r)
        # V=1 order: the first half of each lattice is even
        assert np.all((gi[: Vl // 2] < V // 2)) and np.all(gi[Vl // 2:] >= V // 2)


def test_fat_naik_slab_phases():
    """A rank's slab of the fat+Naik field carries the phases of its global
    sites; the whole lattice as one slab is fat_naik_links itself."""
    gdims = (4, 4, 4, 12)
    assert np.array_equal(F.fat_naik_slab(gdims, gdims, (0, 0, 0, 0), 21), F.fat_naik_links(gdims, 21))
    ldims = (4, 4, 4, 6)
    for r in range(2):
        off = (0, 0, 0, 6 * r)
        g = F.fat_naik_slab(gdims, ldims, off, 21 + r)
        # undo the phases with the global signs: what is left is unphased, the
        # same draws as the slab's own unphased links
        raw = F.fat_naik_slab(ldims, ldims, (0, 0, 0, 0), 21 + r)
        raw = F.apply_phases(ldims, raw)  # apply_phases twice = identity: raw is now unphased
        from qex_b200.domain import rank_sites
        gi = rank_sites(gdims, ldims, (1, 2), r)
        for k in range(8):
            mu, hop = k // 2, (3 if k % 2 else 1)
            sg = F.link_signs(gdims, mu, hop)[gi]
            assert np.array_equal(g[k], raw[k] * sg[:, None, None])
