"""GPU tests of the domain decomposition along t (qexstag_domain_*): every
rank's slab held in one process on one device (ghost exchanges by device
copies), against the single-lattice operator and the oracle's CG; and the
NCCL exchange path with one rank (NCCL send/receive to itself)."""
import numpy as np
import pytest

from oracle import oracle as O
from qex_b200 import _lib as L
from qex_b200 import domain as DD
from qex_b200 import fields as F
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


# slabs thicker than 4 x the hop reach (12 with Naik links, 4 without) run
# the sweeps next to the ghosts after the exchange and the rest during it;
# thinner slabs run both sweeps after the exchange
CASES = [((8, 8, 8, 24), 8, [1, 2, 3, 4]), ((8, 4, 6, 16), 4, [1, 2, 4]), ((4, 4, 8, 32), 8, [2])]


@pytest.mark.parametrize("dims,nl,ranks", CASES)
def test_schur_matches_single_lattice(cuda, dims, nl, ranks):
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 5) if nl == 8 else F.naive_links(dims, 0.4, 5)
    x = F.gaussian_vector(V, 6)
    ref = x.copy()
    S.Staggered(S.Layout(dims), g).stagD2ee(ref, x, 0.04)
    for R in ranks:
        d = DD.DomainSet(dims, R, nl)
        d.set_links(g)
        # every slab's long links pass the 12-real check against signs
        # rebuilt from global time
        assert d.recon12 == (nl == 8), R
        r = x.copy()
        d.stagD2ee(r, x, 0.04)
        # even sites bit-exact (the same kernels, the same order per site);
        # odd sites untouched
        assert np.array_equal(r[: V // 2], ref[: V // 2]), R
        assert np.array_equal(r[V // 2:], x[V // 2:])


@pytest.mark.parametrize("dims,nl,ranks", CASES)
def test_cg_matches_oracle(cuda, dims, nl, ranks):
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 7) if nl == 8 else F.naive_links(dims, 0.4, 7)
    b = F.even_source(dims, 8)
    o = O.Oracle(dims, g)
    xo = o.vec()
    its_o, _ = o.cg(0, xo, b, 0.01, 1e-20)
    for R in ranks:
        d = DD.DomainSet(dims, R, nl)
        d.set_links(g)
        x = np.zeros_like(b)
        sp = S.SolverParams(r2req=1e-20)
        d.solveEE(x, b, 0.1, sp)
        assert abs(sp.iterations - its_o) <= 2, (R, sp.iterations, its_o)
        assert sp.r2 <= 1e-20 * 1.0001
        assert rel(x[: V // 2], xo[: V // 2]) < 1e-8
        assert not np.any(x[V // 2:])
        ax = o.vec()
        o.stagD2ee(ax, x, 0.01)
        assert np.linalg.norm(ax[: V // 2] - b[: V // 2]) ** 2 <= 1e-20 * np.linalg.norm(b[: V // 2]) ** 2 * 1.0001


def test_nccl_self_exchange(cuda):
    """One rank over an NCCL communicator of size 1: the boundary slices go
    to itself through ncclSend/ncclRecv and the sums through ncclAllReduce;
    results equal the in-process path's."""
    dims = (8, 8, 8, 8)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 9)
    x = F.gaussian_vector(V, 10)
    local = DD.DomainSet(dims, 1, 8)
    local.set_links(g)
    viaccl = DD.DomainSet(dims, 1, 8, nccl_id=DD.nccl_unique_id())
    viaccl.set_links(g)
    a, b = x.copy(), x.copy()
    local.stagD2ee(a, x, 0.09)
    viaccl.stagD2ee(b, x, 0.09)
    assert np.array_equal(a, b)
    src = F.even_source(dims, 11)
    ya, yb = np.zeros_like(src), np.zeros_like(src)
    spa, spb = S.SolverParams(r2req=1e-18), S.SolverParams(r2req=1e-18)
    local.solveEE(ya, src, 0.2, spa)
    viaccl.solveEE(yb, src, 0.2, spb)
    assert spa.iterations == spb.iterations and np.array_equal(ya, yb)
    # the 16-bit domain solve: the ghost exchange of p through ncclSend /
    # ncclRecv and every sum through ncclAllReduce give the in-process result
    ya, yb = np.zeros_like(src), np.zeros_like(src)
    spa = S.SolverParams(r2req=1e-18, sloppySolve=S.L.SLOPPY_HALF, delta=0.1)
    spb = S.SolverParams(r2req=1e-18, sloppySolve=S.L.SLOPPY_HALF, delta=0.1)
    local.solveEE(ya, src, 0.2, spa)
    viaccl.solveEE(yb, src, 0.2, spb)
    assert spa.iterations == spb.iterations and np.array_equal(ya, yb)
    assert spb.r2 <= 1e-18 and spb.reliable_updates >= 1


def test_domain_errors(cuda):
    lib = L.load()
    import ctypes as C
    h = C.c_void_p()
    dims = (C.c_int * 4)(8, 8, 8, 20)
    assert lib.qexstag_domain_create(dims, 3, 0, 8, C.byref(h)) == L.ERR_ARG  # 20 not a multiple of 3
    dims = (C.c_int * 4)(8, 8, 8, 16)
    assert lib.qexstag_domain_create(dims, 4, 0, 8, C.byref(h)) == L.ERR_ARG  # slabs of 4 < 6 ghosts
    assert lib.qexstag_domain_create(dims, 2, 2, 8, C.byref(h)) == L.ERR_ARG
    assert lib.qexstag_domain_create(dims, 8, 0, 4, C.byref(h)) == L.ERR_ARG  # slabs of 2 < 4


def test_torchrun_one_rank_per_gpu(cuda, tmp_path):
    """The one-rank-per-GPU driver under torchrun with the ranks this
    machine has (one here): NCCL id broadcast, slab solve, true residual."""
    import json
    import subprocess
    import sys
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=1",
           "--master-addr=127.0.0.1", "--master-port=29517", "-m", "qex_b200.domain_run", "--dims", "8,8,8,16"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [ln for ln in out.stdout.splitlines() if ln.startswith("{")][-1]
    res = json.loads(line)
    assert res["ranks"] == 1 and res["true_r2"] <= 1e-20 * 1.0001 and res["status"] == 0


# splits along t and z: (dims, nlinks, [(Rz, Rt), ...]); (1, 1) keeps z ghosts
# and exchanges them with itself
ZT_CASES = [((4, 4, 12, 12), 8, [(1, 1), (2, 1), (1, 2), (2, 2)]),
            ((4, 4, 8, 8), 4, [(1, 1), (2, 2)]),
            ((4, 4, 16, 8), 4, [(4, 2)])]


@pytest.mark.parametrize("dims,nl,grids", ZT_CASES)
def test_zt_schur_matches_single_lattice(cuda, dims, nl, grids):
    """Every rank of an Rz x Rt split in one process: even sites of the Schur
    operator bit-exact against the single lattice (the corner ghosts reach
    the second half sweep through the Naik hops), odd sites untouched."""
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 5) if nl == 8 else F.naive_links(dims, 0.4, 5)
    x = F.gaussian_vector(V, 6)
    ref = x.copy()
    S.Staggered(S.Layout(dims), g).stagD2ee(ref, x, 0.04)
    for Rz, Rt in grids:
        d = DD.DomainSet(dims, Rz * Rt, nl, grid=(Rz, Rt))
        assert d.ldims == (dims[0], dims[1], dims[2] // Rz, dims[3] // Rt)
        d.set_links(g)
        assert d.recon12 == (nl == 8), (Rz, Rt)
        r = x.copy()
        d.stagD2ee(r, x, 0.04)
        assert np.array_equal(r[: V // 2], ref[: V // 2]), (Rz, Rt)
        assert np.array_equal(r[V // 2:], x[V // 2:])


@pytest.mark.parametrize("dims,nl,grids", ZT_CASES)
def test_zt_cg_matches_oracle(cuda, dims, nl, grids):
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 7) if nl == 8 else F.naive_links(dims, 0.4, 7)
    b = F.even_source(dims, 8)
    o = O.Oracle(dims, g)
    xo = o.vec()
    its_o, _ = o.cg(0, xo, b, 0.01, 1e-20)
    for Rz, Rt in grids:
        d = DD.DomainSet(dims, Rz * Rt, nl, grid=(Rz, Rt))
        d.set_links(g)
        x = np.zeros_like(b)
        sp = S.SolverParams(r2req=1e-20)
        d.solveEE(x, b, 0.1, sp)
        assert abs(sp.iterations - its_o) <= 2, (Rz, Rt, sp.iterations, its_o)
        assert sp.r2 <= 1e-20 * 1.0001
        assert rel(x[: V // 2], xo[: V // 2]) < 1e-8
        assert not np.any(x[V // 2:])


def test_zt_nccl_self_exchange(cuda):
    """A 1 x 1 grid over an NCCL communicator of size 1: the z faces are
    packed, sent to the rank itself and unpacked; results equal the
    in-process path's."""
    dims = (4, 4, 8, 8)
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 9)
    x = F.gaussian_vector(V, 10)
    local = DD.DomainSet(dims, 1, 8, grid=(1, 1))
    local.set_links(g)
    viaccl = DD.DomainSet(dims, 1, 8, nccl_id=DD.nccl_unique_id(), grid=(1, 1))
    viaccl.set_links(g)
    a, b = x.copy(), x.copy()
    local.stagD2ee(a, x, 0.09)
    viaccl.stagD2ee(b, x, 0.09)
    assert np.array_equal(a, b)
    ref = x.copy()
    S.Staggered(S.Layout(dims), g).stagD2ee(ref, x, 0.09)
    assert np.array_equal(a[: V // 2], ref[: V // 2])
    src = F.even_source(dims, 11)
    ya, yb = np.zeros_like(src), np.zeros_like(src)
    spa, spb = S.SolverParams(r2req=1e-18), S.SolverParams(r2req=1e-18)
    local.solveEE(ya, src, 0.2, spa)
    viaccl.solveEE(yb, src, 0.2, spb)
    assert spa.iterations == spb.iterations and np.array_equal(ya, yb)


def test_zt_errors(cuda):
    lib = L.load()
    import ctypes as C
    h = C.c_void_p()
    dims = (C.c_int * 4)(4, 4, 12, 12)
    assert lib.qexstag_domain_create_zt(dims, (C.c_int * 2)(4, 1), 0, 8, C.byref(h)) == L.ERR_ARG  # Z = 3
    assert lib.qexstag_domain_create_zt(dims, (C.c_int * 2)(5, 1), 0, 8, C.byref(h)) == L.ERR_ARG  # 12 % 5
    assert lib.qexstag_domain_create_zt(dims, (C.c_int * 2)(2, 2), 4, 8, C.byref(h)) == L.ERR_ARG  # rank 4 of 4
