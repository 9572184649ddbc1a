"""The domain-decomposed operator and CG with the ranks in separate
processes (QEX's one rank per process, src/layout/shifts.nim:76-103,
263-294, src/comms/commsUtils.nim:136-273): two processes, each owning a
slab of the same lattice, exchange boundary slices and sum dot products
through qexstag_domain_connect_host with TorchHostComm over a gloo process
group.  Both processes use the one GPU of the machine; every exchange and
sum is ordered on the host, so no kernel waits for the other process.
The Schur operator equals the single-lattice one bit for bit; the CG takes
the oracle's iteration count (+-1) and gives its solution."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

M = 0.05


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q, dims, grid):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import datetime
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        from qex_b200 import domain as DD
        from qex_b200 import fields as F
        from qex_b200 import stag as S
        g = F.fat_naik_links(dims, 21)
        b = F.even_source(dims, 31)
        x = F.gaussian_vector(F.volume(dims), 32)
        x[F.volume(dims) // 2:] = 0
        d = DD.DomainSet(dims, world, 8, ranks=[rank], grid=grid, host_comm=DD.TorchHostComm(), device=0)
        d.set_links(g)
        r = np.zeros_like(x)
        d.stagD2ee(r, x, M * M)
        y = np.zeros_like(b)
        sp = S.SolverParams(r2req=1e-20)
        d.solveEE(y, b, M, sp)
        y16 = np.zeros_like(b)
        sp16 = S.SolverParams(r2req=1e-20, sloppySolve=S.L.SLOPPY_HALF, delta=0.1)
        if grid is None:  # the 16-bit domain solve: splits along t
            d.solveEE(y16, b, M, sp16)
        ix = d.gidx[0]
        q.put((rank, ix, r[ix], y[ix], sp.iterations, sp.r2, sp.status, y16[ix], sp16.r2, sp16.status,
               sp16.reliable_updates, d.recon12))
        del d
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("dims,grid", [((8, 8, 8, 12), None), ((8, 8, 12, 8), (2, 1))])
def test_two_process_domain_solve(cuda, dims, grid):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q, dims, grid)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted([q.get(timeout=300) for _ in ps], key=lambda t: t[0])
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    from oracle import oracle as O
    from qex_b200 import fields as F
    from qex_b200 import stag as S
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 21)
    b = F.even_source(dims, 31)
    x = F.gaussian_vector(V, 32)
    x[V // 2:] = 0
    r = np.zeros_like(x)
    y = np.zeros_like(b)
    y16 = np.zeros_like(b)
    for rank, ix, rp, yp, its, r2, status, y16p, r216, st16, rel16, rc12 in out:
        r[ix] = rp
        y[ix] = yp
        y16[ix] = y16p
        assert status == 0 and r2 <= 1e-20
        # each slab's long links carry the global time boundary, so the
        # 16-bit links keep 12 reals on both ranks
        assert rc12
        if grid is None:
            assert st16 == 0 and r216 <= 1e-20 and rel16 >= 1
    # the Schur operator: bit for bit the single-lattice one
    s = S.Staggered(S.Layout(dims), g)
    r1 = np.zeros_like(x)
    s.stagD2ee(r1, x, M * M)
    assert np.array_equal(r[: V // 2], r1[: V // 2])
    # the CG: the oracle's iteration count and solution
    o = O.Oracle(dims, g)
    yo = o.vec()
    its_o, _ = o.solveXX(0, yo, b, M, 1e-20)
    assert out[0][4] == out[1][4] and abs(out[0][4] - its_o) <= 1
    assert np.abs(y - yo).max() / np.abs(yo).max() < 1e-8
    if grid is None:
        # the 16-bit reliable-update CG over the two processes, FP64 defect
        # correction: the oracle's solution and the FP64 true residual
        assert np.abs(y16 - yo).max() / np.abs(yo).max() < 1e-8
        ay = o.vec()
        o.stagD2ee(ay, y16, M * M)
        assert np.linalg.norm(ay[: V // 2] - b[: V // 2]) ** 2 <= 1e-20 * np.linalg.norm(b[: V // 2]) ** 2
        assert not np.any(y16[V // 2:])


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (8, 4, 6, 12)])
def test_one_domain_mixed_solve(cuda, dims):
    """The 16-bit domain solve with one domain holding the whole lattice
    (its ghosts exchanged with itself): the oracle's solution, the FP64
    true residual, and the error reported for what it does not take."""
    from oracle import oracle as O
    from qex_b200 import domain as DD
    from qex_b200 import fields as F
    from qex_b200 import stag as S
    V = F.volume(dims)
    g = F.fat_naik_links(dims, 23)
    b = F.even_source(dims, 24)
    d = DD.DomainSet(dims, 1, 8)
    d.set_links(g)
    # the ghost slices wrap around the antiperiodic boundary: the long-link
    # signs rebuilt from global time match, and 12 reals are kept
    assert d.recon12
    y = np.zeros_like(b)
    sp = S.SolverParams(r2req=1e-20, sloppySolve=S.L.SLOPPY_HALF, delta=0.1)
    d.solveEE(y, b, M, sp)
    assert sp.status == 0 and sp.r2 <= 1e-20 and sp.reliable_updates >= 1
    o = O.Oracle(dims, g)
    yo = o.vec()
    o.solveXX(0, yo, b, M, 1e-22)
    assert np.abs(y - yo).max() / np.abs(yo).max() < 1e-8
    with pytest.raises(S.L.QexStagError):
        d.solveEE(y, b, M, S.SolverParams(r2req=1e-20, sloppySolve=S.L.SLOPPY_SINGLE))
