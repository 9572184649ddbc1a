"""The host-communicator transport of the domain decomposition on CPU, two
processes over gloo: TorchHostComm (qexstag_host_comm over
torch.distributed) called through its C function pointers as the library
calls them, and the ghost exchange the library makes through it, replayed
on numpy extended lattices: posts receive-down (tag 0), receive-up (tag 1),
send-up (tag 0), send-down (tag 1) for t, tags 2 and 3 for z, then waits.
The peers and the order of messages are those of the NCCL transport, so
this also checks its pairing."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _swap(comm, dnr, upr, sdn, sup, rdn, rup, tag_up, tag_dn):
    c = comm.struct
    nb = sdn.nbytes
    p = lambda a: C.c_void_p(a.ctypes.data)
    assert c.push_recv(None, dnr, tag_up, p(rdn), nb) == 0
    assert c.push_recv(None, upr, tag_dn, p(rup), nb) == 0
    assert c.push_send(None, upr, tag_up, p(sup), nb) == 0
    assert c.push_send(None, dnr, tag_dn, p(sdn), nb) == 0
    assert c.wait_all(None) == 0


def _worker(rank, world, port, q, case):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import datetime
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from qex_b200 import fields as F
    from qex_b200.domain import TorchHostComm
    comm = TorchHostComm()
    try:
        if case == "messages":
            other = 1 - rank
            a = np.full(5, 10.0 * rank + 1.0)
            b = np.full(5, 10.0 * rank + 2.0)
            ra, rb = np.zeros(5), np.zeros(5)
            _swap(comm, other, other, a, b, ra, rb, 0, 1)
            # to itself (a grid with one rank along a direction)
            s1, s2 = np.arange(4.0), np.arange(4.0) + 7
            r1, r2 = np.zeros(4), np.zeros(4)
            _swap(comm, rank, rank, s1, s2, r1, r2, 2, 3)
            x = np.array([1.0 + rank, 0.5])
            assert comm.struct.all_reduce_sum(None, x.ctypes.data_as(C.POINTER(C.c_double)), 2) == 0
            q.put((rank, ra.tolist(), rb.tolist(), r1.tolist(), r2.tolist(), x.tolist()))
        else:
            gdims, Rz, Rt, h = case
            L0, L1, L2, L3 = gdims
            Z, T = L2 // Rz, L3 // Rt
            Ze, Te = Z + 2 * h, T + 2 * h
            edims = (L0, L1, Ze, Te)
            Ve = F.volume(edims)
            nh, P = Ve // 2, L0 * L1 // 2
            sh = P * Ze
            glob = np.arange(F.volume(gdims)) + 1.0
            ec = F.coords(edims)
            g = ec.copy()
            g[:, 2] = (g[:, 2] - h + (rank % Rz) * Z) % L2
            g[:, 3] = (g[:, 3] - h + (rank // Rz) * T) % L3
            ideal = glob[F.index_of(gdims, g)]
            inter = (ec[:, 2] >= h) & (ec[:, 2] < h + Z) & (ec[:, 3] >= h) & (ec[:, 3] < h + T)
            f = np.where(inter, ideal, 0.0)
            rank_of = lambda rz, rt: rz % Rz + Rz * (rt % Rt)
            rz, rt = rank % Rz, rank // Rz
            # t phase: whole slices, as domain.cu's host-communicator branch
            upr, dnr = rank_of(rz, rt + 1), rank_of(rz, rt - 1)
            for o in (0, nh):
                sup = f[o + T * sh:o + (T + h) * sh].copy()
                sdn = f[o + h * sh:o + 2 * h * sh].copy()
                rdn, rup = np.zeros_like(sup), np.zeros_like(sup)
                _swap(comm, dnr, upr, sdn, sup, rdn, rup, 0, 1)
                f[o:o + h * sh] = rdn
                f[o + (h + T) * sh:o + (T + 2 * h) * sh] = rup
            # z phase: rows [hz, 2hz) and [Z, Z + hz) of every slice, packed
            upz, dnz = rank_of(rz + 1, rt), rank_of(rz - 1, rt)
            for o in (0, nh):
                rows = lambda r0: np.concatenate([f[o + s * sh + r0 * P:o + s * sh + (r0 + h) * P] for s in range(Te)])
                sdn, sup = rows(h), rows(Z)
                rdn, rup = np.zeros_like(sdn), np.zeros_like(sup)
                _swap(comm, dnz, upz, sdn, sup, rdn, rup, 2, 3)
                w = h * P
                for s in range(Te):
                    b = o + s * sh
                    f[b:b + w] = rdn[s * w:(s + 1) * w]
                    f[b + (h + Z) * P:b + (Z + 2 * h) * P] = rup[s * w:(s + 1) * w]
            q.put((rank, bool(np.array_equal(f, ideal))))
    finally:
        dist.destroy_process_group()


def _run(case):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q, case)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    return sorted(out)


def test_torch_host_comm_messages():
    out = _run("messages")
    for rank, ra, rb, r1, r2, x in out:
        other = 1 - rank
        # my lower side receives what the other sent up (its upper face, tag 0),
        # my upper side what it sent down (its lower face, tag 1)
        assert ra == [10.0 * other + 2.0] * 5
        assert rb == [10.0 * other + 1.0] * 5
        assert r1 == list(np.arange(4.0) + 7) and r2 == list(np.arange(4.0))
        assert x == [3.0, 1.0]


@pytest.mark.parametrize("case", [((4, 4, 12, 12), 1, 2, 6), ((4, 4, 12, 12), 2, 1, 6), ((4, 4, 8, 8), 2, 1, 2)])
def test_host_comm_exchange_fills_every_ghost(case):
    """Two ranks split along t (grid 1 x 2) or along z (2 x 1, t ghosts
    exchanged with the rank itself): every extended-lattice site, corners
    included, equals the global field after the exchange."""
    assert _run(case) == [(0, True), (1, True)]
