"""Domain decomposition along t through the C ABI (qexstag_domain_*): QEX's
rank split of the lattice (rankGeom; src/layout/shifts.nim, qshifts.nim)
with ghost-slice exchanges.  A process holds either every rank's domain
(one device, exchanges by device copies) or one (one rank per process,
exchanges and sums by NCCL, or through a host communicator such as
TorchHostComm over a torch.distributed process group).

Global host fields are split into rank slabs here for convenience: links
(nlinks, V, 3, 3) and colour vectors (V, 3) in the global V=1 order.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from . import fields as F
from . import stag as S


def _arr(ptrs):
    return (C.c_void_p * len(ptrs))(*ptrs)


_PUSH = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_size_t)
_WAIT = C.CFUNCTYPE(C.c_int, C.c_void_p)
_SUM = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_double), C.c_int)


class HostCommC(C.Structure):
    """qexstag_host_comm"""
    _fields_ = [("ctx", C.c_void_p), ("push_send", _PUSH), ("push_recv", _PUSH), ("wait_all", _WAIT),
                ("all_reduce_sum", _SUM)]


class TorchHostComm:
    """qexstag_host_comm over a torch.distributed process group (gloo, or
    any backend that sends CPU tensors): the shape of QEX's Comm object
    (src/comms/comms.nim: pushSend, pushRecv, waitSends/waitRecvs,
    allReduce).  Messages to this process's own rank (a grid with one rank
    along a direction) are copied in memory.  Callbacks return 1 on any
    exception, which the library reports as an error."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.me = dist.get_rank(group)
        self.reqs = []
        self.self_recv = []  # (tag, address, bytes) posted to this rank itself
        self._cbs = (_PUSH(self._send), _PUSH(self._recv), _WAIT(self._wait), _SUM(self._sum))
        self.struct = HostCommC(None, *self._cbs)

    @staticmethod
    def _view(addr, nbytes):
        import torch
        return torch.from_numpy(np.ctypeslib.as_array((C.c_uint8 * nbytes).from_address(addr)))

    def _send(self, ctx, rank, tag, buf, nbytes):
        try:
            if rank == self.me:
                for i, (t, a, n) in enumerate(self.self_recv):
                    if t == tag and n == nbytes:
                        C.memmove(a, buf, nbytes)
                        del self.self_recv[i]
                        return 0
                return 1
            t = self._view(buf, nbytes)
            self.reqs.append((self.dist.isend(t, dst=rank, group=self.group, tag=tag), t))
            return 0
        except Exception:
            return 1

    def _recv(self, ctx, rank, tag, buf, nbytes):
        try:
            if rank == self.me:
                self.self_recv.append((tag, buf, nbytes))
                return 0
            t = self._view(buf, nbytes)
            self.reqs.append((self.dist.irecv(t, src=rank, group=self.group, tag=tag), t))
            return 0
        except Exception:
            return 1

    def _wait(self, ctx):
        try:
            for r, _ in self.reqs:
                r.wait()
            self.reqs.clear()
            return 0 if not self.self_recv else 1
        except Exception:
            return 1

    def _sum(self, ctx, x, n):
        try:
            import torch
            t = torch.from_numpy(np.ctypeslib.as_array(x, shape=(n,)))
            self.dist.all_reduce(t, group=self.group)
            return 0
        except Exception:
            return 1


def rank_sites(global_dims, local_dims, grid, rank: int) -> np.ndarray:
    """Global V=1 index of each site of rank's local lattice, in the local
    V=1 order: rank = rz + Rz rt holds z rows [rz Z, (rz+1) Z) of slices
    [rt T, (rt+1) T)."""
    g = F.coords(tuple(local_dims))
    g[:, 2] += (rank % grid[0]) * local_dims[2]
    g[:, 3] += (rank // grid[0]) * local_dims[3]
    return F.index_of(tuple(global_dims), g)


class DomainSet:
    """The domains this process holds: ranks[0..] of an nranks split along t,
    or, with grid = (Rz, Rt), of an Rz x Rt split along t and z (nranks =
    Rz Rt, rank = rz + Rz rt)."""

    def __init__(self, global_dims, nranks: int, nlinks: int, ranks=None, nccl_id: bytes | None = None,
                 grid=None, host_comm: TorchHostComm | None = None, device: int = 0):
        S.init(device)
        self.lib = L.load()
        self.gdims = tuple(int(d) for d in global_dims)
        self.grid = (1, nranks) if grid is None else (int(grid[0]), int(grid[1]))
        if grid is not None and self.grid[0] * self.grid[1] != nranks:
            raise ValueError("grid does not hold nranks ranks")
        self.nranks = nranks
        self.nl = nlinks
        self.ranks = list(range(nranks)) if ranks is None else list(ranks)
        self.handles = []
        dims = (C.c_int * 4)(*self.gdims)
        for r in self.ranks:
            h = C.c_void_p()
            if grid is None:
                rc = self.lib.qexstag_domain_create(dims, nranks, r, nlinks, C.byref(h))
            else:
                rc = self.lib.qexstag_domain_create_zt(dims, (C.c_int * 2)(*self.grid), r, nlinks, C.byref(h))
            L.check(rc, "domain_create")
            self.handles.append(h)
        ld = (C.c_int * 4)()
        L.check(self.lib.qexstag_domain_local_dims(self.handles[0], ld), "domain_local_dims")
        self.ldims = tuple(ld)
        self.host_comm = host_comm  # keeps the callbacks alive
        if host_comm is not None:
            for h in self.handles:
                L.check(self.lib.qexstag_domain_connect_host(h, C.byref(host_comm.struct)), "domain_connect_host")
        elif nccl_id is None:
            L.check(self.lib.qexstag_domain_connect_local(self._set(), len(self.handles)), "domain_connect_local")
        else:
            buf = C.create_string_buffer(bytes(nccl_id), 128)
            for h in self.handles:
                L.check(self.lib.qexstag_domain_connect_nccl(h, buf), "domain_connect_nccl")
        # global index of each local site, per rank
        self.gidx = [rank_sites(self.gdims, self.ldims, self.grid, r) for r in self.ranks]

    def _set(self):
        return _arr([h.value for h in self.handles])

    def __del__(self):
        try:
            for h in getattr(self, "handles", []):
                self.lib.qexstag_domain_destroy(h)
            self.handles = []
        except Exception:
            pass

    def split_links(self, g: np.ndarray):
        return [np.ascontiguousarray(g[:, ix]) for ix in self.gidx]

    def split_vector(self, x: np.ndarray):
        return [np.ascontiguousarray(x[ix]) for ix in self.gidx]

    def gather_vector(self, parts, out: np.ndarray):
        for ix, p in zip(self.gidx, parts):
            out[ix] = p
        return out

    @property
    def recon12(self) -> bool:
        """True when every domain keeps 12-real reduced-precision long links."""
        return all(self.lib.qexstag_domain_recon12(h) == 1 for h in self.handles)

    def set_links(self, g: np.ndarray) -> None:
        self._links = self.split_links(np.ascontiguousarray(g, dtype=np.complex128))
        L.check(self.lib.qexstag_domain_links(self._set(), len(self.handles),
                                              _arr([a.ctypes.data for a in self._links]), L.MEM_HOST),
                "domain_links")

    def set_links_local(self, parts) -> None:
        """Each domain's links in its local V=1 order, (nlinks, Vloc, 3, 3)
        host arrays or (nlinks, 3, 3, Vloc) device tensors, phases folded in
        with global coordinates."""
        self._links = list(parts)
        ptrs, mem = zip(*[S._ptr(a) for a in self._links])
        if len(set(mem)) != 1:
            raise ValueError("mixing host and device links")
        L.check(self.lib.qexstag_domain_links(self._set(), len(self.handles), _arr([p.value for p in ptrs]), mem[0]),
                "domain_links")

    def solveEE_local(self, xs, bs, m: float, sp: S.SolverParams) -> None:
        """solveEE with each domain's fields in its local V=1 order (host
        (Vloc, 3) arrays or device (3, Vloc) tensors)."""
        mem = S._mem_of(*xs, *bs)
        st = L.SolverStatsC()
        pc = sp.c_params()
        rc = self.lib.qexstag_domain_solveEE(self._set(), len(self.handles), _arr([S._ptr(a, True)[0].value for a in xs]),
                                             _arr([S._ptr(a)[0].value for a in bs]), m, C.byref(pc), C.byref(st), mem)
        L.check(rc, "domain_solveEE")
        sp.take(st, rc)

    def stagD2ee(self, r: np.ndarray, x: np.ndarray, m2: float) -> None:
        xs = self.split_vector(x)
        rs = self.split_vector(r)
        L.check(self.lib.qexstag_domain_stagD2ee(self._set(), len(self.handles), _arr([a.ctypes.data for a in rs]),
                                                 _arr([a.ctypes.data for a in xs]), m2, L.MEM_HOST),
                "domain_stagD2ee")
        self.gather_vector(rs, r)

    def solveEE(self, x: np.ndarray, b: np.ndarray, m: float, sp: S.SolverParams) -> None:
        bs = self.split_vector(b)
        xs = [np.zeros_like(v) for v in bs]
        st = L.SolverStatsC()
        pc = sp.c_params()
        rc = self.lib.qexstag_domain_solveEE(self._set(), len(self.handles), _arr([a.ctypes.data for a in xs]),
                                             _arr([a.ctypes.data for a in bs]), m, C.byref(pc), C.byref(st),
                                             L.MEM_HOST)
        L.check(rc, "domain_solveEE")
        sp.take(st, rc)
        self.gather_vector(xs, x)


def nccl_unique_id() -> bytes:
    buf = C.create_string_buffer(128)
    L.check(L.load().qexstag_nccl_unique_id(buf), "nccl_unique_id")
    return buf.raw


def main():
    """Device seconds of the FP64 domain CG for stagD2ee(m^2) y = b at --dims
    (fat + Naik fields and source as the 32^4 benchmark's, m = 0.01,
    r2req = 1e-20) with R ranks held by this process on one device, for each
    R in --ranks, beside the one-lattice FP64 CG on the same problem."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="32,32,32,32")
    ap.add_argument("--ranks", default="1,2")
    ap.add_argument("--grids", default="", help="splits along t and z as RzxRt, e.g. 2x1,2x2")
    ap.add_argument("--mass", type=float, default=0.01)
    ap.add_argument("--r2req", type=float, default=1e-20)
    a = ap.parse_args()
    dims = tuple(int(v) for v in a.dims.split(","))
    S.init(0)
    g = F.fat_naik_links(dims, 21)
    b = F.even_source(dims, 31)
    one = S.Staggered(S.Layout(dims), g)
    x = np.zeros_like(b)
    sp = S.SolverParams(r2req=a.r2req)
    one.solveEE(x, b, a.mass, sp)  # warm-up
    sp = S.SolverParams(r2req=a.r2req)
    one.solveEE(x, b, a.mass, sp)
    out = {"dims": dims, "mass": a.mass, "one_lattice": {"iterations": sp.iterations, "seconds": sp.seconds}}
    for R in (int(v) for v in a.ranks.split(",")):
        d = DomainSet(dims, R, 8)
        d.set_links(g)
        for _ in range(2):  # warm-up, then the timed solve
            y = np.zeros_like(b)
            sp = S.SolverParams(r2req=a.r2req)
            d.solveEE(y, b, a.mass, sp)
        out[f"ranks_{R}"] = {"slab": d.ldims[3], "iterations": sp.iterations, "seconds": sp.seconds,
                             "true_r2": sp.r2, "max_diff_vs_one_lattice": float(np.abs(y - x).max())}
        del d
    for spec in (v for v in a.grids.split(",") if v):
        Rz, Rt = (int(v) for v in spec.split("x"))
        d = DomainSet(dims, Rz * Rt, 8, grid=(Rz, Rt))
        d.set_links(g)
        for _ in range(2):
            y = np.zeros_like(b)
            sp = S.SolverParams(r2req=a.r2req)
            d.solveEE(y, b, a.mass, sp)
        out[f"grid_{Rz}x{Rt}"] = {"local": d.ldims, "iterations": sp.iterations, "seconds": sp.seconds,
                                  "true_r2": sp.r2, "max_diff_vs_one_lattice": float(np.abs(y - x).max())}
        del d
    print(json.dumps(out))


if __name__ == "__main__":
    main()
