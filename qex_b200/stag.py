"""Host-side mirror of QEX's staggered operator interface over the C ABI.

Names, argument meaning and error behaviour follow QEX:
  Layout            newLayout with SIMD width 1 (src/layout/layoutX.nim:71-180)
  Staggered         newStag / newStag3 (src/physics/stagD.nim:573-615)
    .stagD2 .stagD .D .Ddag .stagD2ee .stagD2oo   (stagD.nim:383-520, 617-622)
    .solveEE .solveOO .solve .solve_multi         (src/physics/stagSolve.nim)
    .cgm_ee                                       (src/solvers/cgm.nim)
    .force .ferm_force                            (src/hmc/hmcAction.nim:669-790)
  SolverParams      src/solvers/solverBase.nim:10-28

Fields are either host numpy arrays in QEX V=1 order, complex128 of shape
(V, 3) for colour vectors and (nlinks, V, 3, 3) for link lists, or CUDA
torch tensors in the device layout, complex128 of shape (3, V) and
(nlinks, 3, 3, V).  Host fields go through the library's host path (copies
inside the call); device fields are used in place.  A non-zero error status
from the library raises QexStagError (QEX's qexError).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

_initialised = {}


def init(device: int = 0) -> None:
    lib = L.load()
    if not _initialised.get(device):
        L.check(lib.qexstag_init(device), "qexstag_init")
        _initialised[device] = True


def set_stream(stream_ptr: int | None) -> None:
    L.check(L.load().qexstag_set_stream(C.c_void_p(stream_ptr or 0)), "qexstag_set_stream")


def synchronize() -> None:
    L.check(L.load().qexstag_synchronize(), "qexstag_synchronize")


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x, writable=False):
    """(pointer, mem flag) of a field."""
    if _is_torch(x):
        if not x.is_cuda:
            raise ValueError("torch fields must be CUDA tensors in the device layout")
        if not x.is_contiguous():
            raise ValueError("device fields must be contiguous")
        return C.c_void_p(x.data_ptr()), L.MEM_DEVICE
    if not isinstance(x, np.ndarray) or x.dtype != np.complex128 or not x.flags.c_contiguous:
        raise ValueError("host fields must be C-contiguous complex128 numpy arrays")
    if writable and not x.flags.writeable:
        raise ValueError("output field is read-only")
    return C.c_void_p(x.ctypes.data), L.MEM_HOST


def _mem_of(*fields) -> int:
    mems = {_ptr(f)[1] for f in fields}
    if len(mems) != 1:
        raise ValueError("mixing host and device fields in one call")
    return mems.pop()


class Layout:
    """V=1 checkerboard layout of a 4-d lattice."""

    def __init__(self, dims, device: int = 0):
        init(device)
        self.dims = tuple(int(d) for d in dims)
        self._lib = L.load()
        h = C.c_void_p()
        arr = (C.c_int * 4)(*self.dims)
        L.check(self._lib.qexstag_layout_create(arr, C.byref(h)), "layout_create")
        self.handle = h
        self.V = int(np.prod(self.dims))
        self.nEven = self.V - self.V // 2
        self.nOdd = self.V // 2
        self.physVol = self.V

    def index(self, x) -> int:
        out = C.c_int64()
        arr = (C.c_int * 4)(*[int(v) for v in x])
        L.check(self._lib.qexstag_layout_index(self.handle, arr, C.byref(out)), "layout_index")
        return out.value

    def shift_table(self, mu: int, length: int, subset: int) -> np.ndarray:
        n = self.V if subset == L.ALL else self.nEven
        out = np.empty(n, dtype=np.int32)
        L.check(self._lib.qexstag_layout_shift_table(self.handle, mu, length, subset,
                                                      out.ctypes.data_as(C.c_void_p)),
                "layout_shift_table")
        return out

    def ColorVector(self) -> np.ndarray:
        return np.zeros((self.V, 3), dtype=np.complex128)

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self._lib.qexstag_layout_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


@dataclass
class SolverParams:
    """Inputs and outputs of a solve, as QEX's SolverParams."""
    r2req: float = 1e-6
    maxits: int = 50000
    sloppySolve: int = L.SLOPPY_NONE
    delta: float = 0.0  # reliable-update threshold; 0 = the library's default
    verbosity: int = 0
    usePrevSoln: bool = False
    # outputs
    calls: int = 0
    iterations: int = 0
    outer_iterations: int = 0
    reliable_updates: int = 0
    seconds: float = 0.0
    flops: float = 0.0
    r2: float = 0.0
    kernel_launches: int = 0
    status: int = 0

    def c_params(self) -> L.SolverParamsC:
        p = L.SolverParamsC()
        p.r2req = self.r2req
        p.maxits = self.maxits
        p.sloppy = self.sloppySolve
        p.delta = self.delta
        p.verbosity = self.verbosity
        p.use_prev_soln = 1 if self.usePrevSoln else 0
        return p

    def take(self, st: L.SolverStatsC, status: int) -> None:
        self.calls = st.calls
        self.iterations = st.iterations
        self.outer_iterations = st.outer_iterations
        self.reliable_updates = st.reliable_updates
        self.seconds = st.seconds
        self.flops = st.flops
        self.r2 = st.r2
        self.kernel_launches = st.kernel_launches
        self.status = status

    def getStats(self) -> str:
        gf = 1e-9 * self.flops / max(self.seconds, 1e-12)
        return f"{self.iterations}  {self.seconds:.4g}s  {gf:.4g}Gf/s  {self.r2:.4g}"


class Staggered:
    """Staggered operator on a layout with a link list (4 naive or 8 fat+Naik
    interleaved, phases folded in)."""

    def __init__(self, layout: Layout, links, long_coeff: float = 1.0):
        self.l = layout
        self._lib = layout._lib
        nl = int(links.shape[0])
        if nl not in (4, 8):
            raise ValueError("link list must hold 4 (naive) or 8 (fat+Naik) fields")
        ptr, mem = _ptr(links)
        if mem == L.MEM_HOST and links.shape != (nl, layout.V, 3, 3):
            raise ValueError("host links must have shape (nlinks, V, 3, 3)")
        if mem == L.MEM_DEVICE and tuple(links.shape) != (nl, 3, 3, layout.V):
            raise ValueError("device links must have shape (nlinks, 3, 3, V)")
        h = C.c_void_p()
        L.check(self._lib.qexstag_links_create(layout.handle, nl, ptr, mem, float(long_coeff),
                                                C.byref(h)), "links_create")
        self.handle = h
        self.nlinks = nl

    def update_links(self, links) -> None:
        """New link data for this operator (QEX's Staggered.g changed)."""
        ptr, mem = _ptr(links)
        L.check(self._lib.qexstag_links_update(self.handle, ptr, mem), "links_update")

    @classmethod
    def from_milc(cls, layout: Layout, fat: np.ndarray, lng: np.ndarray | None = None,
                  long_coeff: float = 1.0) -> "Staggered":
        """Operator from links in MILC order, as QUDA's MILC interface takes
        them (qudaWrapperImpl.nim:205-245): host complex128 arrays of shape
        (V, 4, 3, 3), the four directions of a site together; lng None for a
        naive operator."""
        self = cls.__new__(cls)
        self.l = layout
        self._lib = layout._lib
        fat = cls._milc_array(layout, fat)
        lp = None if lng is None else cls._milc_array(layout, lng)
        h = C.c_void_p()
        L.check(self._lib.qexstag_links_create_milc(layout.handle, C.c_void_p(fat.ctypes.data),
                                                    None if lp is None else C.c_void_p(lp.ctypes.data),
                                                    float(long_coeff), C.byref(h)), "links_create_milc")
        self.handle = h
        self.nlinks = 4 if lng is None else 8
        return self

    @staticmethod
    def _milc_array(layout, a):
        if not isinstance(a, np.ndarray) or a.dtype != np.complex128 or not a.flags.c_contiguous \
                or a.shape != (layout.V, 4, 3, 3):
            raise ValueError("MILC-order links must be C-contiguous complex128 arrays of shape (V, 4, 3, 3)")
        return a

    def update_links_milc(self, fat: np.ndarray, lng: np.ndarray | None = None) -> None:
        fat = self._milc_array(self.l, fat)
        lp = None if lng is None else self._milc_array(self.l, lng)
        L.check(self._lib.qexstag_links_update_milc(self.handle, C.c_void_p(fat.ctypes.data),
                                                    None if lp is None else C.c_void_p(lp.ctypes.data)),
                "links_update_milc")

    def links_milc(self):
        """The operator's FP64 links in MILC order: (fat, long) arrays of
        shape (V, 4, 3, 3); long is None for a naive operator."""
        fat = np.empty((self.l.V, 4, 3, 3), dtype=np.complex128)
        lng = np.empty_like(fat) if self.nlinks == 8 else None
        L.check(self._lib.qexstag_links_get_milc(self.handle, C.c_void_p(fat.ctypes.data),
                                                 None if lng is None else C.c_void_p(lng.ctypes.data)),
                "links_get_milc")
        return fat, lng

    def rephase(self) -> None:
        """QEX's rephase(s) exactly: setBC + stagPhase on the first four
        fields of the link list (for a fat+Naik list: fat_0, long_0, fat_1,
        long_1, as QEX's own call does)."""
        L.check(self._lib.qexstag_links_rephase(self.handle), "links_rephase")

    def rephase_all(self) -> None:
        """Fold the staggered phases and boundary signs into (or out of)
        every field of the list by its own direction and hop."""
        L.check(self._lib.qexstag_links_rephase_all(self.handle), "links_rephase_all")

    @property
    def recon12(self) -> bool:
        return bool(self._lib.qexstag_links_recon12(self.handle))

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self._lib.qexstag_links_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    # ---- Dslash ----
    def stagD2(self, subset: int, r, x, a: float, b: float) -> None:
        mem = _mem_of(r, x)
        L.check(self._lib.qexstag_stagD2(self.handle, subset, _ptr(r, True)[0], _ptr(x)[0],
                                         float(a), float(b), mem), "stagD2")

    def stagDN(self, subset: int, rs, xs, m: float) -> None:
        """stagDN (stagD.nim:451-455): rs[i] = m xs[i] + (2D) xs[i] on the
        subset for every i, each link read once per site for up to 8
        fields."""
        if len(rs) != len(xs) or not rs:
            raise ValueError("stagDN needs equally many (>= 1) outputs and inputs")
        mem = _mem_of(*rs, *xs)
        n = len(rs)
        ra = (C.c_void_p * n)(*[_ptr(r, True)[0] for r in rs])
        xa = (C.c_void_p * n)(*[_ptr(x)[0] for x in xs])
        L.check(self._lib.qexstag_stagDN(self.handle, subset, n, ra, xa, float(m), mem), "stagDN")

    def stagD(self, subset: int, r, x, m: float, sc: float = 1.0, a: float = 0.0) -> None:
        mem = _mem_of(r, x)
        L.check(self._lib.qexstag_stagD(self.handle, subset, _ptr(r, True)[0], _ptr(x)[0],
                                        float(m), float(sc), float(a), mem), "stagD")

    def D(self, r, x, m: float) -> None:
        mem = _mem_of(r, x)
        L.check(self._lib.qexstag_D(self.handle, _ptr(r, True)[0], _ptr(x)[0], float(m), mem), "D")

    def Ddag(self, r, x, m: float) -> None:
        mem = _mem_of(r, x)
        L.check(self._lib.qexstag_Ddag(self.handle, _ptr(r, True)[0], _ptr(x)[0], float(m), mem),
                "Ddag")

    def stagD2ee(self, r, x, m2: float) -> None:
        mem = _mem_of(r, x)
        L.check(self._lib.qexstag_stagD2ee(self.handle, _ptr(r, True)[0], _ptr(x)[0], float(m2),
                                           mem), "stagD2ee")

    def stagD2oo(self, r, x, m2: float) -> None:
        mem = _mem_of(r, x)
        L.check(self._lib.qexstag_stagD2oo(self.handle, _ptr(r, True)[0], _ptr(x)[0], float(m2),
                                           mem), "stagD2oo")

    # ---- solvers ----
    def _solve_call(self, fn, name, out, inp, m, sp: SolverParams) -> None:
        mem = _mem_of(out, inp)
        p = sp.c_params()
        st = L.SolverStatsC()
        rc = fn(self.handle, _ptr(out, True)[0], _ptr(inp)[0], float(m), C.byref(p), C.byref(st),
                mem)
        L.check(rc, name)
        sp.take(st, rc)

    def solveEE(self, r, x, m: float, sp: SolverParams) -> None:
        """solveEE: stagD2ee(m^2) r = x on even sites (stagSolve.nim:423)."""
        self._solve_call(self._lib.qexstag_solveEE, "solveEE", r, x, m, sp)

    def solveOO(self, r, x, m: float, sp: SolverParams) -> None:
        self._solve_call(self._lib.qexstag_solveOO, "solveOO", r, x, m, sp)

    def solve(self, x, b, m: float, sp: SolverParams) -> None:
        """solve: D(m) x = b on all sites (stagSolve.nim:469)."""
        self._solve_call(self._lib.qexstag_solve, "solve", x, b, m, sp)

    def solve_multi(self, xs, b, ms, sp: SolverParams) -> None:
        """Multi-mass solve: D(ms[k]) xs[k] = b (stagSolve.nim:560)."""
        mem = _mem_of(b, *xs)
        n = len(xs)
        arr = (C.c_void_p * n)(*[_ptr(x, True)[0] for x in xs])
        msa = (C.c_double * n)(*[float(v) for v in ms])
        p = sp.c_params()
        st = L.SolverStatsC()
        rc = self._lib.qexstag_solve_multishift(self.handle, n, arr, _ptr(b)[0], msa, C.byref(p),
                                                C.byref(st), mem)
        L.check(rc, "solve_multishift")
        sp.take(st, rc)

    def cgm_ee(self, m: float, sigmas, bs, ys, sp: SolverParams) -> np.ndarray:
        """(A + sigma_k) y[j][k] = b[j] on even sites, A = stagD2ee(m^2).
        ys is a list over right-hand sides of lists over shifts.  Returns the
        final true relative residuals, shape (nrhs, nshift)."""
        nrhs, nsh = len(bs), len(sigmas)
        flat = [y for row in ys for y in row]
        mem = _mem_of(*bs, *flat)
        barr = (C.c_void_p * nrhs)(*[_ptr(b)[0] for b in bs])
        yarr = (C.c_void_p * (nrhs * nsh))(*[_ptr(y, True)[0] for y in flat])
        sarr = (C.c_double * nsh)(*[float(s) for s in sigmas])
        r2 = np.zeros(nrhs * nsh, dtype=np.float64)
        p = sp.c_params()
        st = L.SolverStatsC()
        rc = self._lib.qexstag_cgm_ee(self.handle, float(m), nsh, sarr, nrhs, barr, yarr, C.byref(p),
                                      C.byref(st), r2.ctypes.data_as(L.DP), mem)
        L.check(rc, "cgm_ee")
        sp.take(st, rc)
        return r2.reshape(nrhs, nsh)

    def bench_schur(self, prec: int, nrep: int = 20, m2: float = 1e-4) -> float:
        """Seconds per even-parity Schur operator call in precision prec
        (0 FP64, 1 FP32, 2 FP16), timed with CUDA events in the library."""
        out = C.c_double()
        L.check(self._lib.qexstag_bench_schur(self.handle, prec, nrep, m2, C.byref(out)),
                "bench_schur")
        return out.value

    # ---- force ----
    def force(self, f, phi, m: float, sp: SolverParams) -> None:
        """stagForceSolve + fermForce (no smearing): f receives the force QEX
        hands to addForce(gf, 0.25*dtau, f)."""
        mem = _mem_of(f, phi)
        p = sp.c_params()
        st = L.SolverStatsC()
        rc = self._lib.qexstag_force(self.handle, _ptr(f, True)[0], _ptr(phi)[0], float(m),
                                     C.byref(p), C.byref(st), mem)
        L.check(rc, "force")
        sp.take(st, rc)

    def force_solve(self, psi, phi, m: float, sp: SolverParams) -> None:
        """stagForceSolve: psi = (4y, (2D)_oe 4y), stagD2ee(m^2) y = phi_e."""
        self._solve_call(self._lib.qexstag_force_solve, "force_solve", psi, phi, m, sp)

    def ferm_outer(self, f, psi) -> None:
        """fermForce's outer products f1 (and f3 for long links), odd sites
        negated, before the chain rule and projection."""
        mem = _mem_of(f, psi)
        L.check(self._lib.qexstag_ferm_outer(self.handle, _ptr(f, True)[0], _ptr(psi)[0], mem),
                "ferm_outer")

    def ferm_force(self, f, psi) -> None:
        mem = _mem_of(f, psi)
        L.check(self._lib.qexstag_ferm_force(self.handle, _ptr(f, True)[0], _ptr(psi)[0], mem),
                "ferm_force")


def solve_batched(stags, xs, bs, masses, sp: SolverParams):
    """Independent even-site solves stagD2ee(m_j^2) x_j = b_j for operators
    on different lattices, all in one persistent launch.  Returns per-problem
    iterations, true relative residuals and the launch configuration."""
    lib = L.load()
    n = len(stags)
    mem = _mem_of(*xs, *bs)
    harr = (C.c_void_p * n)(*[s.handle for s in stags])
    xarr = (C.c_void_p * n)(*[_ptr(x, True)[0] for x in xs])
    barr = (C.c_void_p * n)(*[_ptr(b)[0] for b in bs])
    marr = (C.c_double * n)(*[float(m) for m in masses])
    its = (C.c_int * n)()
    r2 = np.zeros(n, dtype=np.float64)
    info = (C.c_int * 3)()
    p = sp.c_params()
    st = L.SolverStatsC()
    rc = lib.qexstag_solve_batched(n, harr, marr, xarr, barr, C.byref(p), its, r2.ctypes.data_as(L.DP),
                                   info, C.byref(st), mem)
    L.check(rc, "solve_batched")
    sp.take(st, rc)
    return {"iterations": list(its), "r2": r2, "block": info[0], "blocks_per_sm": info[1],
            "graph": bool(info[2])}


def newStag(layout: Layout, g) -> Staggered:
    """Naive staggered operator from 4 phased link fields."""
    return Staggered(layout, g)


def newStag3(layout: Layout, fat, lng, long_coeff: float = 1.0) -> Staggered:
    """Fat+Naik operator from 4 fat and 4 long phased link fields."""
    if _is_torch(fat):
        import torch
        g = torch.empty((8,) + tuple(fat.shape[1:]), dtype=fat.dtype, device=fat.device)
        g[0::2] = fat
        g[1::2] = lng
    else:
        from .fields import interleave
        g = interleave(np.asarray(fat), np.asarray(lng))
    return Staggered(layout, g, long_coeff)


def to_device_vector(x: np.ndarray, device="cuda"):
    """Host (V, 3) colour vector -> device layout (3, V) complex128 tensor."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(x.T)).to(device)


def to_host_vector(t) -> np.ndarray:
    return np.ascontiguousarray(t.detach().cpu().numpy().T)


def to_device_links(g: np.ndarray, device="cuda"):
    """Host (n, V, 3, 3) links -> device layout (n, 3, 3, V) tensor."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.moveaxis(g, 1, 3))).to(device)


def to_host_links(t) -> np.ndarray:
    return np.ascontiguousarray(np.moveaxis(t.detach().cpu().numpy(), 3, 1))
