"""ctypes wrapper of the CPU oracle (qexstag_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, the smoke check and the CPU
baseline leg of bench.py, as the checker.  Parity is pinned against QEX's
logged solver output on the free HISQ field and otherwise by known answers:
see the header of qexstag_oracle.c.

Fields use the QEX V=1 host layout: complex128 (V, 3) colour vectors and
(nlinks, V, 3, 3) link lists.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"

_lib = None


def build() -> Path:
    srcs = [HERE / "qexstag_oracle.c", HERE / "smear_oracle.c", HERE / "io_oracle.c", HERE / "hmc_oracle.c"]
    if not LIB.exists() or any(LIB.stat().st_mtime < s.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        l = C.CDLL(str(LIB))
        P, D, I = C.c_void_p, C.c_double, C.c_int
        DP = C.POINTER(C.c_double)
        sig = {
            "or_index": (C.c_long, [C.POINTER(C.c_int), C.POINTER(C.c_int)]),
            "or_coords": (None, [C.POINTER(C.c_int), P]),
            "or_shift_table": (None, [C.POINTER(C.c_int), I, I, I, P]),
            "or_ctx_create": (P, [C.POINTER(C.c_int), I, P]),
            "or_ctx_set_links": (None, [P, P]),
            "or_ctx_destroy": (None, [P]),
            "or_stag_eta": (I, [I, C.POINTER(C.c_int)]),
            "or_apply_phases": (None, [C.POINTER(C.c_int), I, P]),
            "or_stagD2": (None, [P, I, P, P, D, D]),
            "or_stagD": (None, [P, I, P, P, D, D, D]),
            "or_D": (None, [P, P, P, D]),
            "or_Ddag": (None, [P, P, P, D]),
            "or_stagD2ee": (None, [P, P, P, D]),
            "or_stagD2oo": (None, [P, P, P, D]),
            "or_stagD2ee_par": (None, [P, I, P, P, D]),
            "or_norm2": (D, [P, I, P]),
            "or_redot": (D, [P, I, P, P]),
            "or_cg_xx": (I, [P, I, P, P, D, D, I, DP]),
            "or_cg_begin": (P, [P, I, P, P, D, D]),
            "or_cg_run": (I, [P, I]),
            "or_cg_converged": (I, [P]),
            "or_cg_end": (I, [P, DP]),
            "or_solveXX": (I, [P, I, P, P, D, D, I, DP]),
            "or_eoReconstruct": (None, [P, P, P, D]),
            "or_solve": (I, [P, P, P, D, D, I, DP]),
            "or_cgm_xx": (I, [P, I, I, C.POINTER(C.c_void_p), DP, P, D, D, I, DP]),
            "or_solve_multishift": (I, [P, I, C.POINTER(C.c_void_p), P, DP, D, I, DP]),
            "or_project_tah": (None, [P, P]),
            "or_force_solve": (I, [P, P, P, D, D, I, DP]),
            "or_ferm_force": (None, [P, P, P]),
            "or_ferm_outer": (None, [P, P, P]),
            "or_force": (I, [P, P, P, D, D, I, DP]),
            "or_num_threads": (I, []),
            "or_fat7": (None, [C.POINTER(C.c_int), DP, P, P, P, P, D]),
            "or_project_u": (None, [C.c_long, P, P, D]),
            "or_hisq_smear": (None, [C.POINTER(C.c_int), DP, DP, D, D, P, P, P]),
            "or_fat7_deriv": (None, [C.POINTER(C.c_int), DP, P, P, P, P, P, P, D]),
            "or_project_u_deriv": (None, [C.c_long, P, P, P, P, D]),
            "or_sylsolve": (None, [C.c_long, P, P, P]),
            "or_hisq_deriv": (None, [C.POINTER(C.c_int), DP, DP, D, D, P, P, P, P]),
            "or_crc32": (C.c_uint32, [P, C.c_size_t]),
            "or_gauge_action": (D, [C.POINTER(C.c_int), D, D, P]),
            "or_gauge_force": (None, [C.POINTER(C.c_int), D, D, P, P]),
            "or_exp_ah": (None, [C.c_long, P, D, P]),
            "or_link_update": (None, [C.c_long, P, P, D]),
            "or_scidac_checksum": (None, [P, C.c_long, C.c_long, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
            "or_milc_checksum": (None, [P, C.c_long, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return C.c_void_p(a.ctypes.data)


def _dims(dims):
    return (C.c_int * 4)(*[int(d) for d in dims])


def index(dims, x) -> int:
    return lib().or_index(_dims(dims), (C.c_int * 4)(*[int(v) for v in x]))


def shift_table(dims, mu, length, parity) -> np.ndarray:
    V = int(np.prod(dims))
    n = V if parity == 2 else V // 2
    out = np.empty(n, dtype=np.int32)
    lib().or_shift_table(_dims(dims), mu, length, parity, _p(out))
    return out


def apply_phases(dims, links: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(links.copy())
    lib().or_apply_phases(_dims(dims), out.shape[0], _p(out))
    return out


def project_tah(m: np.ndarray) -> np.ndarray:
    m = np.ascontiguousarray(m, dtype=np.complex128)
    out = np.empty_like(m)
    lib().or_project_tah(_p(out), _p(m))
    return out


class Oracle:
    """The oracle's operator on one lattice and link list."""

    def __init__(self, dims, links: np.ndarray):
        self.dims = tuple(int(d) for d in dims)
        self.V = int(np.prod(self.dims))
        self.links = np.ascontiguousarray(links, dtype=np.complex128)
        assert self.links.shape[1:] == (self.V, 3, 3)
        self.nlinks = self.links.shape[0]
        self.ctx = lib().or_ctx_create(_dims(self.dims), self.nlinks, _p(self.links))

    def __del__(self):
        if getattr(self, "ctx", None):
            lib().or_ctx_destroy(self.ctx)
            self.ctx = None

    def vec(self) -> np.ndarray:
        return np.zeros((self.V, 3), dtype=np.complex128)

    def stagD2(self, parity, r, x, a, b):
        lib().or_stagD2(self.ctx, parity, _p(r), _p(x), a, b)

    def stagD(self, parity, r, x, m, sc=1.0, a=0.0):
        lib().or_stagD(self.ctx, parity, _p(r), _p(x), m, sc, a)

    def D(self, r, x, m):
        lib().or_D(self.ctx, _p(r), _p(x), m)

    def Ddag(self, r, x, m):
        lib().or_Ddag(self.ctx, _p(r), _p(x), m)

    def stagD2ee(self, r, x, m2):
        lib().or_stagD2ee(self.ctx, _p(r), _p(x), m2)

    def stagD2oo(self, r, x, m2):
        lib().or_stagD2oo(self.ctx, _p(r), _p(x), m2)

    def norm2(self, parity, x) -> float:
        return lib().or_norm2(self.ctx, parity, _p(x))

    def cg(self, parity, x, b, m2, r2req, maxits=100000):
        r2 = C.c_double()
        its = lib().or_cg_xx(self.ctx, parity, _p(x), _p(b), m2, r2req, maxits, C.byref(r2))
        return its, r2.value

    def cg_steps(self, parity, x, b, m2, r2req):
        """The same CG as cg(), run in pieces: returns a CgRun whose
        run(n) performs up to n more iterations."""
        return CgRun(self, parity, x, b, m2, r2req)

    def solveXX(self, parity, r, x, m, r2req, maxits=100000):
        r2 = C.c_double()
        its = lib().or_solveXX(self.ctx, parity, _p(r), _p(x), m, r2req, maxits, C.byref(r2))
        return its, r2.value

    def solve(self, x, b, m, r2req, maxits=100000):
        r2 = C.c_double()
        its = lib().or_solve(self.ctx, _p(x), _p(b), m, r2req, maxits, C.byref(r2))
        return its, r2.value

    def cgm(self, parity, xs, sg, b, m2, r2req, maxits=100000):
        n = len(xs)
        arr = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
        sga = (C.c_double * n)(*[float(s) for s in sg])
        r2 = C.c_double()
        its = lib().or_cgm_xx(self.ctx, parity, n, arr, sga, _p(b), m2, r2req, maxits, C.byref(r2))
        return its, r2.value

    def solve_multishift(self, xs, b, ms, r2req, maxits=100000):
        n = len(xs)
        arr = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
        msa = (C.c_double * n)(*[float(s) for s in ms])
        r2 = C.c_double()
        its = lib().or_solve_multishift(self.ctx, n, arr, _p(b), msa, r2req, maxits, C.byref(r2))
        return its, r2.value

    def force_solve(self, psi, phi, m, r2req, maxits=100000):
        r2 = C.c_double()
        its = lib().or_force_solve(self.ctx, _p(psi), _p(phi), m, r2req, maxits, C.byref(r2))
        return its, r2.value

    def ferm_force(self, f, psi):
        lib().or_ferm_force(self.ctx, _p(f), _p(psi))

    def ferm_outer(self, f, psi):
        lib().or_ferm_outer(self.ctx, _p(f), _p(psi))

    def force(self, f, phi, m, r2req, maxits=100000):
        r2 = C.c_double()
        its = lib().or_force(self.ctx, _p(f), _p(phi), m, r2req, maxits, C.byref(r2))
        return its, r2.value


def num_threads() -> int:
    return lib().or_num_threads()


# ---- HISQ smearing (smear_oracle.c) ------------------------------------
# coefficient order {oneLink, threeStaple, fiveStaple, sevenStaple, lepage}


def hisq_fat7_coefs(f7lf: float, naik: float):
    """setHisqFat7 (src/physics/hisqLinks.nim:10-15)."""
    return [(1.0 + 3.0 * f7lf + naik) / 8.0, -1.0 / 16.0, 1.0 / 64.0, -1.0 / 384.0, -f7lf / 16.0]


def hisq_coefs(lepage: float = 0.0, naik: float = 1.0):
    """newHISQ (src/gauge/hisqsmear.nim:53-64): (first, second, naik)."""
    return hisq_fat7_coefs(lepage, 0.0), hisq_fat7_coefs(2.0 - lepage, naik), -naik / 24.0


def _coef(c):
    return (C.c_double * 5)(*[float(v) for v in c])


def fat7(dims, coefs, gf: np.ndarray, gfl: np.ndarray | None = None, naik: float = 0.0):
    """makeImpLinks (src/gauge/fat7l.nim:70-154) on (4, V, 3, 3) fields;
    returns fl, or (fl, ll) when gfl is given."""
    gf = np.ascontiguousarray(gf, dtype=np.complex128)
    fl = np.empty_like(gf)
    if gfl is None:
        lib().or_fat7(_dims(dims), _coef(coefs), _p(gf), _p(fl), None, None, 0.0)
        return fl
    gfl = np.ascontiguousarray(gfl, dtype=np.complex128)
    ll = np.zeros_like(gfl)  # left untouched when naik == 0, as makeImpLinks does
    lib().or_fat7(_dims(dims), _coef(coefs), _p(gf), _p(fl), _p(gfl), _p(ll), naik)
    return fl, ll


def project_u(x: np.ndarray, eps: float = 1e-20) -> np.ndarray:
    """projectU (src/maths/matrixFunctions.nim:340-351) of (..., 3, 3)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().or_project_u(x.size // 9, _p(x), _p(out), eps)
    return out


def hisq_smear(dims, g: np.ndarray, lepage: float = 0.0, naik: float = 1.0, eps: float = 1e-20):
    """HisqCoefs.smear (src/physics/hisqLinks.nim:40-46): (fat, long)."""
    first, second, cn = hisq_coefs(lepage, naik)
    g = np.ascontiguousarray(g, dtype=np.complex128)
    fl, ll = np.empty_like(g), np.empty_like(g)
    lib().or_hisq_smear(_dims(dims), _coef(first), _coef(second), cn, eps, _p(g), _p(fl), _p(ll))
    return fl, ll



def fat7_deriv(dims, coefs, gauge, mid, llgauge=None, llmid=None, naik: float = 0.0):
    """fat7lDeriv (src/gauge/fat7lderiv.nim:122-331): derivative of
    sum Re Tr mid^dag fat7(gauge) (+ llmid^dag naik-product(llgauge)) with
    respect to gauge (and llgauge): (deriv, llderiv or None)."""
    gauge = np.ascontiguousarray(gauge, dtype=np.complex128)
    mid = np.ascontiguousarray(mid, dtype=np.complex128)
    d = np.zeros_like(gauge)
    if llgauge is None:
        lib().or_fat7_deriv(_dims(dims), _coef(coefs), _p(gauge), _p(mid), _p(d), None, None, None, 0.0)
        return d, None
    llgauge = np.ascontiguousarray(llgauge, dtype=np.complex128)
    llmid = np.ascontiguousarray(llmid, dtype=np.complex128)
    dl = np.zeros_like(gauge)
    lib().or_fat7_deriv(_dims(dims), _coef(coefs), _p(gauge), _p(mid), _p(d), _p(llgauge), _p(llmid), _p(dl),
                        naik)
    return d, dl


def project_u_deriv(u, x, chain, eps: float = 1e-20):
    """projectUderiv (src/maths/matrixFunctions.nim:368-390)."""
    u, x, chain = (np.ascontiguousarray(a, dtype=np.complex128) for a in (u, x, chain))
    r = np.empty_like(x)
    lib().or_project_u_deriv(x.size // 9, _p(u), _p(x), _p(chain), _p(r), eps)
    return r


def sylsolve(a, c):
    """x with a x + x a = c (src/maths/projUderiv.nim:96-145)."""
    a, c = (np.ascontiguousarray(v, dtype=np.complex128) for v in (a, c))
    x = np.empty_like(c)
    lib().or_sylsolve(c.size // 9, _p(a), _p(c), _p(x))
    return x


def hisq_deriv(dims, g, cfat, clong, lepage: float = 0.0, naik: float = 1.0, eps: float = 1e-20,
               coefs=None):
    """smearGetForce's chain rule (src/gauge/hisqsmear.nim:66-105): the
    derivative of sum Re Tr (cfat^dag fat(g) + clong^dag long(g)) w.r.t. g.
    coefs = (first, second, naik) overrides newHISQ(lepage, naik)."""
    first, second, cn = coefs if coefs is not None else hisq_coefs(lepage, naik)
    g, cfat, clong = (np.ascontiguousarray(a, dtype=np.complex128) for a in (g, cfat, clong))
    d = np.empty_like(g)
    lib().or_hisq_deriv(_dims(dims), _coef(first), _coef(second), cn, eps, _p(g), _p(cfat), _p(clong), _p(d))
    return d



# ---- gauge action, force and link update (hmc_oracle.c) -----------------

def gauge_action(dims, u, plaq: float, rect: float = 0.0) -> float:
    """gaugeAction1 (src/gauge/gaugeAction.nim:487-571) of (4, V, 3, 3) links."""
    u = np.ascontiguousarray(u, dtype=np.complex128)
    return lib().or_gauge_action(_dims(dims), plaq, rect, _p(u))


def gauge_force(dims, u, plaq: float, rect: float = 0.0):
    """gaugeForce (gaugeAction.nim:576-779): projectTAH(U f^dagger)."""
    u = np.ascontiguousarray(u, dtype=np.complex128)
    f = np.empty_like(u)
    lib().or_gauge_force(_dims(dims), plaq, rect, _p(u), _p(f))
    return f


def exp_ah(m, eps: float = 1.0):
    """expAH(eps m) (src/maths/matexp.nim:316-346) of (..., 3, 3)."""
    m = np.ascontiguousarray(m, dtype=np.complex128)
    out = np.empty_like(m)
    lib().or_exp_ah(m.size // 9, _p(m), eps, _p(out))
    return out


def link_update(u, p, eps: float):
    """axexpmuly(u, eps, p, u) (src/gauge/gaugeUtils.nim:452-459)."""
    u = np.ascontiguousarray(u, dtype=np.complex128).copy()
    p = np.ascontiguousarray(p, dtype=np.complex128)
    lib().or_link_update(u.size // 9, _p(u), _p(p), eps)
    return u


class CgRun:
    """One oracle CG solve (or_cg_begin / or_cg_run / or_cg_end), run a
    bounded number of iterations at a time.  Holds references to the
    operator, solution and source for its lifetime."""

    def __init__(self, o: Oracle, parity, x, b, m2, r2req):
        self.o, self.x, self.b = o, x, b
        self.state = lib().or_cg_begin(o.ctx, parity, _p(x), _p(b), m2, r2req)
        self.iterations = 0

    def run(self, n: int) -> int:
        """Up to n more iterations; returns the iterations done so far."""
        self.iterations = lib().or_cg_run(self.state, self.iterations + int(n))
        return self.iterations

    @property
    def converged(self) -> bool:
        return bool(lib().or_cg_converged(self.state))

    def end(self):
        """Frees the state; returns (iterations, |r|^2/|b|^2)."""
        r2 = C.c_double()
        its = lib().or_cg_end(self.state, C.byref(r2))
        self.state = None
        return its, r2.value

    def __del__(self):
        if getattr(self, "state", None):
            lib().or_cg_end(self.state, None)
            self.state = None
