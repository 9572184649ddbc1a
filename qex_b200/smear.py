"""HISQ link smearing through the C ABI: QEX's Fat7lCoefs / HisqCoefs
(src/gauge/fat7l.nim:5-10, src/physics/hisqLinks.nim:3-46,
src/gauge/hisqsmear.nim:53-64) with makeImpLinks, projectU and smear run by
the library's kernels (qex_b200/csrc/smear.cu).

Gauge fields are four directions: host (4, V, 3, 3) complex128 arrays or
device (4, 3, 3, V) complex128 tensors, as for ``Staggered``'s link lists.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .stag import Layout, SolverParams, Staggered, _is_torch, _mem_of, _ptr


@dataclass
class Fat7lCoefs:
    oneLink: float = 0.0
    threeStaple: float = 0.0
    fiveStaple: float = 0.0
    sevenStaple: float = 0.0
    lepage: float = 0.0

    def setHisqFat7(self, f7lf: float, naik: float) -> "Fat7lCoefs":
        """hisqLinks.nim:10-15."""
        c = L.Fat7CoefsC()
        L.load().qexstag_fat7_coefs_set_hisq(C.byref(c), float(f7lf), float(naik))
        self.oneLink, self.threeStaple = c.one_link, c.three_staple
        self.fiveStaple, self.sevenStaple, self.lepage = c.five_staple, c.seven_staple, c.lepage
        return self

    def c(self) -> L.Fat7CoefsC:
        return L.Fat7CoefsC(self.oneLink, self.threeStaple, self.fiveStaple, self.sevenStaple, self.lepage)

    def as_list(self):
        return [self.oneLink, self.threeStaple, self.fiveStaple, self.sevenStaple, self.lepage]


@dataclass
class HisqCoefs:
    fat7first: Fat7lCoefs = field(default_factory=Fat7lCoefs)
    fat7second: Fat7lCoefs = field(default_factory=Fat7lCoefs)
    naik: float = 0.0
    reunit_eps: float = 1e-20

    def c(self) -> L.HisqCoefsC:
        return L.HisqCoefsC(self.fat7first.c(), self.fat7second.c(), self.naik, self.reunit_eps)


def newHISQ(lepage: float = 0.0, naik: float = 1.0) -> HisqCoefs:
    """hisqsmear.nim:53-64 (coefficients filled in by the library)."""
    c = L.HisqCoefsC()
    L.load().qexstag_hisq_coefs_init(C.byref(c), float(lepage), float(naik))
    def f7(x):
        return Fat7lCoefs(x.one_link, x.three_staple, x.five_staple, x.seven_staple, x.lepage)
    return HisqCoefs(f7(c.fat7first), f7(c.fat7second), c.naik, c.reunit_eps)


def _check_gauge(layout: Layout, g) -> None:
    shape = tuple(g.shape)
    want = (4, 3, 3, layout.V) if _is_torch(g) else (4, layout.V, 3, 3)
    if shape != want:
        raise ValueError(f"gauge field must have shape {want}, got {shape}")


class Smear:
    """Smearing handle: the device scratch of the staple sweeps on one layout."""

    def __init__(self, layout: Layout):
        self.l = layout
        self._lib = layout._lib
        h = C.c_void_p()
        L.check(self._lib.qexstag_smear_create(layout.handle, C.byref(h)), "smear_create")
        self.handle = h

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                self._lib.qexstag_smear_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    def makeImpLinks(self, fl, gf, coef: Fat7lCoefs, ll=None, gfLong=None, naik: float = 0.0) -> None:
        """fat7l.nim:70-154: fl = fat7(gf); with ll, gfLong and naik != 0 also
        ll = naik gfLong(x) gfLong(x+mu) gfLong(x+2mu)."""
        for f in (fl, gf) + ((ll, gfLong) if ll is not None else ()):
            _check_gauge(self.l, f)
        fields = (fl, gf) + ((ll, gfLong) if ll is not None else ())
        mem = _mem_of(*fields)
        pll = _ptr(ll, True)[0] if ll is not None else None
        pgl = _ptr(gfLong)[0] if gfLong is not None else None
        cc = coef.c()
        L.check(self._lib.qexstag_fat7(self.handle, C.byref(cc), _ptr(gf)[0], _ptr(fl, True)[0], pgl, pll,
                                       float(naik), mem), "fat7")

    def projectU(self, u, x, eps: float = 1e-20) -> None:
        """u = x (x^dag x + eps)^(-1/2) per link (matrixFunctions.nim:340-351)."""
        _check_gauge(self.l, x)
        _check_gauge(self.l, u)
        mem = _mem_of(u, x)
        L.check(self._lib.qexstag_project_u(self.handle, _ptr(x)[0], _ptr(u, True)[0], float(eps), mem),
                "project_u")

    def smear(self, coef: HisqCoefs, g, fl, ll) -> None:
        """HisqCoefs.smear (hisqLinks.nim:40-46)."""
        for f in (g, fl, ll):
            _check_gauge(self.l, f)
        mem = _mem_of(g, fl, ll)
        cc = coef.c()
        L.check(self._lib.qexstag_hisq_smear(self.handle, C.byref(cc), _ptr(g)[0], _ptr(fl, True)[0],
                                             _ptr(ll, True)[0], mem), "hisq_smear")

    def fat7Deriv(self, deriv, gauge, mid, coef: Fat7lCoefs, llderiv=None, llgauge=None, llmid=None,
                  naik: float = 0.0) -> None:
        """fat7lDeriv (fat7lderiv.nim:122-331): adds to deriv (and llderiv) the
        derivative of sum Re Tr (mid^dag fat7(gauge) + llmid^dag naik-product(llgauge))."""
        fields = [deriv, gauge, mid] + ([llderiv, llgauge, llmid] if llderiv is not None else [])
        for f in fields:
            _check_gauge(self.l, f)
        mem = _mem_of(*fields)
        cc = coef.c()
        ld = _ptr(llderiv, True)[0] if llderiv is not None else None
        lg = _ptr(llgauge)[0] if llgauge is not None else None
        lm = _ptr(llmid)[0] if llmid is not None else None
        L.check(self._lib.qexstag_fat7_deriv(self.handle, C.byref(cc), _ptr(gauge)[0], _ptr(mid)[0],
                                             _ptr(deriv, True)[0], lg, lm, ld, float(naik), mem), "fat7_deriv")

    def projectUderiv(self, r, u, x, chain, eps: float = 1e-20) -> None:
        """projectUderiv (matrixFunctions.nim:368-390) per link."""
        for f in (r, u, x, chain):
            _check_gauge(self.l, f)
        mem = _mem_of(r, u, x, chain)
        L.check(self._lib.qexstag_project_u_deriv(self.handle, _ptr(u)[0], _ptr(x)[0], _ptr(chain)[0],
                                                  _ptr(r, True)[0], float(eps), mem), "project_u_deriv")

    def smearDeriv(self, coef: HisqCoefs, g, cfat, clong, deriv) -> None:
        """smearGetForce's chain rule (hisqsmear.nim:66-105): deriv = d/dg of
        sum Re Tr (cfat^dag fat(g) + clong^dag long(g))."""
        for f in (g, cfat, clong, deriv):
            _check_gauge(self.l, f)
        mem = _mem_of(g, cfat, clong, deriv)
        cc = coef.c()
        L.check(self._lib.qexstag_hisq_deriv(self.handle, C.byref(cc), _ptr(g)[0], _ptr(cfat)[0], _ptr(clong)[0],
                                             _ptr(deriv, True)[0], mem), "hisq_deriv")

    def force(self, stag: Staggered, coef: HisqCoefs, thin, f, phi, m: float, sp: SolverParams) -> None:
        """QEX's force with HISQ smearing (hmcAction.nim:851-885): f =
        projectTAH(ff U^dag) on the thin links, ff the chain rule of the
        fermion force's outer products; stag's links become the smeared ones."""
        _check_gauge(self.l, thin)
        _check_gauge(self.l, f)
        mem = _mem_of(thin, f, phi)
        st = L.SolverStatsC()
        pc = sp.c_params()
        cc = coef.c()
        rc = self._lib.qexstag_hisq_force(stag.handle, self.handle, C.byref(cc), _ptr(thin)[0], _ptr(f, True)[0],
                                          _ptr(phi)[0], float(m), C.byref(pc), C.byref(st), mem)
        L.check(rc, "hisq_force")
        sp.take(st, rc)

    def smear_into(self, stag: Staggered, coef: HisqCoefs, g) -> None:
        """Smear thin links g into a fat+Naik operator's link list and rebuild
        its reduced-precision copies."""
        _check_gauge(self.l, g)
        cc = coef.c()
        ptr, mem = _ptr(g)
        L.check(self._lib.qexstag_links_hisq(stag.handle, self.handle, C.byref(cc), ptr, mem), "links_hisq")


def hisq_smear(layout: Layout, g, coef: HisqCoefs | None = None):
    """Convenience: (fat, long) HISQ links of g in g's memory space."""
    coef = coef or newHISQ()
    if _is_torch(g):
        import torch
        fl, ll = torch.empty_like(g), torch.empty_like(g)
    else:
        fl, ll = np.empty_like(g), np.empty_like(g)
    Smear(layout).smear(coef, g, fl, ll)
    return fl, ll
