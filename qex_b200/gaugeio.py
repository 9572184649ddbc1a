"""Gauge-field files through the C ABI: QEX's loadGauge / saveGauge
(src/gauge/gaugeUtils.nim:96-131) and getFileLattice
(src/io/readerQiolite.nim:11-17) for SciDAC and ILDG (LIME) files, and MILC
binary files (src/new/milcIO.nim).  Byte order, precision, site reordering
and checksums run on the GPU (qex_b200/csrc/gaugeio.cu).

Links are a 4-direction gauge field without staggered phases: host
(4, V, 3, 3) complex128 arrays or device (4, 3, 3, V) complex128 tensors.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .stag import Layout, _is_torch, _ptr

FORMATS = {"scidac": L.GAUGE_SCIDAC, "ildg": L.GAUGE_ILDG, "milc": L.GAUGE_MILC}
FORMAT_NAMES = {v: k for k, v in FORMATS.items()}


@dataclass
class GaugeFileInfo:
    format: str
    dims: tuple
    precision: int
    has_checksum: bool
    file_checksum: tuple
    data_checksum: tuple
    date: str
    file_metadata: str
    record_metadata: str


def _info(c: L.GaugeInfoC) -> GaugeFileInfo:
    return GaugeFileInfo(FORMAT_NAMES.get(c.format, "?"), tuple(c.dims), c.precision, bool(c.has_checksum),
                         tuple(c.file_checksum), tuple(c.data_checksum), c.date.decode(errors="replace"),
                         c.file_metadata.decode(errors="replace"), c.record_metadata.decode(errors="replace"))


def fileInfo(fn: str) -> GaugeFileInfo:
    c = L.GaugeInfoC()
    L.check(L.load().qexstag_gauge_file_info(str(fn).encode(), C.byref(c)), "gauge_file_info")
    return _info(c)


def getFileLattice(fn: str) -> list:
    """readerQiolite.nim:11-17."""
    return list(fileInfo(fn).dims)


def _check(layout: Layout, g) -> None:
    want = (4, 3, 3, layout.V) if _is_torch(g) else (4, layout.V, 3, 3)
    if tuple(g.shape) != want:
        raise ValueError(f"gauge field must have shape {want}, got {tuple(g.shape)}")


def loadGauge(layout: Layout, g, fn: str) -> GaugeFileInfo:
    """Read fn into g (gaugeUtils.nim:96-117); raises on a checksum mismatch."""
    _check(layout, g)
    ptr, mem = _ptr(g, True)
    c = L.GaugeInfoC()
    L.check(L.load().qexstag_gauge_read(layout.handle, str(fn).encode(), ptr, mem, C.byref(c)), "gauge_read")
    return _info(c)


def saveGauge(layout: Layout, g, fn: str, prec: str = "", filemd: str = "", recordmd: str = "",
              format: str = "scidac") -> None:
    """Write g to fn (gaugeUtils.nim:120-131): prec "F" (single), "D"
    (double) or "" (double, the precision the links are held in); format
    "scidac", "ildg" or "milc" (single precision only)."""
    _check(layout, g)
    if format == "milc" and prec == "":
        prec = "F"
    bytes_per = {"": 8, "D": 8, "F": 4}[prec]
    ptr, mem = _ptr(g)
    L.check(L.load().qexstag_gauge_write(layout.handle, str(fn).encode(), ptr, mem, FORMATS[format], bytes_per,
                                         filemd.encode(), recordmd.encode()), "gauge_write")


def read_gauge(layout: Layout, fn: str, device: bool = False):
    """Convenience: (links, info) for a new field."""
    if device:
        import torch
        g = torch.empty((4, 3, 3, layout.V), dtype=torch.complex128, device="cuda")
    else:
        g = np.empty((4, layout.V, 3, 3), dtype=np.complex128)
    return g, loadGauge(layout, g, fn)
