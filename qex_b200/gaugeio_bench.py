"""Gauge-file I/O on one GPU: write and read a 32^4 field.

  python -m qex_b200.gaugeio_bench [--dims 32,32,32,32] [--dir /tmp]

Times qexstag_gauge_write / qexstag_gauge_read (device links) in SciDAC F64,
SciDAC F32 and MILC, wall clock around the call (file system included), and
reports the file size.  The pack / unpack kernels' own device times come
from the ncu launch list of the same command.
"""
from __future__ import annotations

import argparse
import json
import os
import time

from . import fields as F
from . import gaugeio as G
from . import stag as S


def run(dims, d):
    import torch
    S.init(0)
    lay = S.Layout(dims)
    g = S.to_device_links(F.gauge_warm(dims, 0.3, 3))
    out = {"dims": dims, "V": lay.V, "cases": {}}
    for fmt, prec in (("scidac", "D"), ("scidac", "F"), ("milc", "F")):
        p = os.path.join(d, f"bench_{fmt}_{prec}")
        G.saveGauge(lay, g, p, prec, format=fmt)  # warm-up (allocations, tables)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        G.saveGauge(lay, g, p, prec, format=fmt)
        tw = time.perf_counter() - t0
        h = torch.empty_like(g)
        G.loadGauge(lay, h, p)
        t0 = time.perf_counter()
        info = G.loadGauge(lay, h, p)
        tr = time.perf_counter() - t0
        size = os.path.getsize(p)
        out["cases"][f"{fmt}_{prec}"] = {"bytes": size, "write_s": tw, "read_s": tr,
                                         "write_GBps": size / tw * 1e-9, "read_GBps": size / tr * 1e-9,
                                         "checksum": list(info.data_checksum)}
        os.remove(p)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", default="32,32,32,32")
    ap.add_argument("--dir", default="/tmp")
    a = ap.parse_args()
    print(json.dumps(run(tuple(int(v) for v in a.dims.split(",")), a.dir)))


if __name__ == "__main__":
    main()
