"""GPU gauge-file I/O (qexstag_gauge_read / qexstag_gauge_write) against the
oracle's independent reader and writer: byte order, precision, site order
and checksums, both directions, host and device links.  Bit-exact: the data
are moved and converted, not computed."""
import numpy as np
import pytest

from oracle import io_oracle as IO
from qex_b200 import _lib as L
from qex_b200 import fields as F
from qex_b200 import gaugeio as G
from qex_b200 import stag as S

pytestmark = pytest.mark.gpu
SHAPES = [(4, 4, 4, 4), (6, 4, 8, 4), (8, 8, 8, 16)]


def f32(g):
    return g.astype(np.complex64).astype(np.complex128)


@pytest.mark.parametrize("dims", SHAPES)
def test_library_scidac_read_by_oracle(cuda, tmp_path, dims):
    g = F.gauge_warm(dims, 0.4, 5)
    lay = S.Layout(dims)
    for prec, ildg in (("D", False), ("F", False), ("D", True)):
        p = tmp_path / f"lib_{prec}_{ildg}.lime"
        G.saveGauge(lay, g, p, prec, "<note>file</note>", "<note>rec</note>", "ildg" if ildg else "scidac")
        d, g2, pb, stored, recs = IO.read_scidac(p)
        assert d == dims
        assert np.array_equal(g2, g if prec == "D" else f32(g))
        data = dict((t, x) for t, x, _, _ in recs)["ildg-binary-data" if ildg else "scidac-binary-data"]
        assert stored == IO.scidac_checksum(data, F.volume(dims))
        info = G.fileInfo(p)
        assert info.file_metadata == "<note>file</note>" and info.record_metadata == "<note>rec</note>"
        assert info.format == ("ildg" if ildg else "scidac") and info.precision == (8 if prec == "D" else 4)


@pytest.mark.parametrize("dims", SHAPES)
def test_oracle_files_read_by_library(cuda, tmp_path, dims):
    torch = cuda
    g = F.gauge_warm(dims, 0.4, 6)
    lay = S.Layout(dims)
    cases = [("scidac", "D"), ("scidac", "F"), ("ildg", "F"), ("milc", "<"), ("milc", ">")]
    for fmt, prec in cases:
        p = tmp_path / f"or_{fmt}_{prec}"
        if fmt == "milc":
            sums = IO.write_milc(p, dims, g, prec)
            want = f32(g)
        else:
            sums = IO.write_scidac(p, dims, g, prec, fmt == "ildg")
            want = g if prec == "D" else f32(g)
        h, info = G.read_gauge(lay, p)
        assert np.array_equal(h, want), (fmt, prec)
        assert info.has_checksum and info.file_checksum == sums == info.data_checksum
        assert info.dims == dims and info.format == fmt
        d, info2 = G.read_gauge(lay, p, device=True)
        assert np.array_equal(S.to_host_links(d), want)


def test_round_trip_device_links_and_milc(cuda, tmp_path):
    torch = cuda
    dims = (8, 8, 8, 8)
    lay = S.Layout(dims)
    g = F.gauge_warm(dims, 0.3, 7)
    gd = S.to_device_links(g)
    G.saveGauge(lay, gd, tmp_path / "a.lime", "D")
    back, _ = G.read_gauge(lay, tmp_path / "a.lime", device=True)
    assert torch.equal(back, gd)
    G.saveGauge(lay, gd, tmp_path / "a.milc", format="milc")
    d, g2, stored, recomputed = IO.read_milc(tmp_path / "a.milc")
    assert stored == recomputed and np.array_equal(g2, f32(g))
    assert G.getFileLattice(tmp_path / "a.milc") == list(dims)


def test_corrupt_and_mismatched_files(cuda, tmp_path):
    dims = (4, 4, 4, 4)
    lay = S.Layout(dims)
    g = F.gauge_warm(dims, 0.4, 8)
    p = tmp_path / "c.lime"
    IO.write_scidac(p, dims, g, "D")
    raw = bytearray(p.read_bytes())
    raw[-2000] ^= 0x10  # inside the binary data
    (tmp_path / "bad.lime").write_bytes(bytes(raw))
    h = np.empty_like(g)
    with pytest.raises(L.QexStagError) as e:
        G.loadGauge(lay, h, tmp_path / "bad.lime")
    assert e.value.code == L.ERR_IO and "checksum" in str(e.value)
    with pytest.raises(L.QexStagError) as e:
        G.loadGauge(S.Layout((4, 4, 4, 6)), np.empty((4, 384, 3, 3), complex), p)
    assert e.value.code == L.ERR_IO
    with pytest.raises(L.QexStagError) as e:
        G.loadGauge(lay, h, tmp_path / "missing.lime")
    assert e.value.code == L.ERR_IO
    (tmp_path / "junk").write_bytes(b"\1" * 200)
    with pytest.raises(L.QexStagError) as e:
        G.fileInfo(tmp_path / "junk")
    assert e.value.code == L.ERR_IO
