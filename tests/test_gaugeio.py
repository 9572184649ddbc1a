"""CPU tests that pin the gauge-file oracle (oracle/io_oracle.c, io_oracle.py).

QEX's crc32.nim carries a known answer, which pins the CRC-32; zlib's
CRC-32 gives an independent second implementation of the SciDAC site sums;
the formats are pinned by write/read round trips of the oracle's own writer
and reader (no SciDAC or MILC file from QEX is available)."""
import zlib

import numpy as np
import pytest

from oracle import io_oracle as IO
from qex_b200 import fields as F


def test_crc32_known_answer():
    """src/io/crc32.nim:103-106."""
    s = b"The quick brown fox jumps over the lazy dog"
    assert IO.crc32(s) == 0x414FA339
    assert zlib.crc32(s) == 0x414FA339


def test_scidac_sums_agree_with_zlib():
    rng = np.random.default_rng(1)
    data = rng.integers(0, 256, size=97 * 576, dtype=np.uint8).tobytes()
    assert IO.scidac_checksum(data, 97) == IO.scidac_checksum_zlib(data, 97)


def test_milc_sums_rotate():
    w = np.arange(1, 200, dtype=np.uint32) * np.uint32(2654435761)
    a, b = IO.milc_checksum(w)
    ea = eb = 0
    for k, x in enumerate(w.tolist()):
        ka, kb = k % 29, k % 31
        ea ^= ((x << ka) | (x >> (32 - ka))) & 0xFFFFFFFF if ka else x
        eb ^= ((x << kb) | (x >> (32 - kb))) & 0xFFFFFFFF if kb else x
    assert (a, b) == (ea, eb)


@pytest.mark.parametrize("prec", ["D", "F"])
@pytest.mark.parametrize("ildg", [False, True])
def test_scidac_round_trip(tmp_path, prec, ildg):
    dims = (4, 4, 6, 8)
    g = F.gauge_warm(dims, 0.4, 2)
    p = tmp_path / "g.lime"
    sums = IO.write_scidac(p, dims, g, prec, ildg, "file md", "record md")
    d, g2, pb, stored, recs = IO.read_scidac(p)
    assert d == dims and pb == (8 if prec == "D" else 4) and stored == sums
    want = g if prec == "D" else g.astype(np.complex64).astype(np.complex128)
    assert np.array_equal(g2, want)
    types = [r[0] for r in recs]
    assert types[:4] == ["scidac-private-file-xml", "scidac-file-xml", "scidac-private-record-xml",
                         "scidac-record-xml"]
    assert types[-1] == "scidac-checksum" and recs[0][2] and recs[1][3] and recs[-1][3]


@pytest.mark.parametrize("bo", ["<", ">"])
def test_milc_round_trip(tmp_path, bo):
    dims = (4, 4, 4, 6)
    g = F.gauge_warm(dims, 0.4, 3)
    p = tmp_path / "g.milc"
    sums = IO.write_milc(p, dims, g, bo)
    d, g2, stored, recomputed = IO.read_milc(p)
    assert d == dims and stored == sums == recomputed
    assert np.array_equal(g2, g.astype(np.complex64).astype(np.complex128))
