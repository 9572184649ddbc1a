"""Gauge-file formats restated in numpy: the checker for the library's
qexstag_gauge_read / qexstag_gauge_write.

TEST INFRASTRUCTURE ONLY (tests/ may import it; the product path never does).

Formats, as QEX reads and writes them (src/gauge/gaugeUtils.nim:96-131 over
src/io/readerQiolite.nim / writerQiolite.nim and the third-party qiolite
package, unpinned; MILC as src/new/milcIO.nim):
  - LIME record: 144-byte big-endian header (magic 0x456789ab, version 1,
    message-begin / message-end flags, 64-bit data length, 128-byte type)
    then the data padded to 8 bytes;
  - SciDAC single file: private file XML with <dims>, user file XML, then a
    message of private record XML (precision F/D, typesize, datacount 4),
    user record XML, scidac-binary-data (big-endian, sites in lexicographic
    order x0 fastest, per site 4 row-major 3x3 complex matrices) and
    scidac-checksum (<suma>, <sumb> in hex); ILDG adds ildg-format and names
    the data ildg-binary-data;
  - MILC version 5: 96-byte native-order header (magic 20103, dims, 64-char
    stamp, order 0, sum29, sum31) then F32 data in the same site order.
Checksums come from io_oracle.c (CRC-32 of crc32.nim, the MILC word sums of
milcIO.nim) and, independently, Python's zlib.crc32.
"""
from __future__ import annotations

import ctypes as C
import struct
import zlib

import numpy as np

from . import oracle as O

LIME_MAGIC = 0x456789AB
MILC_MAGIC = 20103


def crc32(b: bytes) -> int:
    return O.lib().or_crc32(C.c_char_p(b), len(b))


def scidac_checksum(data: bytes, nsites: int):
    a, b = C.c_uint32(), C.c_uint32()
    O.lib().or_scidac_checksum(C.c_char_p(data), nsites, len(data) // nsites, C.byref(a), C.byref(b))
    return a.value, b.value


def scidac_checksum_zlib(data: bytes, nsites: int):
    """The same sums with zlib's CRC-32 (an implementation of its own)."""
    size = len(data) // nsites
    a = b = 0
    for r in range(nsites):
        c = zlib.crc32(data[r * size:(r + 1) * size]) & 0xFFFFFFFF
        ka, kb = r % 29, r % 31
        a ^= ((c << ka) | (c >> (32 - ka))) & 0xFFFFFFFF if ka else c
        b ^= ((c << kb) | (c >> (32 - kb))) & 0xFFFFFFFF if kb else c
    return a, b


def milc_checksum(words: np.ndarray):
    w = np.ascontiguousarray(words, dtype=np.uint32)
    a, b = C.c_uint32(), C.c_uint32()
    O.lib().or_milc_checksum(C.c_void_p(w.ctypes.data), w.size, C.byref(a), C.byref(b))
    return a.value, b.value


def lex_order(dims) -> np.ndarray:
    """QEX site index of each lexicographic site (qlayout.nim:108-136)."""
    from qex_b200 import fields as F
    V = int(np.prod(dims))
    lex = np.arange(V)
    x = np.stack([lex % dims[0], lex // dims[0] % dims[1], lex // (dims[0] * dims[1]) % dims[2],
                  lex // (dims[0] * dims[1] * dims[2])], axis=1)
    return F.index_of(dims, x)


def to_file_order(dims, links: np.ndarray) -> np.ndarray:
    """(4, V, 3, 3) in QEX index order -> (V, 4, 3, 3) in lexicographic order."""
    return np.ascontiguousarray(np.moveaxis(links, 0, 1)[lex_order(dims)])


def from_file_order(dims, data: np.ndarray) -> np.ndarray:
    out = np.empty((4,) + data.shape[:1] + (3, 3), dtype=np.complex128)
    out[:, lex_order(dims)] = np.moveaxis(data, 1, 0)
    return out


def lime_records(buf: bytes):
    """[(type, data bytes, mb, me)] of a LIME file."""
    recs, pos = [], 0
    while pos + 144 <= len(buf):
        magic, version, flags, length = struct.unpack(">IHHQ", buf[pos:pos + 16])
        assert magic == LIME_MAGIC and version == 1
        typ = buf[pos + 16:pos + 144].split(b"\0")[0].decode()
        data = buf[pos + 144:pos + 144 + length]
        recs.append((typ, data, bool(flags & 0x8000), bool(flags & 0x4000)))
        pos += 144 + (length + 7) // 8 * 8
    return recs


def lime_record(typ: str, data: bytes, mb: bool, me: bool) -> bytes:
    h = struct.pack(">IHHQ", LIME_MAGIC, 1, (0x8000 if mb else 0) | (0x4000 if me else 0), len(data))
    h += typ.encode().ljust(128, b"\0")
    return h + data + b"\0" * ((8 - len(data) % 8) % 8)


def _tag(x: str, t: str) -> str:
    a, b = x.find(f"<{t}>"), x.find(f"</{t}>")
    return x[a + len(t) + 2:b] if a >= 0 and b > a else ""


def write_scidac(path, dims, links, prec="D", ildg=False, filemd="", recordmd=""):
    V = int(np.prod(dims))
    dt = ">f8" if prec == "D" else ">f4"
    data = to_file_order(dims, links).view(np.float64).astype(dt).tobytes()
    a, b = scidac_checksum(data, V)
    size = 4 * 18 * (8 if prec == "D" else 4)
    pf = ("<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacFile><version>1.1</version><spacetime>4</spacetime>"
          f"<dims>{' '.join(str(d) for d in dims)} </dims><volfmt>0</volfmt></scidacFile>")
    pr = ("<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacRecord><version>1.1</version><date>today</date>"
          f"<recordtype>0</recordtype><datatype>QDP_{prec}3_ColorMatrix</datatype><precision>{prec}</precision>"
          f"<colors>3</colors><spins>4</spins><typesize>{size // 4}</typesize><datacount>4</datacount>"
          "</scidacRecord>")
    ck = ("<?xml version=\"1.0\" encoding=\"UTF-8\"?><scidacChecksum><version>1.0</version>"
          f"<suma>{a:x}</suma><sumb>{b:x}</sumb></scidacChecksum>")
    out = lime_record("scidac-private-file-xml", pf.encode(), True, False)
    out += lime_record("scidac-file-xml", filemd.encode(), False, True)
    out += lime_record("scidac-private-record-xml", pr.encode(), True, False)
    out += lime_record("scidac-record-xml", recordmd.encode(), False, False)
    if ildg:
        fx = ("<?xml version=\"1.0\" encoding=\"UTF-8\"?><ildgFormat><version>1.0</version><field>su3gauge</field>"
              f"<precision>{64 if prec == 'D' else 32}</precision><lx>{dims[0]}</lx><ly>{dims[1]}</ly>"
              f"<lz>{dims[2]}</lz><lt>{dims[3]}</lt></ildgFormat>")
        out += lime_record("ildg-format", fx.encode(), False, False)
    out += lime_record("ildg-binary-data" if ildg else "scidac-binary-data", data, False, False)
    out += lime_record("scidac-checksum", ck.encode(), False, True)
    with open(path, "wb") as f:
        f.write(out)
    return a, b


def read_scidac(path):
    """(dims, links (4, V, 3, 3), precision bytes, (suma, sumb) stored, records)."""
    with open(path, "rb") as f:
        buf = f.read()
    recs = lime_records(buf)
    by = {t: d for t, d, _, _ in recs}
    dims = tuple(int(v) for v in _tag(by["scidac-private-file-xml"].decode(), "dims").split())
    prec = 8 if _tag(by["scidac-private-record-xml"].decode(), "precision") == "D" else 4
    data = by.get("scidac-binary-data", by.get("ildg-binary-data"))
    V = int(np.prod(dims))
    vals = np.frombuffer(data, dtype=">f8" if prec == 8 else ">f4").astype(np.float64)
    links = from_file_order(dims, vals.view(np.complex128).reshape(V, 4, 3, 3))
    ck = by["scidac-checksum"].decode()
    return dims, links, prec, (int(_tag(ck, "suma"), 16), int(_tag(ck, "sumb"), 16)), recs


def write_milc(path, dims, links, byteorder="<"):
    V = int(np.prod(dims))
    data = to_file_order(dims, links).view(np.float64).astype(byteorder + "f4")
    a, b = milc_checksum(data.astype(np.float32).view(np.uint32))
    hdr = struct.pack(byteorder + "i4i64siII", MILC_MAGIC, *dims, b"oracle".ljust(64, b"\0"), 0, a, b)
    with open(path, "wb") as f:
        f.write(hdr + data.tobytes())
    return a, b


def read_milc(path):
    with open(path, "rb") as f:
        buf = f.read()
    bo = "<" if struct.unpack("<i", buf[:4])[0] == MILC_MAGIC else ">"
    magic, d0, d1, d2, d3, _stamp, order, a, b = struct.unpack(bo + "i4i64siII", buf[:96])
    dims = (d0, d1, d2, d3)
    V = int(np.prod(dims))
    vals = np.frombuffer(buf[96:], dtype=bo + "f4")
    links = from_file_order(dims, vals.astype(np.float64).view(np.complex128).reshape(V, 4, 3, 3))
    return dims, links, (a, b), milc_checksum(vals.astype(np.float32).view(np.uint32))
