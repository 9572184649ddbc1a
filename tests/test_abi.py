"""CPU checks of the C ABI: the shared library loads and exports every
function include/qexstag.h declares, and the ctypes signatures cover them."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "qexstag.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qexstag_[A-Za-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ["qexstag_init", "qexstag_stagD2", "qexstag_stagD2ee", "qexstag_solveEE",
                 "qexstag_solve", "qexstag_solve_multishift", "qexstag_cgm_ee", "qexstag_force"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from qex_b200 import _lib
    from qex_b200.build import build
    build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_header():
    from qex_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    from qex_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "nope.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()


def test_last_error_without_gpu():
    """Calls that need a device fail with a status, not a crash, when no GPU
    is visible (this container); with a GPU this just initialises."""
    from qex_b200 import _lib
    lib = _lib.load()
    rc = lib.qexstag_init(0)
    if rc != 0:
        assert rc < 0
        assert lib.qexstag_last_error()
