"""The C-ABI library loads and exports every symbol include/nectb.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "nectb.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|size_t|const char\*|const unsigned int\*)\s+(nectb_\w+)\(", text, re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "nectb_sample" in syms and "nectb_train_step" in syms


def test_library_exports_all_declared_symbols():
    from nect_b200 import _lib

    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"libnectb.so lacks {missing}"


def test_version_and_error_string():
    from nect_b200 import _lib

    assert b"sm_100a" in _lib.lib.nectb_version()
    assert _lib.lib.nectb_last_error() is not None
