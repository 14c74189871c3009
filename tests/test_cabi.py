"""CPU: the C-ABI library loads and exports every entry point the header
declares; the Python binding covers all of them. No compute calls."""
import ctypes
import re
from pathlib import Path

from prismplan_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (ROOT / "include" / "prism_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ps_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in header_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header():
    assert sorted(header_symbols()) == sorted(_lib.EXPORTED_SYMBOLS)


def test_binding_loads_and_reports_version():
    lib = _lib.load()
    assert lib.ps_version().startswith(b"prismplan_b200")
    assert lib.ps_edges_workspace_bytes(65536) >= 65536 * 16


def test_struct_sizes_match_header_layout():
    # ps_model_desc: 4 ints + 18 pointers laid out with natural alignment
    assert ctypes.sizeof(_lib.EdgeParams) == 28
    assert ctypes.sizeof(_lib.CostParams) == 28
