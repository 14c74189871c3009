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


def test_binding_constants_match_header():
    text = (ROOT / "include" / "prism_b200.h").read_text()
    defines = {k: int(v, 0) for k, v in
               re.findall(r"#define\s+(PS_[A-Z0-9_]+)\s+\(?(-?(?:0x[0-9a-fA-F]+|\d+))u?\)?", text)}
    assert len(defines) > 20
    missing = [k for k in defines if not hasattr(_lib, k)]
    assert not missing, missing
    assert {k: getattr(_lib, k) for k in defines} == defines


def test_binding_loads_and_reports_version():
    lib = _lib.load()
    assert lib.ps_version().startswith(b"prismplan_b200")
    assert lib.ps_edges_workspace_bytes(65536) >= 65536 * 16


def test_edges_workspace_layout():
    """The persistent edge workspace: a 64-B header (in its own 256-B block)
    and six 4-B per-edge arrays (G, length, retire flag, clearance, completed
    chunks, the long list), each starting on a 256-B boundary."""
    lib = _lib.load()
    up = lambda x: (x + 255) // 256 * 256
    for n in (1, 7, 1000, 65536):
        assert lib.ps_edges_workspace_bytes(n) == up(64) + 6 * up(4 * n)
    assert lib.ps_edges_workspace_bytes(0) == lib.ps_edges_workspace_bytes(1)


STRUCTS = {   # ctypes mirror -> C struct of include/prism_b200.h
    "ModelDesc": "ps_model_desc", "ModelInfo": "ps_model_info", "SceneView": "ps_scene_view",
    "EdgeParams": "ps_edge_params", "CostParams": "ps_cost_params", "BatchLimits": "ps_batch_limits",
    "BatchTuning": "ps_batch_tuning", "ChompParams": "ps_chomp_params", "StompParams": "ps_stomp_params",
    "StompLayout": "ps_stomp_layout", "EdgeTuning": "ps_edge_tuning", "ConfigTuning": "ps_config_tuning",
}


def test_struct_layouts_match_header(tmp_path):
    """Compile a C program against the header that prints sizeof and every
    field offset, and compare them with the ctypes mirrors."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        import pytest

        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "prism_b200.h"', "int main(void) {"]
    for py, c in STRUCTS.items():
        lines.append(f'printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(_lib, py)._fields_:
            lines.append(f'printf("{py}.{name} %zu\\n", offsetof({c}, {name}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                              text=True).stdout.splitlines())
    for py in STRUCTS:
        cls = getattr(_lib, py)
        assert int(got[f"{py} size"]) == ctypes.sizeof(cls), py
        for name, _ in cls._fields_:
            assert int(got[f"{py}.{name}"]) == getattr(cls, name).offset, f"{py}.{name}"
