"""CPU-side checks of the C ABI: the library loads, exports every function
include/*.h declares, and the parameters.txt reader follows the reference's
rules. No compute call is made (there may be no GPU)."""
import re
from pathlib import Path

import pytest

from conftest import REPO

HEADERS = sorted((REPO / "include").glob("*.h"))
DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b((?:dwf|wil)_\w+)\s*\(", re.M)


def declared_functions():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in DECL.finditer(text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_functions()
    assert "dwf_ctx_create" in names and "dwf_cg" in names
    assert len(names) >= 10


def test_library_exports_every_declared_symbol():
    import ctypes
    from three_part_dwf_study_b200 import _capi

    if not _capi.LIB_PATH.exists():
        from three_part_dwf_study_b200 import build
        build.build()
    lib = ctypes.CDLL(str(_capi.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the binding's signature table covers the header too
    assert set(declared_functions()) <= set(_capi.SIGNATURES)


def test_status_strings_without_gpu():
    from three_part_dwf_study_b200 import _capi
    assert _capi.status_string(2) == "CG encountered a zero denominator"
    assert _capi.status_string(0) == "ok"


def test_parameters_reader_semantics(tmp_path):
    from three_part_dwf_study_b200.params import ConfigError, TextConfig, dwf_parameters

    ref_params = REPO / "tests" / "golden" / "dwf_8x8x4" / "parameters.txt"
    cfg = TextConfig(ref_params)
    p = dwf_parameters(cfg)
    assert p["Nt"] == 8 and p["N5"] == 4 and p["Ndof"] == 4 * 8 * 8 * 2
    bad = tmp_path / "p.txt"
    bad.write_text("dwf.Nt = 8\nnot a pair\n")
    with pytest.raises(ConfigError, match=r"p.txt:2: expected key = value"):
        TextConfig(bad)
    bad.write_text("dwf.Nt =   # comment\n")
    with pytest.raises(ConfigError, match="empty key or value"):
        TextConfig(bad)
    bad.write_text("dwf.Nt = 8x\n")
    with pytest.raises(ConfigError, match="Invalid numeric value for dwf.Nt: 8x"):
        TextConfig(bad).integer("dwf.Nt")
    with pytest.raises(ConfigError, match="Missing required parameter: dwf.Nx"):
        TextConfig(bad).integer("dwf.Nx")
    ok = TextConfig(text="a = 1.5e-3 # x\nb = -2\n")
    assert ok.real("a") == 1.5e-3 and ok.integer("b") == -2
    assert ok.unsigned_integer("b") == (1 << 64) - 2
