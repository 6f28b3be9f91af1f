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


def test_host_random_streams_match_reference_draws():
    """The product's host RNG reproduces the reference's streams (pinned by the
    known answers and by the oracle, which the reference's own HMC runs pin)."""
    import numpy as np
    from oracle import oracle as O
    from three_part_dwf_study_b200.rng import Rng, z4_digits

    assert Rng(1234).normals(2).tolist() == [0.20515413959099182, -0.33619173225969745]
    assert z4_digits(918273, 8).tolist() == [1, 0, 2, 1, 1, 3, 1, 0]
    ndof, ng = 64, 32
    chi, mom, u = O.dwf_draws(77, 2, ndof, ng)
    r = Rng(77)
    for k in range(2):   # domain wall order: chi, mom, u
        assert np.array_equal(r.pseudofermion(ndof), chi[k])
        assert np.array_equal(r.normals(ng), mom[k])
        assert r.uniform() == u[k]
    mom, chi, u = O.wil_draws(78, 2, ndof, ng)
    r = Rng(78)
    for k in range(2):   # Wilson order: mom, chi, u
        assert np.array_equal(r.normals(ng), mom[k])
        assert np.array_equal(r.pseudofermion(ndof), chi[k])
        assert r.uniform() == u[k]
    assert np.array_equal(z4_digits(5, 1000), O.rng_z4(5, 1000))


def _rr_worker(path, q):
    import ctypes as C
    from three_part_dwf_study_b200 import _capi as A
    dev = C.c_int(-1)
    st = A.lib().dwf_round_robin_device(4, str(path).encode(), C.byref(dev))
    q.put((st, dev.value))


def test_round_robin_device_hands_out_each_gpu_in_turn(tmp_path):
    """DWF_B200_DEVICE=auto: concurrent processes (here 8, for 4 GPUs) take the
    counter under a lock, so every device index is handed out exactly twice."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    path = tmp_path / "counter"
    procs = [ctx.Process(target=_rr_worker, args=(path, q)) for _ in range(8)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    assert all(st == 0 for st, _ in got)
    assert sorted(d for _, d in got) == [0, 0, 1, 1, 2, 2, 3, 3]
    assert path.read_text().strip() == "8"
