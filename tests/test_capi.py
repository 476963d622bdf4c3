"""The C-ABI library loads and exports every declared entry point (CPU only, no device work)."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO

HEADERS = [os.path.join(REPO, "include", h) for h in sorted(os.listdir(os.path.join(REPO, "include")))]


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(issl_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_headers_declare_entry_points():
    names = declared_symbols()
    for n in ["issl_open", "issl_open_arrays", "issl_build", "issl_close", "issl_score", "issl_score_sigs",
              "issl_score_device", "issl_export", "issl_save", "issl_last_error", "issl_synth", "issl_tables",
              "issl_module_run"]:
        assert n in names


def test_library_exports_every_declared_symbol(native):
    path = native.library_path()
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = declared_symbols() - exported
    assert not missing, missing
    lib = C.CDLL(path)
    for n in declared_symbols():
        assert getattr(lib, n) is not None


def test_bindings_cover_declarations(native):
    from cracklingplusplus_gpu_b200._lib import SIGNATURES
    bound = {n for n, _, _ in SIGNATURES}
    assert declared_symbols() <= bound


def test_tables_equal_reference(native, penalties):
    masks, scores, pos, pam = native.tables()
    np.testing.assert_array_equal(masks, penalties["mit_masks"])
    np.testing.assert_array_equal(scores, penalties["mit_vals"])  # formula, bit-exact
    np.testing.assert_array_equal(pos, penalties["cfd_pos"])
    np.testing.assert_array_equal(pam, penalties["cfd_pam"])


def test_open_missing_file_reports_io_error(native):
    with pytest.raises(native.IsslError) as e:
        native.Index.open("/nonexistent/index.issl")
    assert e.value.code == -2
    assert "could not open" in str(e.value)


def test_null_arguments_rejected(native):
    lib = native.lib()
    assert lib.issl_score(None, None, 0, 0, 2, 75.0, 4, None, None, None, None, None) == -1
    assert lib.issl_close(None) == 0
    assert b"null" in lib.issl_last_error() or lib.issl_last_error() is not None


def test_python_module_rejects_bad_method(native):
    with pytest.raises(RuntimeError, match="not valid"):
        native.ISSLScoringModule(native.CracklingConfig("x.issl", method="bogus"))


def test_no_fallback_when_library_missing(tmp_path, monkeypatch):
    import cracklingplusplus_gpu_b200._lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "library_path", lambda: str(tmp_path / "libissl_b200.so"))
    with pytest.raises(ImportError, match="no CPU fallback"):
        L.lib()
