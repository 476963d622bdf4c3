"""The C-ABI library loads and exports every declared entry point (CPU only, no device work)."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO

HEADERS = sorted(os.path.join(d, f) for d, _, fs in os.walk(os.path.join(REPO, "include")) for f in fs
                 if f.endswith((".h", ".hpp")))


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


def test_library_exports_no_module_class(native):
    """The module class is header-only: the library exports no C++ symbol tied to the layout of
    cracklingConfig or guideResults, so a program compiled against the reference's own types
    cannot bind to a definition built against other ones."""
    out = subprocess.run(["nm", "-DC", "--defined-only", native.library_path()], capture_output=True, text=True,
                         check=True).stdout
    assert "ISSLScoringModule" not in out and "cracklingConfig" not in out and "guideResults" not in out
    for n in ["issl_module_open", "issl_module_run", "issl_module_release_all"]:
        assert re.search(rf"\bT {n}$", out, flags=re.M), n


def test_module_header_compiles_with_mirror_types(native, tmp_path):
    """A standalone program (no reference checkout) builds the class from the mirror types."""
    src = tmp_path / "m.cpp"
    src.write_text('#include "issl_b200_module.hpp"\n'
                   "int main() {\n"
                   "  cracklingConfig cfg;\n"
                   '  cfg.input.offtargetSites = "x.issl";\n'
                   "  cfg.offTarget.enabled = false;\n"
                   "  ISSLScoringModule m(cfg);\n"
                   "  std::vector<guideResults> g(3);\n"
                   "  m.run(g);\n"
                   "  return g[0].passedOffTargetScore == '?' ? 0 : 1;\n"
                   "}\n")
    exe = tmp_path / "m"
    lib_dir = os.path.dirname(native.library_path())
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe),
                    "-L", lib_dir, "-lissl_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)  # disabled: no device work
    assert r.returncode == 0 and "Skipping Off-target scoring" in r.stdout


DROPIN = os.path.join(REPO, "oracle", "_ref", "module_dropin")


@pytest.mark.skipif(not os.path.exists(os.path.join(REPO, "oracle", "_ref", "ref_module_driver")),
                    reason="needs the reference checkout (oracle/_ref is built from it)")
def test_dropin_driver_builds_against_reference_types(native):
    """oracle/_ref/module_dropin: the reference's module driver compiled with the reference's own
    cracklingConfig / guideResults, include/dropin/ISSLScoringModule.hpp in place of the
    reference's header, linked against libissl_b200.so (oracle/Makefile)."""
    assert os.path.exists(DROPIN)
    ldd = subprocess.run(["ldd", DROPIN], capture_output=True, text=True, check=True).stdout
    assert "libissl_b200.so" in ldd
    syms = subprocess.run(["nm", "-C", DROPIN], capture_output=True, text=True, check=True).stdout
    assert "ISSLScoringModule::run(std::vector<guideResults" in syms  # compiled in the program itself


def test_python_module_rejects_bad_method(native):
    with pytest.raises(RuntimeError, match="not valid"):
        native.ISSLScoringModule(native.CracklingConfig("x.issl", method="bogus"))


def test_no_fallback_when_library_missing(tmp_path, monkeypatch):
    import cracklingplusplus_gpu_b200._lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "library_path", lambda: str(tmp_path / "libissl_b200.so"))
    with pytest.raises(ImportError, match="no CPU fallback"):
        L.lib()
