"""CPU checks of the drop-in boundary: the C-ABI library loads and exports
every entry point include/dgv_b200.h declares.  No compute calls."""
import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "dgv_b200.h")
LIB = os.path.join(ROOT, "dgv0d3v_direct_collision_b200", "libdgv_b200.so")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dgv_[a-zA-Z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def built_lib():
    if not os.path.exists(LIB):
        from dgv0d3v_direct_collision_b200 import build
        build.build()
    return LIB


def test_header_declares_the_python_export_list():
    from dgv0d3v_direct_collision_b200 import _lib
    assert header_functions() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(built_lib):
    out = subprocess.check_output(["nm", "-D", "--defined-only", built_lib], text=True)
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [f for f in header_functions() if f not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(built_lib)
    for f in header_functions():
        assert hasattr(lib, f)


def test_library_has_no_torch_dependency(built_lib):
    out = subprocess.check_output(["ldd", built_lib], text=True)
    assert "torch" not in out and "libc10" not in out


def test_every_entry_point_cites_a_reference_location():
    """Each declaration's comment names the reference routine (file:line) it
    replaces, or says it has none."""
    src = open(HEADER).read()
    decl = re.compile(r"^(?:int|const char \*)\s*(dgv_[a-z0-9_]+)\s*\([^;]*\);", re.M)
    prev = 0
    for m in decl.finditer(src):
        blk = src[prev:m.end()]
        prev = m.end()
        name = m.group(1)
        if name in ("dgv_ctx_destroy", "dgv_last_error", "dgv_set_stream", "dgv_set_async",
                    "dgv_set_option", "dgv_grid_info", "dgv_A_info", "dgv_export_A", "dgv_step_ab",
                    "dgv_collide_batched", "dgv_apply_linear", "dgv_project", "dgv_vjp"):
            continue  # plumbing, or covered by the comment of a neighbouring declaration
        assert re.search(r"\.f90:\d+|no reference counterpart|no counterpart in the reference", blk, re.I), name


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from dgv0d3v_direct_collision_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(ImportError):
        _lib.load()


def test_status_codes_match_header():
    from dgv0d3v_direct_collision_b200 import _lib
    src = open(HEADER).read()
    for name in ("DGV_OK", "DGV_EINVAL", "DGV_ERANGE", "DGV_ECUDA", "DGV_ETIMEOUT", "DGV_ENOMEM",
                 "DGV_ESTATE", "DGV_EUNSUP", "DGV_PREC_F64", "DGV_PREC_F32C", "DGV_PREC_TC", "DGV_OPT_PROJECT",
                 "DGV_OPT_NCHUNKS", "DGV_OPT_KTIMING", "DGV_OPT_TCFORM", "DGV_OPT_TCTILES", "DGV_OPT_TCSETMB",
                 "DGV_OPT_WAIT_LIMIT_US", "DGV_OPT_TEST_WITHHOLD", "DGV_OPT_TCAUTOTUNE", "DGV_OPT_FGLOBAL",
                 "DGV_OPT_TCPERSIST", "DGV_LAYOUT_F32", "DGV_LAYOUT_TC_CHUNK", "DGV_LAYOUT_TC_BLOCK",
                 "DGV_LAYOUT_TC_ADJ"):
        val = int(re.search(r"#define\s+%s\s+(\d+)" % name, src).group(1))
        assert getattr(_lib, name) == val, name
