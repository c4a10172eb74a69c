"""The C ABI library loads without a GPU and exports every declared symbol."""

from __future__ import annotations

import pathlib
import re

import pytest

REPO = pathlib.Path(__file__).resolve().parents[1]
HEADERS = sorted((REPO / "include").glob("*.h"))


def declared_functions() -> set[str]:
    names: set[str] = set()
    for header in HEADERS:
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(gf_[a-zA-Z0-9_]+)\s*\(", text))
    return names


def test_header_declares_functions():
    names = declared_functions()
    assert "gf_pcg_solve" in names and "gf_bicgstab_solve" in names and "gf_assemble" in names


def test_library_exports_every_declared_symbol():
    from gridfoam_b200 import _lib

    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built (run __graft_entry__.build())")
    lib = _lib.load()
    missing = [n for n in sorted(declared_functions()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_lib.EXPORTED) == declared_functions()
    assert lib.gf_version() >= 1
    # Pure-host query: workspace sizing needs no device.
    assert lib.gf_krylov_workspace_size(1000, 3, 1) > 18000


def test_invalid_arguments_fail_loudly():
    """Argument validation runs on the host and reports through gf_last_error."""
    from gridfoam_b200 import _lib

    if not _lib.LIB_PATH.exists():
        pytest.skip("library not built")
    lib = _lib.load()
    status = lib.gf_pcg_solve(None, None)
    assert status == _lib.GF_ERR_INVALID
    assert b"invalid" in lib.gf_last_error()
    with pytest.raises(_lib.GfError):
        _lib.call("gf_spmv", None, 1, None, None, None, None, None)
