"""The C-ABI library builds, loads without a GPU and exports every symbol ``include/cdftb.h`` declares."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared() -> list[str]:
    names = []
    for header in sorted((ROOT / "include").glob("*.h")):
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(cdftb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = _declared()
    for needed in ("cdftb_cusp_apply", "cdftb_chebyshev_filter", "cdftb_measure_cross_f64", "cdftb_weighted_divergence_f64"):
        assert needed in names


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg._lib.library()
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_signatures_cover_header(pkg):
    pkg._lib.library()
    declared = set(_declared())
    bound = set(pkg._lib.SIGNATURES)
    assert declared <= bound, sorted(declared - bound)


def test_version_and_status_without_gpu(pkg):
    lib = pkg._lib.library()
    assert lib.cdftb_version() >= 10000
    assert lib.cdftb_status_string(0) == b"ok"
    assert b"argument" in lib.cdftb_status_string(1)


def test_argument_errors_need_no_gpu(pkg):
    """Shape errors are rejected on the host before any launch."""
    with pytest.raises(pkg._lib.CdftbError):
        pkg._lib.call("cdftb_weighted_divergence_f64", None, None, 1, 0, 4, 4, None, None, None, 0.5, 8, None)
    with pytest.raises(pkg._lib.CdftbError):
        pkg._lib.call("cdftb_small_eigh_f64", None, None, None, 40, 1, None)
