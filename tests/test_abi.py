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


@pytest.mark.parametrize("dtype", [0, 1])  # CDFTB_F64, CDFTB_F32
def test_work_sizes_cover_the_wide_lanes(pkg, dtype):
    """Host-side size queries: the work buffers hold the 16-byte wide lanes (four float32 or two
    float64 orbitals per point) as well as the 8-byte ones. With one shared geometry the lanes run
    over the whole batch; with per-system geometry both layouts start each orbital group on a
    fresh lane. The filter holds three lane copies and the apply one, beside the same geometry
    copies, so the two sizes differ by two lane copies."""
    lib = pkg._lib.library()
    op = pkg._lib.Operator()
    op.nx, op.ny, op.nz = 9, 9, 13
    op.accuracy, op.spacing, op.dtype, op.orbitals_per_group = 8, 0.3, dtype, 5
    points = 9 * 9 * 14  # nz padded to even
    batch, groups = 10, 2
    per_wide = 4 if dtype == 1 else 2
    narrow_shared = (batch + 1) // 2 if dtype == 1 else batch   # float2 pairs / one orbital per lane
    narrow_grouped = groups * 3 if dtype == 1 else batch        # 3 pairs per 5-orbital group / 10
    wide_shared = -(-batch // per_wide)                         # 3 / 5
    wide_grouped = groups * -(-5 // per_wide)                   # 2 x 2 / 2 x 3
    lane_shared = max(narrow_shared * 8, wide_shared * 16) * points
    lane_grouped = max(narrow_grouped * 8, wide_grouped * 16) * points
    assert lane_grouped > lane_shared
    op.per_system_geometry = 0
    filt_shared = lib.cdftb_chebyshev_filter_work_bytes(ctypes.byref(op), batch)
    apply_shared = lib.cdftb_cusp_apply_work_bytes(ctypes.byref(op), batch)
    op.per_system_geometry = 1
    filt_grouped = lib.cdftb_chebyshev_filter_work_bytes(ctypes.byref(op), batch)
    apply_grouped = lib.cdftb_cusp_apply_work_bytes(ctypes.byref(op), batch)
    assert filt_shared - apply_shared == 2 * lane_shared
    assert filt_grouped - apply_grouped == 2 * lane_grouped
    assert filt_grouped > filt_shared and apply_grouped > apply_shared  # two geometry copies, wider lanes
