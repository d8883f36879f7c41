"""The slab Chebyshev filter (order 8) against the oracle on random operators.

Covers the internal layout's edge cases: odd and even nz (padding column), grids smaller than a
tile or than a group of 8 planes, both z tiles (32 and 36 columns), x chunking, an odd number of
float32 orbitals (a half-empty lane), several systems with their own potentials and coefficient
tables in one call (a lane whose two orbitals belong to different systems), and degrees 1 and 2.
"""

from __future__ import annotations

import ctypes
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import eigen as oeigen
from oracle.grid import Grid
from oracle.operators import CuspHamiltonian

pytestmark = pytest.mark.gpu


def _t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _random_operator(shape, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    faces = (rng.uniform(0.5, 1.5, (nx + 8, ny, nz)), rng.uniform(0.5, 1.5, (nx, ny + 8, nz)),
             rng.uniform(0.5, 1.5, (nx, ny, nz + 8)))
    inv = rng.uniform(0.5, 1.5, shape).ravel()
    q = rng.uniform(0.5, 1.5, shape).ravel()
    return faces, inv, q


def _pair(pkg, cuda, shape, spacing, faces, inv, q, pot, dtype=torch.float64):
    grid_o = Grid(shape, spacing, (0.0, 0.0, 0.0))
    ham_o = CuspHamiltonian(grid_o, SimpleNamespace(face_weights=lambda order: faces), None, bare=(pot, inv, q))
    grid = pkg.UniformGrid(shape, spacing, (0.0, 0.0, 0.0), device=cuda)
    dev_faces = tuple(_t(w, cuda) for w in faces)
    bare = (_t(pot, cuda), _t(inv, cuda), pkg.Measure(grid, _t(q, cuda)))
    ham = pkg.CuspFactoredHamiltonian(grid, SimpleNamespace(face_weights=lambda acc: dev_faces), bare=bare,
                                      dtype=dtype)
    return ham_o, ham


def _device_status(pkg):
    flags = ctypes.c_int(-1)
    status = pkg._lib.library().cdftb_device_status(ctypes.byref(flags))
    return status, flags.value


SHAPES = [(9, 11, 13), (12, 17, 24), (5, 9, 40), (33, 20, 70), (21, 8, 65)]


@pytest.fixture(params=[1, 0], ids=["wide", "narrow"])
def lanes(request, pkg):
    """The lane layout: 16-byte lane points (the default) or 8-byte ones."""
    lib = pkg._lib.library()
    lib.cdftb_filter_wide(request.param)
    yield request.param
    lib.cdftb_filter_wide(1)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("batch", [1, 3, 4])
def test_slab_filter_float64(pkg, cuda, shape, batch, lanes):
    faces, inv, q = _random_operator(shape, seed=sum(shape) + batch)
    pot = np.random.default_rng(7).standard_normal(int(np.prod(shape)))
    ham_o, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot)
    block = np.random.default_rng(batch).standard_normal((batch, int(np.prod(shape))))
    for degree in (1, 2, 5):
        want = oeigen.chebyshev_filter(ham_o, block, degree, 0.5, 3.0, -1.0)
        got = pkg.chebyshev_filter(ham, _t(block, cuda), degree, 0.5, 3.0, -1.0).cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-12 * np.abs(want).max())
    assert _device_status(pkg) == (0, 0)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("batch", [1, 3, 4])
def test_slab_filter_float32(pkg, cuda, shape, batch, lanes):
    faces, inv, q = _random_operator(shape, seed=sum(shape) + batch)
    pot = np.random.default_rng(7).standard_normal(int(np.prod(shape)))
    ham_o, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot, dtype=torch.float32)
    block = np.random.default_rng(batch).standard_normal((batch, int(np.prod(shape))))
    want = oeigen.chebyshev_filter(ham_o, block, 5, 0.5, 3.0, -1.0)
    got = pkg.chebyshev_filter(ham, _t(block, cuda), 5, 0.5, 3.0, -1.0).cpu().numpy()
    assert got.dtype == np.float64
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-5 * np.abs(want).max())
    assert _device_status(pkg) == (0, 0)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_slab_filter_many_systems(pkg, cuda, dtype, lanes):
    """Three systems x three orbitals: per-system potentials and coefficient tables in one call."""
    from importlib import import_module

    eigen = import_module(pkg.__name__ + ".eigen")
    shape = (14, 13, 29)
    n = int(np.prod(shape))
    faces, inv, q = _random_operator(shape, seed=3)
    rng = np.random.default_rng(5)
    pots = rng.standard_normal((3, n))
    blocks = rng.standard_normal((3, 3, n))
    bounds = [(0.5, 3.0, -1.0), (0.2, 4.0, -0.5), (1.0, 2.5, -2.0)]
    degree = 6
    table = torch.tensor([eigen.chebyshev_coefficients(degree, *b) for b in bounds], dtype=torch.float64,
                         device=cuda)
    _, ham = _pair(pkg, cuda, shape, 0.25, faces, inv, q, pots[0], dtype=dtype)
    got = eigen.filter_with_table(ham, _t(blocks, cuda), table, degree, orbitals_per_group=3,
                                  potential=_t(pots, cuda)).cpu().numpy()
    tol = 1e-12 if dtype == torch.float64 else 2e-5
    for s in range(3):
        ham_o, _ = _pair(pkg, cuda, shape, 0.25, faces, inv, q, pots[s])
        want = oeigen.chebyshev_filter(ham_o, blocks[s], degree, *bounds[s])
        np.testing.assert_allclose(got[s], want, rtol=0, atol=tol * np.abs(want).max())
    assert _device_status(pkg) == (0, 0)


def test_filter_work_bytes_is_checked(pkg, cuda):
    shape = (9, 11, 13)
    faces, inv, q = _random_operator(shape, seed=1)
    pot = np.zeros(int(np.prod(shape)))
    _, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot, dtype=torch.float32)
    op = ham.operator()
    lib = pkg._lib.library()
    need = lib.cdftb_chebyshev_filter_work_bytes(ctypes.byref(op), 3)
    assert need >= 3 * 2 * 9 * 11 * 14 * 8  # three blocks of two float2 lanes of (9, 11, 14), plus geometry
    block = torch.zeros((3, int(np.prod(shape))), dtype=torch.float64, device=cuda)
    out = torch.empty_like(block)
    work = torch.empty(need - 8, dtype=torch.uint8, device=cuda)
    table = torch.zeros((1, 2, 3), dtype=torch.float64, device=cuda)
    status = lib.cdftb_chebyshev_filter(ctypes.byref(op), block.data_ptr(), 0, out.data_ptr(), 0, work.data_ptr(),
                                        need - 8, 3, table.data_ptr(), 2, None)
    assert status == 1  # CDFTB_ERR_ARGUMENT: the work buffer is too small


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_autotuned_tiling_is_bit_identical(pkg, cuda, dtype):
    """The tile autotuner only changes the tiling: its choice gives the heuristic's result bit for bit.

    The shape is used by no other test, so its first call with the autotuner off runs the heuristic
    tiling and leaves no table entry; the next call, with it on, times the candidates and keeps one.
    """
    shape = (37, 23, 71) if dtype == torch.float64 else (35, 21, 69)
    faces, inv, q = _random_operator(shape, seed=11)
    pot = np.random.default_rng(12).standard_normal(int(np.prod(shape)))
    _, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot, dtype=dtype)
    block = _t(np.random.default_rng(13).standard_normal((5, int(np.prod(shape)))), cuda)
    lib = pkg._lib.library()
    # CDFTB_F32 / CDFTB_F64 plus CDFTB_WIDE_LANES: 5 orbitals in 2 float32 or 3 float64 wide lanes
    code = (1 if dtype == torch.float32 else 0) + 16
    lanes = 2 if dtype == torch.float32 else 3
    tz, xc = ctypes.c_int(-1), ctypes.c_int(-1)
    try:
        lib.cdftb_filter_autotune(0)
        heuristic = pkg.chebyshev_filter(ham, block, 6, 0.5, 3.0, -1.0)
        assert lib.cdftb_filter_tuned_tile(*shape, code, lanes, ctypes.byref(tz), ctypes.byref(xc)) == 0
        assert (tz.value, xc.value) == (0, 0)
        lib.cdftb_filter_autotune(1)
        tuned = pkg.chebyshev_filter(ham, block, 6, 0.5, 3.0, -1.0)
        assert lib.cdftb_filter_tuned_tile(*shape, code, lanes, ctypes.byref(tz), ctypes.byref(xc)) == 0
        assert tz.value in (24, 32, 36) and 1 <= xc.value <= shape[0]
        again = pkg.chebyshev_filter(ham, block, 6, 0.5, 3.0, -1.0)
    finally:
        lib.cdftb_filter_autotune(1)
    assert torch.equal(tuned, heuristic) and torch.equal(again, heuristic)
    assert _device_status(pkg) == (0, 0)


def test_autotuned_apply_is_bit_identical(pkg, cuda):
    """The one-launch apply tunes its own (grid, precision, lanes) key the same way, bit for bit."""
    shape = (33, 19, 67)
    faces, inv, q = _random_operator(shape, seed=21)
    pot = np.random.default_rng(22).standard_normal(int(np.prod(shape)))
    _, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot)
    block = _t(np.random.default_rng(23).standard_normal((3, int(np.prod(shape)))), cuda)
    lib = pkg._lib.library()
    tz, xc = ctypes.c_int(-1), ctypes.c_int(-1)
    try:
        lib.cdftb_filter_autotune(0)
        heuristic = ham.apply(block)
        lib.cdftb_filter_autotune(1)
        tuned = ham.apply(block)
        assert lib.cdftb_filter_tuned_tile(*shape, 0 + 16, 2, ctypes.byref(tz), ctypes.byref(xc)) == 0
        assert tz.value in (24, 32, 36) and 1 <= xc.value <= shape[0]
    finally:
        lib.cdftb_filter_autotune(1)
    assert torch.equal(tuned, heuristic)
    assert _device_status(pkg) == (0, 0)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("shape", [(14, 13, 29), (21, 9, 65)])
def test_wide_lanes_many_systems(pkg, cuda, shape, dtype):
    """16-byte lane points (four float32 or two float64 orbitals): 23 systems x 3 orbitals (lanes
    that mix systems, an empty last slot), both z tiles (nz 29 -> 32 columns, nz 65 -> 36), against
    the oracle and against the 8-byte lanes."""
    from importlib import import_module

    eigen = import_module(pkg.__name__ + ".eigen")
    n = int(np.prod(shape))
    systems, per = 23, 3
    faces, inv, q = _random_operator(shape, seed=31)
    rng = np.random.default_rng(32)
    pots = rng.standard_normal((systems, n))
    blocks = rng.standard_normal((systems, per, n))
    bounds = [(0.5 + 0.01 * s, 3.0 + 0.05 * s, -1.0 - 0.02 * s) for s in range(systems)]
    degree = 5
    table = torch.tensor([eigen.chebyshev_coefficients(degree, *b) for b in bounds], dtype=torch.float64,
                         device=cuda)
    _, ham = _pair(pkg, cuda, shape, 0.25, faces, inv, q, pots[0], dtype=dtype)
    lib = pkg._lib.library()
    tol = 2e-5 if dtype == torch.float32 else 1e-12

    def run():
        return eigen.filter_with_table(ham, _t(blocks, cuda), table, degree, orbitals_per_group=per,
                                       potential=_t(pots, cuda)).cpu().numpy()

    try:
        lib.cdftb_filter_wide(1)
        wide = run()
        lib.cdftb_filter_wide(0)
        narrow = run()
    finally:
        lib.cdftb_filter_wide(1)
    for s in (0, 7, 22):
        ham_o, _ = _pair(pkg, cuda, shape, 0.25, faces, inv, q, pots[s])
        want = oeigen.chebyshev_filter(ham_o, blocks[s], degree, *bounds[s])
        np.testing.assert_allclose(wide[s], want, rtol=0, atol=tol * np.abs(want).max())
    np.testing.assert_allclose(wide, narrow, rtol=0, atol=tol * np.abs(narrow).max())
    assert not np.array_equal(wide, narrow)  # the wide kernel ran (its sums run in another order)
    assert _device_status(pkg) == (0, 0)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("shape", [(14, 13, 23), (11, 26, 47)])
def test_wide_tile_of_13_rows(pkg, cuda, shape, dtype):
    """The 13 x 24 tile of the wide kernel: 13 and 26 rows, nzp 24 and 48. With the autotuner off the
    heuristic takes the tile with the fewest padded points, 13 x 24 here (8 x 32 and 8 x 36 pad the
    rows to 16 or 32 and z to 32, 36, 64 or 72); against the oracle, and the autotuner's choice (8 or
    13 rows) bit for bit the same."""
    n = int(np.prod(shape))
    faces, inv, q = _random_operator(shape, seed=51)
    pot = np.random.default_rng(52).standard_normal(n)
    ham_o, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot, dtype=dtype)
    block = np.random.default_rng(53).standard_normal((6, n))
    lib = pkg._lib.library()
    code = (1 if dtype == torch.float32 else 0) + 16
    lanes = 2 if dtype == torch.float32 else 3
    rows = ctypes.c_int(-1)
    tol = 2e-5 if dtype == torch.float32 else 1e-12
    try:
        lib.cdftb_filter_autotune(0)
        heuristic = pkg.chebyshev_filter(ham, _t(block, cuda), 5, 0.5, 3.0, -1.0)
        lib.cdftb_filter_autotune(1)
        tuned = pkg.chebyshev_filter(ham, _t(block, cuda), 5, 0.5, 3.0, -1.0)
        assert lib.cdftb_filter_tuned_tile_rows(*shape, code, lanes, ctypes.byref(rows)) == 0
        assert rows.value in (8, 13)
    finally:
        lib.cdftb_filter_autotune(1)
    want = np.stack([oeigen.chebyshev_filter(ham_o, b, 5, 0.5, 3.0, -1.0) for b in block[:2]])
    got = heuristic.cpu().numpy()
    np.testing.assert_allclose(got[:2], want, rtol=0, atol=tol * np.abs(want).max())
    assert torch.equal(tuned, heuristic)
    assert _device_status(pkg) == (0, 0)


@pytest.mark.parametrize("kinetic", [False, True])
def test_wide_lanes_apply(pkg, cuda, kinetic):
    """The one-launch apply on 40 float64 orbitals (20 wide lanes) against the oracle and against the
    8-byte lanes, with and without the potential."""
    shape = (17, 15, 37)
    n = int(np.prod(shape))
    faces, inv, q = _random_operator(shape, seed=41)
    pot = np.random.default_rng(42).standard_normal(n)
    ham_o, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot)
    block = np.random.default_rng(43).standard_normal((40, n))
    lib = pkg._lib.library()
    run = ham.kinetic_apply if kinetic else ham.apply
    try:
        lib.cdftb_filter_wide(1)
        wide = run(_t(block, cuda)).cpu().numpy()
        lib.cdftb_filter_wide(0)
        narrow = run(_t(block, cuda)).cpu().numpy()
    finally:
        lib.cdftb_filter_wide(1)
    want = np.stack([ham_o.kinetic_apply(b) if kinetic else ham_o.apply(b) for b in block[:3]])
    np.testing.assert_allclose(wide[:3], want, rtol=0, atol=1e-12 * np.abs(want).max())
    np.testing.assert_allclose(wide, narrow, rtol=0, atol=1e-13 * np.abs(narrow).max())
    assert not np.array_equal(wide, narrow)
    assert _device_status(pkg) == (0, 0)


def test_more_than_65535_lanes(pkg, cuda, lanes):
    """131075 float64 orbitals on a 2 x 2 x 2 grid: more than 65535 lanes in either layout (65538
    wide, 131075 narrow), so the filter splits into launches with a lane offset. Sampled orbitals
    from every launch against the oracle."""
    shape = (2, 2, 2)
    n = int(np.prod(shape))
    faces, inv, q = _random_operator(shape, seed=51)
    pot = np.random.default_rng(52).standard_normal(n)
    ham_o, ham = _pair(pkg, cuda, shape, 0.3, faces, inv, q, pot)
    batch = 131075
    block = np.random.default_rng(53).standard_normal((batch, n))
    got = pkg.chebyshev_filter(ham, _t(block, cuda), 3, 0.5, 3.0, -1.0).cpu().numpy()
    rows = np.array([0, 1, 2, 3, 65534, 65535, 65536, 65537, 131069, 131070, 131071, 131072, 131073, 131074])
    want = oeigen.chebyshev_filter(ham_o, block[rows], 3, 0.5, 3.0, -1.0)
    np.testing.assert_allclose(got[rows], want, rtol=0, atol=1e-12 * np.abs(want).max())
    assert np.isfinite(got).all()
    assert _device_status(pkg) == (0, 0)
