"""The threaded CPU baseline: the timed filter is the oracle's, bit for bit, on any thread count."""

from __future__ import annotations

import numpy as np
import pytest


@pytest.mark.parametrize("threads", [1, 3, 8, 16])
def test_threaded_filter_is_the_oracle_filter(threads):
    import bench
    from oracle import eigen as oeigen
    from oracle import scf as oscf
    from oracle.operators import CuspHamiltonian

    system = oscf.h_atom(points_per_edge=17, half_box=4.0)
    grid, factor, quad = oscf.build_geometry(system)
    ham = CuspHamiltonian(grid, factor, quad)
    block = np.random.default_rng(3).standard_normal((5, grid.n_points))
    want = oeigen.chebyshev_filter(ham, block, 6, 0.5, 30.0, -1.0)
    got, used = bench._threaded_filter(ham, block, 6, 0.5, 30.0, -1.0, threads)
    assert np.array_equal(got, want)
    assert used == (min(threads, 5) if threads < 15 else 15)


@pytest.mark.parametrize("name", ["lda_vwn", "pbe"])
def test_chunked_xc_is_the_oracle_xc(name):
    from concurrent.futures import ThreadPoolExecutor

    import bench
    from oracle import xc as oxc

    rng = np.random.default_rng(9)
    density = rng.uniform(1e-6, 2.0, 1001)
    sigma = rng.uniform(0.0, 1.0, 1001) if name == "pbe" else None
    want = oxc.evaluate(name, density, sigma)
    with ThreadPoolExecutor(4) as pool:
        got = bench._chunked_xc(oxc.evaluate, pool, 7)(name, density, sigma)
    for g, w in zip(got, want):
        assert (g is None and w is None) or np.array_equal(g, w)


def test_row_block_products_keep_the_potentials():
    """The interpolant and lift as threaded row blocks leave the oracle's potentials bit for bit."""
    from concurrent.futures import ThreadPoolExecutor

    import bench
    from oracle import scf as oscf

    system = oscf.he_lda(spacing=0.5, edge=8.0)
    grid, factor, quad = oscf.build_geometry(system)
    step = oscf.KohnShamStep(system, grid, factor, quad)
    n0 = oscf.initial_density(step)
    want = step.potentials(n0)
    serial = quad.L, quad.LT
    with ThreadPoolExecutor(3) as pool:
        quad.L, quad.LT = bench._RowBlocks(serial[0], pool, 5), bench._RowBlocks(serial[1], pool, 5)
        try:
            got = step.potentials(n0)
        finally:
            quad.L, quad.LT = serial
    for key, value in want.items():
        assert np.array_equal(np.asarray(got[key]), np.asarray(value)), key


def test_threaded_whole_solve_is_the_oracle_solve():
    """The timed CPU solve (the oracle's own solve with its parts on host threads) gives the oracle's
    energies and density bit for bit, and the patched functions are restored afterwards."""
    import bench
    from oracle import operators as oops
    from oracle import scf as oscf
    from oracle import xc as oxc

    system = oscf.he_lda(spacing=0.5, edge=8.0)
    geometry = oscf.build_geometry(system)
    want = oscf.solve_self_consistent(system, geometry)
    from oracle import eigen as oeigen

    saved = (oxc.evaluate, oops.CuspHamiltonian.kinetic_apply, oops.CoulombCutoffPoisson.solve,
             oscf.KohnShamStep.potentials, oeigen.chebyshev_filter, geometry[2].L, geometry[2].LT)
    got, seconds, breakdown = bench.oracle_solve(system, geometry, 4)
    assert (oxc.evaluate, oops.CuspHamiltonian.kinetic_apply, oops.CoulombCutoffPoisson.solve,
            oscf.KohnShamStep.potentials, oeigen.chebyshev_filter, geometry[2].L, geometry[2].LT) == saved
    assert got["scf_iterations"] == want["scf_iterations"]
    # the FFTs differ (scipy on threads vs numpy): the Poisson solution agrees to rounding only
    assert abs(got["energies"]["total"] - want["energies"]["total"]) < 1e-12
    assert np.abs(got["density"] - want["density"]).max() < 1e-10
    # the operator applications plus one kinetic application per energy evaluation
    assert breakdown["block_applications"] == want["applications"] + want["scf_iterations"] + 1
    assert seconds > 0.0


@pytest.mark.parametrize("which", ["he65", "he101", "h2plus_short", "h2plus_long"])
def test_workload_systems_are_the_oracle_systems(pkg, which):
    """The measured workloads build their grids from the package's own system definitions; the CPU
    baseline and the parity tests from the oracle's. Both describe the same nuclei, electrons, box,
    spacing and anchoring."""
    from oracle import scf as oscf

    ours, theirs = {
        "he65": (pkg.systems.he_lda(), oscf.he_lda()),
        "he101": (pkg.systems.he_lda(spacing=0.16, edge=16.0), oscf.he_lda(spacing=0.16, edge=16.0)),
        "h2plus_short": (pkg.systems.h2_plus(0.8), oscf.h2_plus(0.8, spacing=0.25, transverse=12.0)),
        "h2plus_long": (pkg.systems.h2_plus(6.0, spacing=0.4, transverse=10.0), oscf.h2_plus(6.0, 0.4, 10.0)),
    }[which]
    for field in ("charges", "positions", "n_electrons", "box_lengths", "spacing", "anchor"):
        assert getattr(ours, field) == getattr(theirs, field), field
