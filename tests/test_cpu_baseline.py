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
