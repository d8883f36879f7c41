"""Failure detection on the device: a slab-filter launch whose bounded waits run out.

``cdftb_filter_test_withhold(k)`` makes the next slab launch's producer issue the TMA copies of its
first k planes and no more. Nothing is then in flight when the consumers' bounded waits (2 s) give
up: the launch records the timeout and leaves, the device stays usable, the drivers' status check
raises, and the next call is clean and correct. No GPU fault, trap or hang is involved.
"""

from __future__ import annotations

import time
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import eigen as oeigen
from oracle.grid import Grid
from oracle.operators import CuspHamiltonian

pytestmark = pytest.mark.gpu


def _operator(pkg, cuda, shape, spacing=0.3, seed=5):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    faces = (rng.uniform(0.5, 1.5, (nx + 8, ny, nz)), rng.uniform(0.5, 1.5, (nx, ny + 8, nz)),
             rng.uniform(0.5, 1.5, (nx, ny, nz + 8)))
    inv = rng.uniform(0.5, 1.5, shape).ravel()
    q = rng.uniform(0.5, 1.5, shape).ravel()
    pot = rng.uniform(-1.0, 1.0, shape).ravel()
    ham_o = CuspHamiltonian(Grid(shape, spacing, (0.0, 0.0, 0.0)), SimpleNamespace(face_weights=lambda o: faces),
                            None, bare=(pot, inv, q))
    grid = pkg.UniformGrid(shape, spacing, (0.0, 0.0, 0.0), device=cuda)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    dev_faces = tuple(t(w) for w in faces)
    ham = pkg.CuspFactoredHamiltonian(grid, SimpleNamespace(face_weights=lambda acc: dev_faces),
                                      bare=(t(pot), t(inv), pkg.Measure(grid, t(q))))
    return ham_o, ham


@pytest.mark.parametrize("wide", [1, 0], ids=["wide", "narrow"])
def test_withheld_copies_time_out_and_the_next_call_is_clean(pkg, cuda, wide):
    lib = pkg._lib.library()
    lib.cdftb_filter_wide(wide)
    try:
        shape = (20, 17, 24)
        ham_o, ham = _operator(pkg, cuda, shape)
        block = np.random.default_rng(11).standard_normal((5, int(np.prod(shape))))
        args = (3, 0.5, 30.0, -1.0)
        want = oeigen.chebyshev_filter(ham_o, block, *args)
        x = torch.from_numpy(block).to(cuda)
        first = pkg.chebyshev_filter(ham, x, *args)  # tunes this shape; a normal call
        torch.cuda.synchronize()
        pkg._lib.check_device_status("before the test")
        assert np.abs(first.cpu().numpy() - want).max() < 1e-12 * np.abs(want).max()

        pkg._lib.call("cdftb_filter_test_withhold", 3)
        t0 = time.perf_counter()
        pkg.chebyshev_filter(ham, x, *args)
        torch.cuda.synchronize()
        waited = time.perf_counter() - t0
        with pytest.raises(pkg._lib.DeviceTimeout):
            pkg._lib.check_device_status("the withheld launch")
        assert waited > 1.5, "the consumers gave up before their 2 s limit"
        assert waited < 30.0
        pkg._lib.check_device_status("after the flag was read")  # read and cleared: no raise

        again = pkg.chebyshev_filter(ham, x, *args)
        torch.cuda.synchronize()
        pkg._lib.check_device_status("the call after the timeout")
        assert torch.equal(again, first)
    finally:
        lib.cdftb_filter_test_withhold(0)
        lib.cdftb_filter_wide(1)


def test_a_timeout_inside_a_solve_raises(pkg, cuda):
    """The drivers read the device status once per iteration: a timed-out launch stops the solve
    with ``DeviceTimeout`` instead of handing its unwritten outputs to the next step."""
    import __graft_entry__  # noqa: F401
    from oracle import scf as oscf

    system = oscf.h_atom(points_per_edge=17, half_box=4.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    geo = pkg.build_cusp_geometry(grid, system.charges, system.positions)
    pkg.solve_noninteracting(geo, n_electrons=1.0)  # tunes the shapes
    pkg._lib.call("cdftb_filter_test_withhold", 2)
    try:
        with pytest.raises(pkg._lib.DeviceTimeout):
            pkg.solve_noninteracting(geo, n_electrons=1.0)
    finally:
        pkg._lib.library().cdftb_filter_test_withhold(0)
    torch.cuda.synchronize()
    pkg._lib.check_device_status("after the failed solve")
    out = pkg.solve_noninteracting(geo, n_electrons=1.0)
    assert out["converged"]
