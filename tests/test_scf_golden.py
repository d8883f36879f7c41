"""The oracle's SCF-driver pieces against the reference's own (``tests/golden/scf_fixtures.npz``,
written by ``make_scf_golden.py``): the Kerker preconditioner."""

from __future__ import annotations

from pathlib import Path

import numpy as np

from oracle import scf as oscf

FIXTURES = Path(__file__).resolve().parent / "golden" / "scf_fixtures.npz"


def test_kerker_matches_the_reference():
    with np.load(FIXTURES) as f:
        shape, h = tuple(int(n) for n in f["kerker_shape"]), float(f["kerker_spacing"])
        residual, want = f["kerker_residual"], f["kerker_out"]
    got = oscf.KerkerPreconditioner(shape, h, 1.5)(residual)
    assert np.abs(got - want).max() < 1e-13 * np.abs(want).max()
    # the filter removes the mean (q = 0) and leaves the rest of the spectrum nearly unchanged at q >> q0
    assert abs(got.sum(axis=-1)).max() < 1e-10
