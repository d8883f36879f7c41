"""GPU: the batched SCF driver -- many systems per launch -- against the single-system driver and the reference."""

from __future__ import annotations

import pytest
import torch

from oracle import scf as oscf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def he25_geometry(pkg, cuda):
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    return pkg.build_cusp_geometry(grid, system.charges, system.positions)


def test_batch_of_one_is_the_single_solve(pkg, he25_geometry, golden_values):
    single = pkg.solve_self_consistent(pkg.KohnShamStep(he25_geometry, "lda_vwn", 2.0),
                                       pkg.MixingConfig(scheme="linear", alpha=0.3))
    step = pkg.batch.BatchedKohnShamStep(he25_geometry, "lda_vwn", 2.0, 1)
    out = pkg.batch.solve_self_consistent_batch(step, pkg.MixingConfig(scheme="linear", alpha=0.3))
    assert out.converged == [True]
    assert out.scf_iterations[0] == single.scf_iterations
    assert abs(out.energies[0]["total"] - single.energies["total"]) < 1e-12
    assert abs(out.energies[0]["total"] - golden_values["he25_lda_linear"]["total"]) < 1e-11


def test_batch_of_seeds_float64(pkg, he25_geometry, golden_values):
    step = pkg.batch.BatchedKohnShamStep(he25_geometry, "lda_vwn", 2.0, 4, seeds=[0, 1, 2, 3])
    out = pkg.batch.solve_self_consistent_batch(step, pkg.MixingConfig(scheme="linear", alpha=0.3))
    ref = golden_values["he25_lda_linear"]["total"]
    assert all(out.converged)
    for e in out.energies:
        assert abs(e["total"] - ref) < 1e-8
    assert abs(out.energies[0]["total"] - ref) < 1e-11  # seed 0 is the reference's own start
    assert max(out.measurements["charge_error"]) < 1e-12


def test_batch_mixed_precision(pkg, he25_geometry, golden_values):
    step = pkg.batch.BatchedKohnShamStep(he25_geometry, "lda_vwn", 2.0, 3, seeds=[0, 5, 9],
                                         filter_precision=torch.float32)
    out = pkg.batch.solve_self_consistent_batch(step, pkg.MixingConfig(scheme="linear", alpha=0.3))
    ref = golden_values["he25_lda_linear"]
    assert all(out.converged)
    for e, ev in zip(out.energies, out.eigenvalues):
        assert abs(e["total"] - ref["total"]) < 1e-8
        assert abs(ev[0] - ref["eigenvalues"][0]) < 1e-6
    assert out.measurements["filter_precision"] == "float32"
