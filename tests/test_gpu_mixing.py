"""The SCF driver's Kerker preconditioner on the device against the reference's and the oracle's,
and He solves with Kerker mixing against the reference's energies and iteration counts."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import scf as oscf

pytestmark = pytest.mark.gpu

FIXTURES = Path(__file__).resolve().parent / "golden" / "scf_fixtures.npz"


@pytest.fixture(scope="module")
def scf_golden():
    with np.load(FIXTURES) as data:
        return {k: data[k] for k in data.files}


def test_kerker_kernel(pkg, cuda, scf_golden):
    shape = tuple(int(n) for n in scf_golden["kerker_shape"])
    h = float(scf_golden["kerker_spacing"])
    residual = scf_golden["kerker_residual"]
    grid = pkg.UniformGrid(shape, h, (0.0, 0.0, 0.0), device=cuda)
    pre = pkg.scf.KerkerPreconditioner(grid, 1.5)
    x = torch.from_numpy(residual).to(cuda)
    got = pre(x).cpu().numpy()
    want = scf_golden["kerker_out"]
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
    oracle = oscf.KerkerPreconditioner(shape, h, 1.5)(residual)
    assert np.abs(got - oracle).max() < 1e-12 * np.abs(oracle).max()
    assert torch.equal(x, torch.from_numpy(residual).to(cuda))  # input untouched
    # one row, an odd and an even edge, q0 = 0.5
    for shape2 in [(7, 8, 9), (16, 5, 12)]:
        r = np.random.default_rng(1).standard_normal(int(np.prod(shape2)))
        g2 = pkg.UniformGrid(shape2, 0.3, (0.0, 0.0, 0.0), device=cuda)
        got2 = pkg.scf.KerkerPreconditioner(g2, 0.5)(torch.from_numpy(r[None]).to(cuda)).cpu().numpy()[0]
        want2 = oscf.KerkerPreconditioner(shape2, 0.3, 0.5)(r)
        assert np.abs(got2 - want2).max() < 1e-12 * np.abs(want2).max()


@pytest.fixture(scope="module")
def he25(pkg, cuda):
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    return pkg.build_cusp_geometry(grid, system.charges, system.positions)


@pytest.mark.parametrize("tag,mixing", [
    ("scf_kerker", dict(scheme="kerker", kerker_q0=0.5)),
    ("scf_linear_kerker", dict(scheme="linear", alpha=0.3, kerker=True)),
])
def test_he25_scf_with_kerker(pkg, he25, scf_golden, tag, mixing):
    step = pkg.KohnShamStep(he25, "lda_vwn", 2.0)
    out = pkg.solve_self_consistent(step, pkg.MixingConfig(**mixing))
    assert out.converged
    assert out.scf_iterations == int(scf_golden[f"{tag}_iterations"])
    assert abs(out.energies["total"] - float(scf_golden[f"{tag}_total"])) < 1e-10


def test_batched_scf_with_kerker(pkg, he25, scf_golden):
    """Three systems in the batched driver with linear + Kerker mixing (the carried Hartree parts
    are off for a preconditioned residual): each matches the reference."""
    step = pkg.batch.BatchedKohnShamStep(he25, "lda_vwn", 2.0, 3, seeds=[0, 0, 0])
    out = pkg.batch.solve_self_consistent_batch(step, pkg.MixingConfig(scheme="linear", alpha=0.3, kerker=True))
    want = float(scf_golden["scf_linear_kerker_total"])
    for s in range(3):
        assert out.converged[s]
        assert out.scf_iterations[s] == int(scf_golden["scf_linear_kerker_iterations"])
        assert abs(out.energies[s]["total"] - want) < 1e-10


# ------------------------------------------------------------------ LOBPCG, the eigensolver cross-check


@pytest.fixture(scope="module")
def h17(pkg, cuda):
    system = oscf.h_atom(points_per_edge=17, half_box=4.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    return pkg.build_cusp_geometry(grid, system.charges, system.positions)


@pytest.mark.parametrize("k", [1, 2])
def test_lobpcg_matches_the_reference(pkg, h17, scf_golden, k):
    """The bare H atom (box 8, h = 0.5): the reference's LOBPCG eigenvalues, started from the same
    seeded block, in about the same number of iterations."""
    ham = pkg.CuspFactoredHamiltonian(h17.grid, h17.factor, quadrature=h17.quadrature)
    solver = pkg.eigen.LOBPCG(h17.grid, pkg.EigenConfig())
    out = solver.solve(ham, k, generator=pkg.rng.SeededStream(1, h17.grid.device))
    want = scf_golden[f"lobpcg_{k}_eigenvalues"]
    assert out.converged == bool(scf_golden[f"lobpcg_{k}_converged"])
    np.testing.assert_allclose(out.eigenvalues.cpu().numpy(), want, rtol=0, atol=1e-9)
    assert abs(out.n_iterations - int(scf_golden[f"lobpcg_{k}_iterations"])) <= 2


def test_two_solver_cross_check(pkg, h17, scf_golden):
    """``solve_noninteracting(cross_check=True)``: CheFSI and LOBPCG agree to the G2.5 tolerance."""
    out = pkg.solve_noninteracting(h17, 1.0, cross_check=True)
    assert out["two_solver_converged"]
    assert out["two_solver_max_delta"] < 1e-8
    np.testing.assert_allclose(out["eigenvalues"], scf_golden["cross_eigenvalue"], rtol=0, atol=1e-11)
    assert abs(out["lobpcg_iterations"] - float(scf_golden["cross_lobpcg_iterations"])) <= 2
