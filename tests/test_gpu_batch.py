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


# ------------------------------------------------------------------ systems on their own grids


def _scan_geometry(pkg, cuda, bond, spacing=0.25, transverse=12.0):
    system = oscf.h2_plus(bond, spacing=spacing, transverse=transverse)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    return pkg.build_cusp_geometry(grid, system.charges, system.positions)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_multi_grid_filter_matches_single_grids(pkg, cuda, dtype):
    """One launch over systems of different grids (26 x 26 x 33, 26 x 26 x 37, 33 x 33 x 41) equals the
    per-system filters; the tiles wholly beyond a system's own grid (rows from 32 on for the 26-row
    systems) store zeros without computing, and the result equals the launch that computes them (no
    system shapes given)."""
    geos = [_scan_geometry(pkg, cuda, bond, spacing=0.4, transverse=t)
            for bond, t in ((0.8, 10.0), (2.6, 10.0), (4.1, 12.8))]
    assert len({g.grid.shape for g in geos}) == 3
    h = pkg.batch.MultiGeometryHamiltonian(geos)
    if dtype == torch.float32:
        h = h.as_dtype(torch.float32)
    k = 5
    degree = 7
    bounds = [(0.4, 30.0, -1.5), (0.3, 28.0, -1.2), (0.5, 32.0, -1.0)]
    rows = [pkg.chebyshev_coefficients(degree, *bb) for bb in bounds]
    table = torch.tensor(rows, dtype=torch.float64, device=cuda)
    gen = torch.Generator().manual_seed(4)
    blocks = [torch.randn((k, g.grid.n_points), dtype=torch.float64, generator=gen).to(cuda) for g in geos]
    big = torch.stack([h.embed(s, blocks[s]) for s in range(3)])
    got = h.filter(big, table, degree)
    tol = 1e-12 if dtype == torch.float64 else 2e-5
    for s, g in enumerate(geos):
        single = pkg.CuspFactoredHamiltonian(g.grid, g.factor, quadrature=g.quadrature, dtype=dtype)
        want = pkg.chebyshev_filter(single, blocks[s], degree, *bounds[s])
        sub = h.extract(s, got[s])
        torch.testing.assert_close(sub, want, rtol=0, atol=tol * float(want.abs().max()))
        outside = got[s].reshape(-1, *h.grid.shape)
        sx, sy, sz = g.grid.shape
        assert float(outside[:, sx:].abs().max() if sx < h.grid.shape[0] else 0.0) == 0.0
        assert float(outside[:, :, sy:].abs().max() if sy < h.grid.shape[1] else 0.0) == 0.0
        assert float(outside[:, :, :, sz:].abs().max() if sz < h.grid.shape[2] else 0.0) == 0.0
    assert min(s[1] for s in h.shapes) <= 32 < h.grid.shape[1]

    class Unshaped(type(h)):
        def _op(self, k):
            op = super()._op(k)
            op.system_shapes = None
            return op

    full = Unshaped.__new__(Unshaped)
    full.__dict__.update(h.__dict__)
    assert torch.equal(full.filter(big, table, degree), got)


SCAN = tuple(0.8 + k * 5.2 / 47 for k in (0, 11, 23, 35, 47))


@pytest.mark.parametrize("precision", [torch.float64, torch.float32])
def test_batched_scan_matches_the_reference(pkg, cuda, golden_values, precision):
    """Config 4: five members of the H2+ scan (grids 49x49x52 .. 73) in one batched solve."""
    refs = [golden_values.get(f"h2plus_scan_R{bond:.4f}") for bond in SCAN]
    if any(r is None for r in refs):
        pytest.skip("no scan fixtures (make_golden.py --with-scan)")
    geos = [_scan_geometry(pkg, cuda, bond) for bond in SCAN]
    out = pkg.batch.solve_noninteracting_batch(geos, 1.0, filter_precision=precision)
    for res, ref in zip(out, refs):
        assert res["converged"]
        if precision == torch.float64:
            assert abs(res["total"] - ref["total"]) < 1e-11
            assert res["iterations"] == ref["iterations"]
        else:
            assert abs(res["total"] - ref["total"]) < 1e-9


# ------------------------------------------------------------------ GGA and the other functionals in the batch


def test_batched_pbe_h2(pkg, cuda, golden_values):
    """H2 PBE (h = 0.4, box 10 x 10 x 11.2, default periodic Pulay, degree 16): two systems of the
    batched driver each give the reference's energy and iteration count."""
    system = oscf.h2_pbe(spacing=0.4, box=(10.0, 10.0, 11.2))
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    geo = pkg.build_cusp_geometry(grid, system.charges, system.positions)
    step = pkg.batch.BatchedKohnShamStep(geo, "pbe", 2.0, 2, pkg.EigenConfig(chebyshev_degree=16), seeds=[0, 0])
    out = pkg.batch.solve_self_consistent_batch(step, pkg.MixingConfig())
    ref = golden_values["h2_pbe_h04"]
    for s in range(2):
        assert out.converged[s]
        assert out.scf_iterations[s] == ref["iterations"]
        assert abs(out.energies[s]["total"] - ref["total"]) < 1e-10


def test_config3_batched_mixed(pkg, cuda, golden_values):
    """Config 3 (H2 PBE, 81 x 81 x 91, degree 16) batched in the mixed form: float32 filter, float64
    Rayleigh--Ritz and refinement; within 1e-8 Ha of the reference's float64 energy."""
    system = oscf.h2_pbe()
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    geo = pkg.build_cusp_geometry(grid, system.charges, system.positions)
    step = pkg.batch.BatchedKohnShamStep(geo, "pbe", 2.0, 2, pkg.EigenConfig(chebyshev_degree=16), seeds=[0, 3],
                                         filter_precision=torch.float32)
    out = pkg.batch.solve_self_consistent_batch(step, pkg.MixingConfig())
    ref = golden_values["h2_pbe_h020"]["total"]
    assert all(out.converged)
    for e in out.energies:
        assert abs(e["total"] - ref) < 1e-8


def test_batched_blyp_he25(pkg, he25_geometry):
    """A non-VWN functional in the batch (the generic path) equals the single-system solve."""
    mixing = pkg.MixingConfig(scheme="linear", alpha=0.3)
    single = pkg.solve_self_consistent(pkg.KohnShamStep(he25_geometry, "blyp", 2.0), mixing)
    step = pkg.batch.BatchedKohnShamStep(he25_geometry, "blyp", 2.0, 2, seeds=[0, 0])
    out = pkg.batch.solve_self_consistent_batch(step, mixing)
    for s in range(2):
        assert out.converged[s]
        assert out.scf_iterations[s] == single.scf_iterations
        assert abs(out.energies[s]["total"] - single.energies["total"]) < 1e-11


def test_level_shifted_batch_matches_the_single_system_rung(pkg, he25_geometry):
    """The ladder's last rung in the batch: CheFSI on H + 0.5 (1 - P_occ) for two systems gives the
    single-system driver's level-shifted diagonalisation (``loop.py:553-589``)."""
    step = pkg.KohnShamStep(he25_geometry, "lda_vwn", 2.0)
    p = step.potentials(pkg.initial_density(step))
    eigen0, _ = step.diagonalise(step.hamiltonian(p))
    occ = step.occupy(eigen0.eigenvalues)
    shifted = pkg.scf._LevelShifted(step.hamiltonian(p), eigen0, occ, 0.5)
    single, info = step.diagonalise(shifted, initial=eigen0.eigenvectors, max_iterations=4)

    bstep = pkg.batch.BatchedKohnShamStep(he25_geometry, "lda_vwn", 2.0, 2, seeds=[0, 0])
    bh = bstep.hamiltonian(p.effective[None].expand(2, -1).contiguous())
    init = eigen0.eigenvectors[None].expand(2, -1, -1).contiguous()
    op = pkg.batch.LevelShiftedBatch(bh, init[:, :1], 0.5)
    streams = [pkg.rng.SeededStream(0, he25_geometry.grid.device) for _ in range(2)]
    evals, vectors, _, states = pkg.batch.batched_chefsi(op, None, step.n_states, step.eigen, init, streams,
                                                         [None, None], 4, None)
    want = single.eigenvalues.cpu()
    for s in range(2):
        assert states[s].iterations == single.n_iterations
        torch.testing.assert_close(evals[s].cpu(), want, rtol=0, atol=1e-10)
        assert abs(states[s].spectrum[1] - info["eigen_spectral_bounds"][1]) < 1e-9
