"""The graphed Chebyshev filter (``eigen.GraphedChebyshevFilter``, after ``chefsi.py:185-392``).

GPU: a replay is bit for bit the direct library call, for a new block, new coefficients and a new
potential on the same geometry (one capture serves them all), in float64 and float32; solves with
``graphs=True`` give the same energies and iteration counts as without. CPU: the engine's direct
calls, counted by reason, for a block off the GPU and an operator without the graph seam.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import scf as oscf


def _t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def _hamiltonian(pkg, cuda, shape, seed, dtype, potential_seed=None):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    faces = tuple(_t(rng.uniform(0.5, 1.5, s), cuda) for s in
                  ((nx + 8, ny, nz), (nx, ny + 8, nz), (nx, ny, nz + 8)))
    inv = _t(rng.uniform(0.5, 1.5, shape).ravel(), cuda)
    q = _t(rng.uniform(0.5, 1.5, shape).ravel(), cuda)
    prng = np.random.default_rng(seed if potential_seed is None else potential_seed)
    pot = _t(prng.uniform(-2.0, 0.5, shape).ravel(), cuda)
    grid = pkg.UniformGrid(shape, 0.3, (0.0, 0.0, 0.0), device=cuda)
    factor = SimpleNamespace(face_weights=lambda acc: faces)
    return grid, factor, inv, q, pot, dtype


def _build(pkg, grid, factor, inv, q, pot, dtype):
    bare = (pot, inv, pkg.Measure(grid, q))
    return pkg.CuspFactoredHamiltonian(grid, factor, bare=bare, dtype=dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_replay_is_the_direct_call(pkg, cuda, dtype):
    shape = (21, 8, 65)
    grid, factor, inv, q, pot, _ = _hamiltonian(pkg, cuda, shape, 7, dtype)
    ham = _build(pkg, grid, factor, inv, q, pot, dtype)
    engine = pkg.eigen.GraphedChebyshevFilter(cuda)
    gen = torch.Generator(device="cpu").manual_seed(11)
    degree = 9
    bounds = [(0.5, 40.0, -3.0), (0.7, 38.0, -2.5), (0.2, 45.0, -3.5)]
    for call, (lower, upper, smin) in enumerate(bounds):
        if call == 2:  # a new SCF Hamiltonian: same geometry, another potential
            pot2 = pot + _t(np.random.default_rng(5).uniform(-0.1, 0.1, grid.n_points), cuda)
            ham = _build(pkg, grid, factor, inv, q, pot2, dtype)
        block = torch.randn(5, grid.n_points, generator=gen, dtype=torch.float64).to(cuda)
        before = ham.apply_count
        got = engine(ham, block, degree, lower, upper, smin)
        want = pkg.chebyshev_filter(ham, block, degree, lower, upper, smin)
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}: max diff {(got - want).abs().max().item()}"
        assert ham.apply_count - before == 2 * degree
    rec = engine.record()
    assert rec["used"] and rec["captures"] == 1 and rec["replays"] == 2
    assert rec["validation_max_rel_diff"] == 0.0
    assert rec["eager_calls"] == {"validation of a new capture": 1}
    # another block shape captures again
    block = torch.randn(3, grid.n_points, generator=gen, dtype=torch.float64).to(cuda)
    engine(ham, block, degree, 0.5, 40.0, -3.0)
    got = engine(ham, block, degree, 0.6, 40.0, -3.0)
    assert torch.equal(got, pkg.chebyshev_filter(ham, block, degree, 0.6, 40.0, -3.0))
    assert engine.record()["captures"] == 2


@pytest.mark.gpu
def test_noninteracting_solve_with_graphs(pkg, cuda):
    system = oscf.h_atom(points_per_edge=17, half_box=4.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, cuda)
    geo = pkg.build_cusp_geometry(grid, system.charges, system.positions)
    direct = pkg.solve_noninteracting(geo, n_electrons=1.0, seed=system.seed)
    graphed = pkg.solve_noninteracting(geo, n_electrons=1.0, seed=system.seed, graphs=True)
    assert graphed["total"] == direct["total"]
    assert graphed["iterations"] == direct["iterations"]
    assert graphed["applications"] == direct["applications"]
    rec = graphed["cuda_graphs"]
    assert rec["used"] and rec["captures"] == 1 and rec["replays"] == direct["iterations"] - 1


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [torch.float64, torch.float32], ids=["f64", "mixed"])
def test_scf_with_graphs(pkg, cuda, golden_values, precision):
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    geo = pkg.build_cusp_geometry(grid, system.charges, system.positions)
    mixing = pkg.MixingConfig(scheme="linear", alpha=0.3)
    direct = pkg.solve_self_consistent(pkg.KohnShamStep(geo, "lda_vwn", 2.0, filter_precision=precision), mixing)
    graphed = pkg.solve_self_consistent(
        pkg.KohnShamStep(geo, "lda_vwn", 2.0, filter_precision=precision, graphs=True), mixing)
    assert graphed.energies["total"] == direct.energies["total"]
    assert graphed.scf_iterations == direct.scf_iterations
    assert graphed.applications == direct.applications
    rec = graphed.measurements["cuda_graphs"]
    assert rec["used"] and rec["replays"] > 10 * rec["captures"]
    # float64: one capture serves every filter call; mixed: a few (the float and float64 operators,
    # the full and the warm-started diagonalisations)
    assert rec["captures"] == 1 if precision == torch.float64 else rec["captures"] <= 4
    if precision == torch.float64:
        assert abs(graphed.energies["total"] - golden_values["he25_lda_linear"]["total"]) < 1e-11


class _ApplyOnly:
    """An operator with only ``apply`` (as the level-shifted rung): no graph seam."""

    def __init__(self, diag):
        self.diag = diag

    def apply(self, x):
        return x * self.diag


def test_direct_calls_counted_by_reason(pkg):
    engine = pkg.eigen.GraphedChebyshevFilter("cpu")
    diag = torch.linspace(-1.0, 5.0, 40, dtype=torch.float64)
    block = torch.randn(2, 40, dtype=torch.float64, generator=torch.Generator().manual_seed(1))
    out = engine(_ApplyOnly(diag), block, 4, 1.0, 5.5, -1.2)
    assert torch.equal(out, pkg.eigen._eager_filter(_ApplyOnly(diag), block, 4, 1.0, 5.5, -1.2))
    rec = engine.record()
    assert not rec["used"] and rec["replays"] == 0 and rec["captures"] == 0
    assert rec["eager_calls"] == {"block on cpu; graphs are CUDA-only": 1}
    assert rec["reason"] == "no filter call was graph-capable"
    with pytest.raises(ValueError, match="empty"):
        engine(_ApplyOnly(diag), block, 4, 5.5, 1.0, -1.2)
    disabled = pkg.eigen.GraphedChebyshevFilter("cpu", reason_disabled="turned off")
    disabled(_ApplyOnly(diag), block, 4, 1.0, 5.5, -1.2)
    assert disabled.record()["reason"] == "turned off"
    assert disabled.record()["eager_calls"] == {"disabled": 1}
