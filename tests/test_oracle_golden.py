"""The oracle against the reference's own outputs (fixtures made by ``tests/golden/make_golden.py``).

CPU only. These tests pin the numpy restatement in ``oracle/`` to the reference, so that the GPU
parity tests, which compare against the oracle, compare against the reference.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import eigen, scf, xc
from oracle.geometry import CuspFactor, CuspQuadrature
from oracle.grid import Grid, fd_coefficients, staggered_coefficients, weighted_divergence
from oracle.operators import CoulombCutoffPoisson, CuspHamiltonian
from oracle.rng import make_generator

PROBE_SEED = 1234


def _checks(a: np.ndarray):
    flat = a.reshape(-1)
    g = torch.Generator().manual_seed(PROBE_SEED)
    p = torch.randn(flat.size, dtype=torch.float64, generator=g).numpy()
    return np.array([flat.sum(), (flat * flat).sum(), (flat * p).sum()])


def _close(got, want, rtol):
    got, want = np.asarray(got, dtype=np.float64), np.asarray(want, dtype=np.float64)
    scale = np.maximum(np.abs(want), 1e-300)
    assert np.all(np.abs(got - want) <= rtol * np.maximum(scale, np.abs(want).max() * 1e-3)), (got, want)


def test_coefficients(golden_arrays):
    for acc in (2, 4, 6, 8):
        assert np.array_equal(np.array(staggered_coefficients(acc)), golden_arrays[f"staggered_{acc}"])
    assert np.array_equal(np.array(fd_coefficients(1, 8)), golden_arrays["fd1_8"])


def test_weighted_divergence(golden_arrays):
    faces = [golden_arrays[f"div_w{a}"] for a in range(3)]
    out = weighted_divergence(golden_arrays["div_box"], faces, 0.37, 8)
    np.testing.assert_allclose(out, golden_arrays["div_out"], rtol=1e-13, atol=1e-13 * np.abs(out).max())


@pytest.fixture(scope="module")
def he25():
    system = scf.he_lda(spacing=0.5, edge=12.0)
    grid, factor, quad = scf.build_geometry(system)
    return system, grid, factor, quad


def test_he25_geometry(he25, golden_values, golden_arrays):
    _, grid, factor, quad = he25
    g = golden_values["he25"]
    assert list(grid.shape) == g["shape"]
    assert quad.n_nodes == g["n_nodes"]
    _close(_checks(factor.weight), g["f2_grid"], 1e-12)
    _close(_checks(factor.grad_u), g["grad_u"], 1e-12)
    _close(_checks(factor.transformed_potential), g["transformed_potential"], 1e-12)
    for axis, w in enumerate(factor.face_weights(8)):
        _close(_checks(w), g[f"face_{axis}"], 1e-12)
    _close(_checks(quad.points), g["node_points"], 1e-12)
    _close(_checks(quad.weights), g["node_weights"], 1e-11)
    _close(_checks(quad.partition), g["node_partition"], 1e-11)
    _close(_checks(quad.f2), g["node_f2"], 1e-12)
    np.testing.assert_allclose(quad.mass_weights, golden_arrays["he25_mass_weights"], rtol=1e-12)
    potential, inverse_weight, _ = quad.bare_operator_terms()
    np.testing.assert_allclose(potential, golden_arrays["he25_bare_potential"], rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(factor.transformed_potential, golden_arrays["he25_W"], rtol=1e-13)


def test_he25_apply_rr_filter(he25, golden_values, golden_arrays):
    _, grid, factor, quad = he25
    g = golden_values["he25"]
    ham = CuspHamiltonian(grid, factor, quad)
    gen = torch.Generator().manual_seed(11)
    block = torch.randn((5, grid.n_points), dtype=torch.float64, generator=gen).numpy()
    applied = ham.apply(block)
    np.testing.assert_allclose(applied[:, ::97], golden_arrays["he25_apply_sub"], rtol=1e-11, atol=1e-9)
    for i in range(5):
        _close(_checks(applied[i]), g["apply_rows"][i], 1e-11)
    lo, hi = ham.spectral_bounds(generator=make_generator(0))
    _close([lo, hi], g["lanczos_bounds"], 1e-10)
    evals, vectors, orth = eigen.rayleigh_ritz(ham, block, ham.measure)
    _close(evals, g["rr_evals"], 1e-11)
    deg, lower, upper, smin = g["filter_args"]
    rows = eigen.chebyshev_coefficients(deg, lower, upper, smin)
    np.testing.assert_allclose(np.array(rows), np.array(g["cheb_rows"]), rtol=1e-15)
    filtered = eigen.chebyshev_filter(ham, block, deg, lower, upper, smin)
    for i in range(5):
        _close(_checks(filtered[i]), g["filter_rows"][i], 1e-9)


def test_he25_poisson_and_potentials(he25, golden_values, golden_arrays):
    system, grid, factor, quad = he25
    g = golden_values["he25"]
    poisson = CoulombCutoffPoisson(grid, 2.5)
    assert list(poisson.padded_shape) == g["poisson_padded_shape"]
    pts = grid.points()
    rsq = (pts * pts).sum(axis=-1)
    gauss = np.exp(-rsq / (2 * 1.2 ** 2)) / ((2 * np.pi) ** 1.5 * 1.2 ** 3)
    v = poisson.solve(gauss)
    np.testing.assert_allclose(v[::13], golden_arrays["he25_poisson_sub"], rtol=1e-12, atol=1e-14)
    step = scf.KohnShamStep(system, grid, factor, quad)
    n0 = scf.initial_density(step)
    np.testing.assert_allclose(n0[0, ::13], golden_arrays["he25_initial_density_sub"], rtol=1e-12)
    p = step.potentials(n0)
    _close([p["hartree_energy"], p["xc_energy"], p["xc_double_counting"]],
           [g["hartree_energy"], g["xc_energy"], g["xc_double_counting"]], 1e-12)
    np.testing.assert_allclose(p["effective"][::13], golden_arrays["he25_effective_sub"], rtol=1e-11, atol=1e-12)


@pytest.mark.parametrize("name", ["lda", "pbe"])
def test_xc_pointwise(name, golden_arrays):
    n, sigma = golden_arrays["xc_n"], golden_arrays["xc_sigma"]
    if name == "lda":
        e, v, _ = xc.evaluate("lda_vwn", n)
        pairs = [(e, "xc_lda_e"), (v, "xc_lda_v")]
    else:
        e, v, vs = xc.evaluate("pbe", n, sigma)
        pairs = [(e, "xc_pbe_e"), (v, "xc_pbe_v"), (vs, "xc_pbe_vs")]
    for got, key in pairs:
        want = golden_arrays[key]
        atol = 1e-300
        if key == "xc_pbe_vs":
            # v_sigma is the difference of an exchange and a correlation term that each scale as
            # n^(-4/3) and nearly cancel at small gradients; compare at the scale of either term.
            atol = 1e-12 * np.abs(n) ** (-4.0 / 3.0) * 0.75 * 0.2195 / (4 * 9.57)
        atol = np.where(np.isfinite(atol), atol, 0.0)
        bad = np.abs(got - want) > 1e-10 * np.abs(want) + atol
        assert not bad.any(), (key, n[bad][:5], got[bad][:5], want[bad][:5])


def test_reference_pins_h_atom(golden_values):
    """The reference's own golden pins: H at its production grid (box 32, h = 1)."""
    out = scf.solve_noninteracting(scf.h_atom(points_per_edge=33, half_box=16.0))
    pins = golden_values["reference_pins"]
    assert abs(out["eigenvalues"][0] - pins["eigenvalue.ground.h_atom"]) < 1e-9 * 0.5
    assert abs(out["kinetic"] - pins["kinetic.h_atom"]) < 1e-9 * 0.5


def test_reference_pins_checkerboard(golden_values):
    """``checkerboard.rayleigh.Z1/Z2`` of the reference's golden file (no quadrature, 13^3 box)."""
    pins = golden_values["reference_pins"]
    for z in (1.0, 2.0):
        grid = Grid.box((6.0, 6.0, 6.0), 0.5)
        factor = CuspFactor(grid, (z,), ((0.0, 0.0, 0.0),))
        ham = CuspHamiltonian(grid, factor, None)
        idx = np.indices(grid.shape).reshape(3, -1).sum(axis=0)
        alt = ((-1.0) ** idx)[None, :]
        alt = alt / ham.measure.norm(alt)[0]
        quotient = float(ham.measure.cross(alt, ham.apply(alt))[0, 0])
        assert abs(quotient - pins[f"checkerboard.rayleigh.Z{z:g}"]) < 1e-9 * abs(quotient)


def test_config1_h_atom(golden_values):
    out = scf.solve_noninteracting(scf.h_atom())
    ref = golden_values["h33_box8"]
    assert abs(out["total"] - ref["total"]) < 1e-12
    assert out["iterations"] == ref["iterations"]


def test_h2plus_small(golden_values):
    system = scf.h2_plus(2.0, spacing=0.4, transverse=10.0)
    system.box_lengths = (10.0, 10.0, 12.0)
    out = scf.solve_noninteracting(system)
    ref = golden_values["h2plus_R2_h04"]
    assert abs(out["total"] - ref["total"]) < 1e-11
    assert out["iterations"] == ref["iterations"]


def test_he25_scf(golden_values):
    out = scf.solve_self_consistent(scf.he_lda(spacing=0.5, edge=12.0))
    ref = golden_values["he25_lda_linear"]
    assert abs(out["energies"]["total"] - ref["total"]) < 1e-11
    assert out["scf_iterations"] == ref["iterations"]
