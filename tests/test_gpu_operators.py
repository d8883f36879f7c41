"""GPU parity of the apply, filter, reductions, Rayleigh--Ritz and Lanczos kernels against the oracle.

Geometry for these unit tests comes from the oracle (uploaded once); the product's own device
geometry is tested in ``test_gpu_geometry.py``. Tolerances: float64 kernels re-associate sums, so
agreement is to ~1e-13 relative of the field's scale; float32 kernels to ~1e-5.
"""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import eigen as oeigen
from oracle import scf as oscf
from oracle.operators import CuspHamiltonian, lanczos_bounds
from oracle.rng import make_generator

pytestmark = pytest.mark.gpu


def _t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.fixture(scope="module")
def he25(pkg, cuda):
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    grid_o, factor_o, quad_o = oscf.build_geometry(system)
    ham_o = CuspHamiltonian(grid_o, factor_o, quad_o)
    grid = pkg.UniformGrid(grid_o.shape, grid_o.spacing, grid_o.origin, device=cuda)
    faces = tuple(_t(w, cuda) for w in factor_o.face_weights(8))
    pot, inv, q = quad_o.bare_operator_terms()
    factor = SimpleNamespace(face_weights=lambda acc: faces)
    measure = pkg.Measure(grid, _t(q, cuda))
    bare = (_t(pot, cuda), _t(inv, cuda), measure)
    ham = pkg.CuspFactoredHamiltonian(grid, factor, bare=bare)
    return SimpleNamespace(grid_o=grid_o, ham_o=ham_o, grid=grid, ham=ham, bare=bare, factor=factor, q=q)


def test_weighted_divergence_matches_reference(pkg, cuda, golden_arrays):
    box = _t(golden_arrays["div_box"], cuda)
    faces = [_t(golden_arrays[f"div_w{a}"], cuda) for a in range(3)]
    out = pkg.weighted_divergence(box, faces, 0.37, 8, (9, 11, 13)).cpu().numpy()
    want = golden_arrays["div_out"]
    np.testing.assert_allclose(out, want, rtol=0, atol=1e-13 * np.abs(want).max())


@pytest.mark.parametrize("accuracy", [2, 4, 6, 8])
def test_weighted_divergence_orders(pkg, cuda, accuracy):
    from oracle.grid import weighted_divergence

    g = torch.Generator().manual_seed(accuracy)
    shape = (19, 23, 41)
    box = torch.randn((3, *shape), dtype=torch.float64, generator=g)
    faces = []
    for axis in range(3):
        sizes = list(shape)
        sizes[axis] += accuracy
        faces.append(0.1 + torch.rand(sizes, dtype=torch.float64, generator=g))
    want = weighted_divergence(box.numpy(), [f.numpy() for f in faces], 0.3, accuracy)
    got = pkg.weighted_divergence(box.to(cuda), [f.to(cuda) for f in faces], 0.3, accuracy, shape).cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-13 * np.abs(want).max())


def test_apply_f64(he25, cuda):
    g = torch.Generator().manual_seed(11)
    block = torch.randn((5, he25.grid.n_points), dtype=torch.float64, generator=g)
    want = he25.ham_o.apply(block.numpy())
    got = he25.ham.apply(block.to(cuda)).cpu().numpy()
    scale = np.abs(want).max()
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-13 * scale)
    kin_want = he25.ham_o.kinetic_apply(block.numpy())
    kin_got = he25.ham.kinetic_apply(block.to(cuda)).cpu().numpy()
    np.testing.assert_allclose(kin_got, kin_want, rtol=0, atol=1e-13 * np.abs(kin_want).max())
    assert he25.ham.apply_count == 1


def test_apply_f32(pkg, he25, cuda):
    ham32 = pkg.CuspFactoredHamiltonian(he25.grid, he25.factor, bare=he25.bare, dtype=torch.float32)
    g = torch.Generator().manual_seed(12)
    block = torch.randn((5, he25.grid.n_points), dtype=torch.float64, generator=g)
    want = he25.ham_o.apply(block.numpy())
    got = ham32.apply(block.to(cuda).float()).double().cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=0, atol=2e-5 * np.abs(want).max())


def test_measure_cross(pkg, he25, cuda):
    g = torch.Generator().manual_seed(13)
    a = torch.randn((5, he25.grid.n_points), dtype=torch.float64, generator=g)
    b = torch.randn((7, he25.grid.n_points), dtype=torch.float64, generator=g)
    q = he25.q
    want = (a.numpy() * q) @ b.numpy().T
    got = he25.ham.measure.cross(a.to(cuda), b.to(cuda)).cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13 * np.abs(want).max())
    inner = he25.ham.measure.inner(a.to(cuda), a.to(cuda)).cpu().numpy()
    np.testing.assert_allclose(inner, (a.numpy() ** 2 * q).sum(axis=-1), rtol=1e-13)
    # groups of different shapes: 9 x 9 tiles
    c = torch.randn((9, he25.grid.n_points), dtype=torch.float64, generator=g)
    got9 = he25.ham.measure.gram(c.to(cuda)).cpu().numpy()
    np.testing.assert_allclose(got9, (c.numpy() * q) @ c.numpy().T, rtol=1e-12, atol=1e-12)


def test_filter_f64_matches_oracle(pkg, he25, cuda, golden_values):
    g = torch.Generator().manual_seed(11)
    block = torch.randn((5, he25.grid.n_points), dtype=torch.float64, generator=g)
    deg, lower, upper, smin = golden_values["he25"]["filter_args"]
    want = oeigen.chebyshev_filter(he25.ham_o, block.numpy(), deg, lower, upper, smin)
    got = pkg.chebyshev_filter(he25.ham, block.to(cuda), deg, lower, upper, smin).cpu().numpy()
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-11 * np.abs(want).max())


def test_filter_f32(pkg, he25, cuda, golden_values):
    ham32 = pkg.CuspFactoredHamiltonian(he25.grid, he25.factor, bare=he25.bare, dtype=torch.float32)
    g = torch.Generator().manual_seed(11)
    block = torch.randn((5, he25.grid.n_points), dtype=torch.float64, generator=g)
    deg, lower, upper, smin = golden_values["he25"]["filter_args"]
    want = oeigen.chebyshev_filter(he25.ham_o, block.numpy(), deg, lower, upper, smin)
    got = pkg.chebyshev_filter(ham32, block.to(cuda), deg, lower, upper, smin).cpu().numpy()
    assert got.dtype == np.float64
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-4 * np.abs(want).max())


def test_rayleigh_ritz_and_residuals(pkg, he25, cuda, golden_values):
    g = torch.Generator().manual_seed(11)
    block = torch.randn((5, he25.grid.n_points), dtype=torch.float64, generator=g)
    evals, vectors, orth = pkg.rayleigh_ritz(he25.ham, block.to(cuda), he25.ham.measure)
    want = np.array(golden_values["he25"]["rr_evals"])
    np.testing.assert_allclose(evals.cpu().numpy(), want, rtol=1e-11, atol=1e-11)
    assert orth < 1e-12
    res = pkg.residual_norms(he25.ham, evals, vectors, he25.ham.measure).cpu().numpy()
    np.testing.assert_allclose(res, np.array(golden_values["he25"]["rr_residuals"]), rtol=1e-9)


def test_lanczos_bounds(pkg, he25, cuda, golden_values):
    lo, hi = he25.ham.spectral_bounds(generator=make_generator(0))
    want = golden_values["he25"]["lanczos_bounds"]
    np.testing.assert_allclose([lo, hi], want, rtol=1e-10)


def test_chefsi_h_atom_config1(pkg, cuda, golden_values):
    """Config 1 (bare H, 33^3, box 8) with the native CheFSI on oracle geometry: E to 1e-12 Ha."""
    system = oscf.h_atom()
    grid_o, factor_o, quad_o = oscf.build_geometry(system)
    grid = pkg.UniformGrid(grid_o.shape, grid_o.spacing, grid_o.origin, device=cuda)
    faces = tuple(_t(w, cuda) for w in factor_o.face_weights(8))
    pot, inv, q = quad_o.bare_operator_terms()
    bare = (_t(pot, cuda), _t(inv, cuda), pkg.Measure(grid, _t(q, cuda)))
    ham = pkg.CuspFactoredHamiltonian(grid, SimpleNamespace(face_weights=lambda acc: faces), bare=bare)
    solver = pkg.ChebyshevFilteredSubspace(grid, pkg.EigenConfig(), ritz_stop=True)
    result = solver.solve(ham, 1, generator=make_generator(0))
    ref = golden_values["h33_box8"]
    assert abs(float(result.eigenvalues[0]) - ref["eigenvalues"][0]) < 1e-12
    assert result.n_iterations == ref["iterations"]
    assert result.converged
