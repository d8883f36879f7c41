"""The hand-written adjoints (apply, Poisson, XC, filter) and the energy gradients.

Each VJP is checked by its defining identity or by central differences. The Hellmann--Feynman
gradient of the self-consistent energy with respect to a seeded Gaussian external perturbation is
checked against central differences of total energies (step 1e-4 Ha) and against the same quantity
from the reference's own converged density; the nuclear (bond-length) gradient of H2+ by central
differences is checked against the reference's (both from tests/golden, --with-adjoint).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import scf as oscf

pytestmark = pytest.mark.gpu


def _geometry(pkg, system, dev):
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=dev)
    return pkg.build_cusp_geometry(grid, system.charges, system.positions)


@pytest.fixture(scope="module")
def he25(pkg, cuda):
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    return system, _geometry(pkg, system, cuda)


def _rand(shape, seed, dev):
    g = torch.Generator().manual_seed(seed)
    return torch.randn(shape, dtype=torch.float64, generator=g).to(dev)


def test_apply_vjp_is_the_transpose(pkg, he25, cuda):
    _, geo = he25
    ham = pkg.CuspFactoredHamiltonian(geo.grid, geo.factor, quadrature=geo.quadrature)
    n = geo.grid.n_points
    phi = _rand((2, n), 1, cuda).requires_grad_(True)
    pot = (ham.graph_potential() + 0.1 * _rand((n,), 2, cuda)).requires_grad_(True)
    y_bar = _rand((2, n), 3, cuda)
    y = pkg.adjoint.CuspApply.apply(phi, pot, ham)
    (y * y_bar).sum().backward()
    # the bilinear form is exact under central differences
    d_phi, d_pot = _rand((2, n), 4, cuda), _rand((n,), 5, cuda)
    eps = 1e-3
    with torch.no_grad():
        plus = (ham.apply_with_potential(phi + eps * d_phi, pot + eps * d_pot) * y_bar).sum()
        minus = (ham.apply_with_potential(phi - eps * d_phi, pot - eps * d_pot) * y_bar).sum()
    fd = float((plus - minus) / (2 * eps))
    ad = float((phi.grad * d_phi).sum() + (pot.grad * d_pot).sum())
    assert abs(fd - ad) <= 1e-9 * abs(ad)


def test_poisson_is_symmetric(pkg, he25, cuda):
    _, geo = he25
    solver = pkg.CoulombCutoffPoisson(geo.grid, pad_factor=2.5)
    n = geo.grid.n_points
    u, v = _rand((n,), 6, cuda), _rand((n,), 7, cuda)
    lhs = float((u * solver.solve(v)).sum())
    rhs = float((solver.solve(u) * v).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    rho = v.clone().requires_grad_(True)
    (pkg.adjoint.PoissonSolve.apply(rho, solver) * u).sum().backward()
    want = solver.solve(u)
    torch.testing.assert_close(rho.grad, want, rtol=0, atol=1e-14 * float(want.abs().max()))


def test_xc_energy_vjp_central_differences(pkg, cuda):
    p = 4096
    g = torch.Generator().manual_seed(8)
    n = (0.01 + torch.rand(p, dtype=torch.float64, generator=g) * 2.0).to(cuda).requires_grad_(True)
    w = (0.5 + torch.rand(p, dtype=torch.float64, generator=g)).to(cuda)
    e = pkg.adjoint.XCEnergy.apply(n, w, "lda_vwn")
    e.backward()
    dn = _rand((p,), 9, cuda) * 1e-2
    eps = 1e-4
    with torch.no_grad():
        fd = (pkg.adjoint.XCEnergy.apply(n + eps * dn, w, "lda_vwn") -
              pkg.adjoint.XCEnergy.apply(n - eps * dn, w, "lda_vwn")) / (2 * eps)
    ad = (n.grad * dn).sum()
    assert abs(float(fd - ad)) <= 1e-6 * abs(float(ad))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_filter_vjp_is_the_transpose(pkg, he25, cuda, dtype):
    _, geo = he25
    ham = pkg.CuspFactoredHamiltonian(geo.grid, geo.factor, quadrature=geo.quadrature, dtype=dtype)
    n = geo.grid.n_points
    x = _rand((3, n), 10, cuda).requires_grad_(True)
    y_bar = _rand((3, n), 11, cuda)
    y = pkg.adjoint.ChebyshevFilter.apply(x, ham, 8, 2.0, 60.0, -3.0)
    (y * y_bar).sum().backward()
    lhs = float((y.detach() * y_bar).sum())
    rhs = float((x.grad * x.detach()).sum())
    tol = 1e-10 if dtype == torch.float64 else 1e-4
    assert abs(lhs - rhs) <= tol * abs(lhs)


def test_composed_gradient_central_differences(pkg, he25, cuda):
    """The VJPs composed into one end-to-end gradient: a scalar through the filter, the apply, the
    Poisson solve and the XC energy, E(phi, alpha) = <Y, A(V0 + alpha g) Y> + (1/2) <rho, G rho> h^3
    + E_xc[rho + 0.01] with Y = p(A) phi and rho = sum of Y^2, differentiated by autograd through
    the hand-written backward passes, against central differences along a random direction in
    (phi, alpha), to 1e-7 relative."""
    _, geo = he25
    ham = pkg.CuspFactoredHamiltonian(geo.grid, geo.factor, quadrature=geo.quadrature)
    solver = pkg.CoulombCutoffPoisson(geo.grid, pad_factor=2.5)
    n = geo.grid.n_points
    h3 = geo.grid.spacing ** 3
    v0 = ham.graph_potential()
    g = torch.exp(-(geo.grid.points() ** 2).sum(dim=1) / 4.0)  # a smooth external perturbation
    w = torch.full((n,), h3, dtype=torch.float64, device=cuda)
    phi0 = _rand((2, n), 21, cuda)
    phi0 = phi0 / phi0.norm(dim=1, keepdim=True)

    def energy(phi, alpha):
        y = pkg.adjoint.ChebyshevFilter.apply(phi, ham, 4, 2.0, 60.0, -3.0)
        ay = pkg.adjoint.CuspApply.apply(y, v0 + alpha * g, ham)
        rho = (y * y).sum(dim=0)
        e_band = (y * ay).sum()
        e_h = 0.5 * (rho * pkg.adjoint.PoissonSolve.apply(rho, solver)).sum() * h3
        e_xc = pkg.adjoint.XCEnergy.apply(rho + 0.01, w, "lda_vwn")
        return e_band + e_h + e_xc

    phi = phi0.clone().requires_grad_(True)
    alpha = torch.tensor(0.05, dtype=torch.float64, device=cuda, requires_grad=True)
    energy(phi, alpha).backward()
    d_phi, d_alpha = _rand((2, n), 22, cuda) * 1e-2, 0.3
    eps = 1e-4
    with torch.no_grad():
        plus = energy(phi0 + eps * d_phi, alpha.detach() + eps * d_alpha)
        minus = energy(phi0 - eps * d_phi, alpha.detach() - eps * d_alpha)
    fd = float((plus - minus) / (2 * eps))
    ad = float((phi.grad * d_phi).sum() + alpha.grad * d_alpha)
    assert abs(ad) > 1e-6
    assert abs(fd - ad) <= 1e-7 * abs(ad), (fd, ad)


def _solve(pkg, step, tight=True):
    scf = pkg.SCFConfig(energy_tol=1e-11, density_tol=1e-8, max_iterations=400) if tight else None
    out = pkg.solve_self_consistent(step, pkg.MixingConfig(scheme="linear", alpha=0.3), scf)
    assert out.converged
    return out


def test_seeded_gaussians_match_the_reference_harness(pkg, golden_values):
    ref = golden_values.get("he25_external_gradient")
    if ref is None:
        pytest.skip("no reference gradient fixture (make_golden.py --with-adjoint)")
    centres, widths, _ = pkg.adjoint.seeded_gaussians()
    np.testing.assert_array_equal(centres, np.array(ref["centres"]))
    np.testing.assert_array_equal(widths, np.array(ref["widths"]))


def test_bare_nucleus_perturbation_gradient(pkg, cuda):
    """Config 1's H atom: dE/d alpha = <psi|dv|psi> against central differences to 1e-6."""
    system = oscf.h_atom()
    geo = _geometry(pkg, system, cuda)
    centres, widths, _ = pkg.adjoint.seeded_gaussians()
    g_node, g_grid = pkg.adjoint.perturbation_fields(geo, centres, widths)
    dv = pkg.adjoint.effective_perturbation(geo, g_node, g_grid)
    # eigenvalues to ~1e-14 Ha, so that the differences resolve the derivative to 1e-6
    eigen = pkg.EigenConfig(residual_tol=1e-12, cross_check_tol=1e-13, max_iterations=600)
    base = pkg.solve_noninteracting(geo, n_electrons=1.0, eigen=eigen)
    grad = pkg.adjoint.orbital_potential_gradient(geo, base["orbitals"], base["occupations"], g_node,
                                                  g_grid).cpu().numpy()
    step = 1e-4
    for k in range(8):
        plus = pkg.solve_noninteracting(geo, n_electrons=1.0, eigen=eigen, external_potential=step * dv[k])["total"]
        minus = pkg.solve_noninteracting(geo, n_electrons=1.0, eigen=eigen,
                                         external_potential=-step * dv[k])["total"]
        fd = (plus - minus) / (2 * step)
        assert abs(fd - grad[k]) <= 1e-6 * abs(grad[k]) + 1e-10, (k, fd, grad[k])


def test_external_perturbation_gradient(pkg, he25, golden_values):
    system, geo = he25
    centres, widths, _ = pkg.adjoint.seeded_gaussians()
    g_node, g_grid = pkg.adjoint.perturbation_fields(geo, centres, widths)
    dv = pkg.adjoint.effective_perturbation(geo, g_node, g_grid)
    # against the reference's Hellmann--Feynman value (same SCF settings as its run)
    ref = golden_values.get("he25_external_gradient")
    if ref is not None:
        plain = _solve(pkg, pkg.KohnShamStep(geo, "lda_vwn", system.n_electrons), tight=False)
        got = pkg.adjoint.external_potential_gradient(geo, plain.density, g_node, g_grid).cpu().numpy()
        np.testing.assert_allclose(got, np.array(ref["hellmann_feynman"]), rtol=1e-9, atol=1e-12)
    # against central differences of tightly converged total energies
    base = _solve(pkg, pkg.KohnShamStep(geo, "lda_vwn", system.n_electrons))
    grad = pkg.adjoint.external_potential_gradient(geo, base.density, g_node, g_grid).cpu().numpy()
    assert np.all(np.isfinite(grad)) and np.abs(grad).max() > 1e-4
    step = 1e-4
    for k in (0, 3, 6):
        e = []
        for sign in (+1, -1):
            out = _solve(pkg, pkg.KohnShamStep(geo, "lda_vwn", system.n_electrons,
                                               external_potential=sign * step * dv[k]))
            e.append(float(out.energies["total"]))
        fd = (e[0] - e[1]) / (2 * step)
        # The self-consistent energy on the cusp quadrature is not exactly stationary: the discrete
        # Hartree potential is not the exact derivative of the discrete Hartree energy, so the
        # expectation value misses a first-order term (0.3% at h = 0.5 for He).
        assert abs(fd - grad[k]) <= 5e-3 * abs(grad[k]) + 1e-9, (k, fd, grad[k])


def test_h2plus_bond_derivative(pkg, cuda, golden_values):
    """dE/dR of H2+ (R = 2, h = 0.4, fixed grid) by central differences, as the reference takes it."""
    energies = {}

    def energy(bond):
        system = oscf.h2_plus(bond, spacing=0.4, transverse=10.0)
        system.box_lengths = (10.0, 10.0, 12.0)  # the R = 2 box for every displacement: one grid
        return float(pkg.solve_noninteracting(_geometry(pkg, system, cuda), n_electrons=1.0)["total"])

    for sign in (+1, -1):
        energies[sign] = energy(2.0 + sign * 1e-4)
    derivative = (energies[1] - energies[-1]) / 2e-4
    assert np.isfinite(derivative) and abs(derivative) < 1.0
    ref = golden_values.get("h2plus_R2_h04_bond_derivative")
    if ref is not None:
        assert abs(energies[1] - ref["plus"]) < 1e-11 and abs(energies[-1] - ref["minus"]) < 1e-11
        assert abs(derivative - ref["derivative"]) < 1e-7


def test_config5_external_gradient_101(pkg, cuda):
    """Config 5 at its own size (He-LDA, h = 0.16, box 16, 101^3, float64): the gradient with respect to
    the seeded Gaussian perturbation against central differences (step 1e-4) on its three largest
    components, to 1e-6 relative."""
    system = oscf.he_lda(spacing=0.16, edge=16.0)
    geo = _geometry(pkg, system, cuda)
    assert geo.grid.shape == (101, 101, 101)
    centres, widths, _ = pkg.adjoint.seeded_gaussians()
    g_node, g_grid = pkg.adjoint.perturbation_fields(geo, centres, widths)
    dv = pkg.adjoint.effective_perturbation(geo, g_node, g_grid)
    base = _solve(pkg, pkg.KohnShamStep(geo, "lda_vwn", system.n_electrons))
    grad = pkg.adjoint.external_potential_gradient(geo, base.density, g_node, g_grid).cpu().numpy()
    step = 1e-4
    for k in np.argsort(-np.abs(grad))[:3]:
        e = [float(_solve(pkg, pkg.KohnShamStep(geo, "lda_vwn", system.n_electrons,
                                                external_potential=sign * step * dv[k])).energies["total"])
             for sign in (+1, -1)]
        fd = (e[0] - e[1]) / (2 * step)
        assert abs(fd - grad[k]) <= 1e-6 * abs(grad[k]), (int(k), fd, grad[k])


def _scan_system(bond, spacing=0.4):
    system = oscf.h2_plus(bond, spacing=spacing, transverse=10.0)
    system.box_lengths = (10.0, 10.0, 12.6)  # one fixed grid for every displacement
    return system


def test_variational_nuclear_gradient_bare_h2plus(pkg, cuda):
    """dE/dR_a of H2+ (R = 2.6, h = 0.4) from the stationarity of the Lagrangian at the converged
    orbital (no re-solve) against central differences of converged energies (step 1e-4), to 1e-6
    relative on the bond axis and to 1e-6 of it on every other component. The grid is not symmetric
    about the bond axis (26 points per transverse edge with the nuclei on a lattice line: 12 on one
    side, 13 on the other), so the transverse components are small but not zero."""
    system = _scan_system(2.6)
    eigen = pkg.EigenConfig(residual_tol=1e-12)
    geo = _geometry(pkg, system, cuda)
    out = pkg.solve_noninteracting(geo, n_electrons=1.0, eigen=eigen)
    assert out["converged"]
    grid = geo.grid

    def build(positions):
        return pkg.build_cusp_geometry(grid, system.charges, positions)

    grad = pkg.adjoint.nuclear_gradient_variational(build, system.positions, out["orbitals"], out["occupations"],
                                                    torch.tensor(out["eigenvalues"][:1], dtype=torch.float64))

    def energy_at(positions):
        res = pkg.solve_noninteracting(build([tuple(p) for p in positions]), n_electrons=1.0, eigen=eigen)
        return float(res["total"])

    fd = pkg.adjoint.nuclear_gradient(energy_at, system.positions, delta=1e-4)
    assert abs(grad[1, 2]) > 1e-3
    np.testing.assert_allclose(grad[:, 2], fd[:, 2], rtol=1e-6, atol=0)
    np.testing.assert_allclose(grad, fd, rtol=0, atol=1e-6 * abs(grad[1, 2]))
    assert np.abs(grad[:, :2]).max() < 1e-2 * abs(grad[1, 2])  # small off the axis


def test_variational_nuclear_gradient_interacting(pkg, cuda):
    """The self-consistent H2 molecule (LDA, R = 2.0, h = 0.4, fixed grid): the Lagrangian equals the
    converged total energy at the solved geometry, and its bond derivative is checked against
    central differences of tightly converged SCF energies. The discrete Hartree potential's
    non-stationarity leaves a first-order gap at this coarse grid, stated in the tolerance."""
    bond = 2.0

    def system_at(b):
        s = oscf.h2_pbe(bond=b, spacing=0.4, box=(9.0, 9.0, 11.0))
        s.functional = "lda_vwn"
        return s

    system = system_at(bond)
    geo = _geometry(pkg, system, cuda)
    grid = geo.grid
    scf = pkg.SCFConfig(energy_tol=1e-12, density_tol=1e-9, max_iterations=300)
    mixing = pkg.MixingConfig(scheme="linear", alpha=0.3)
    eigen = pkg.EigenConfig(residual_tol=1e-11)

    def build(positions):
        return pkg.build_cusp_geometry(grid, system.charges, positions)

    def solve(g):
        out = pkg.solve_self_consistent(pkg.KohnShamStep(g, "lda_vwn", 2.0, eigen), mixing, scf)
        assert out.converged
        return out

    base = solve(geo)
    step = pkg.KohnShamStep(geo, "lda_vwn", 2.0, eigen)
    p_in = step.potentials(base.density)
    eig, _ = step.diagonalise(step.hamiltonian(p_in))
    occ = step.occupy(eig.eigenvalues)
    lagrangian = pkg.adjoint.fixed_orbital_energy(geo, eig.eigenvectors, occ[0], eig.eigenvalues, "lda_vwn", 2.0)
    assert abs(lagrangian - base.energies["total"]) < 1e-8
    grad = pkg.adjoint.nuclear_gradient_variational(build, system.positions, eig.eigenvectors, occ[0],
                                                    eig.eigenvalues, functional="lda_vwn", n_electrons=2.0,
                                                    components=[(0, 2), (1, 2)])
    variational = 0.5 * (grad[1, 2] - grad[0, 2])
    h = 1e-4
    e = [float(solve(build(system_at(bond + s * h).positions)).energies["total"]) for s in (+1, -1)]
    central = (e[0] - e[1]) / (2 * h)
    print(f"H2 LDA bond derivative: variational {variational:.8f}, central differences {central:.8f}")
    assert abs(central) > 1e-2
    assert abs(variational - central) < 3e-2 * abs(central)
