"""Derivatives of the path: hand-written vector-Jacobian products and energy gradients.

* ``CuspApply``: y = A phi with A = 0.5 (h^3/omega) Div + V and Div = sum_d D_d^T W_d D_d
  symmetric. The VJP is phi_bar = A^T y_bar = 0.5 Div((h^3/omega) y_bar) + V y_bar (one divergence
  launch), and V_bar = sum over orbitals of y_bar * phi.
* ``PoissonSolve``: v = G rho with G = E^T C E (zero-pad, circular convolution with the even kernel
  K(G), restrict) symmetric, so rho_bar = G v_bar (the same solve).
* ``XCEnergy``: E = sum_p w_p e_xc(n_p) at points; n_bar = E_bar w v_xc(n), from the kernels'
  analytic first derivatives (src/cdft/xc/base.py:158 differentiates the same energy by autograd).
* ``ChebyshevFilter``: Y = p(A) X. Since A^T = D^-1 A D with D = diag(h^3/omega), p(A)^T =
  D^-1 p(A) D and X_bar = (omega/h^3) p(A)((h^3/omega) Y_bar): the backward pass is one more
  forward filter, with no stored iterates (memory does not grow with the degree).

Energy gradients. An external perturbation dv = sum_k alpha_k g_k enters the operator as
quadrature.effective_potential(g_node, g_grid) (quadrature.py:747-753). Its first-order effect is
the expectation value Q[n g_k] through the cusp-aware quadrature (Hellmann--Feynman):
* for a bare-nucleus problem that is the exact derivative of the energy (first-order eigenvalue
  perturbation theory of an operator self-adjoint in the measure);
* for the self-consistent energy it is exact only where that energy is stationary. On the cusp
  quadrature the discrete Hartree potential (analytic cusp part plus grid Poisson, lifted to the
  nodes) is not the exact derivative of the discrete Hartree energy, so a first-order term remains:
  0.3% of the gradient for He at h = 0.5.
The derivative with respect to a nuclear position (``nuclear_gradient_variational``) follows from
the stationarity of the Kohn--Sham Lagrangian at the converged orbitals (Hellmann--Feynman plus the
Pulay terms of the cusp factor, face weights, quadrature and measure that move with the nucleus):
no orbital response, no re-solve; the explicit geometry derivative is a central difference of the
device geometry build at fixed orbitals. ``nuclear_gradient`` (central differences of converged
total energies on a fixed, unanchored grid) is the check.
"""

from __future__ import annotations

import numpy as np
import torch

from .operators import weighted_divergence
from .xc import functional_by_name


# ---------------------------------------------------------------------------------------- VJPs
class CuspApply(torch.autograd.Function):
    """``A phi`` with a differentiable orbital block and diagonal potential (float64)."""

    @staticmethod
    def forward(ctx, phi: torch.Tensor, potential: torch.Tensor, hamiltonian) -> torch.Tensor:
        ctx.hamiltonian = hamiltonian
        ctx.save_for_backward(phi, potential)
        return hamiltonian.apply_with_potential(phi, potential)

    @staticmethod
    def backward(ctx, y_bar: torch.Tensor):
        phi, potential = ctx.saved_tensors
        h = ctx.hamiltonian
        grid = h.grid
        n = grid.n_points
        y = y_bar.contiguous()
        scaled = (h._inverse_weight * y).reshape(-1, *grid.shape)
        div = weighted_divergence(scaled, h.factor.face_weights(grid.fd_order), grid.spacing, grid.fd_order,
                                  grid.shape).reshape(y.shape)
        phi_bar = 0.5 * div + potential * y
        potential_bar = (y * phi).reshape(-1, n).sum(dim=0)
        return phi_bar, potential_bar, None


class PoissonSolve(torch.autograd.Function):
    """``v_H`` of a total density through :class:`CoulombCutoffPoisson` (linear and symmetric)."""

    @staticmethod
    def forward(ctx, density: torch.Tensor, solver) -> torch.Tensor:
        ctx.solver = solver
        return solver.solve(density)

    @staticmethod
    def backward(ctx, v_bar: torch.Tensor):
        return ctx.solver.solve(v_bar.contiguous()), None


class XCEnergy(torch.autograd.Function):
    """``sum_p w_p e_xc(n_p)`` for a spin-restricted LDA density at points (e_xc per volume)."""

    @staticmethod
    def forward(ctx, density: torch.Tensor, weights: torch.Tensor, functional: str) -> torch.Tensor:
        out = functional_by_name(functional).evaluate(density[None, :].to(torch.float64))
        ctx.save_for_backward(weights, out.v_xc[0])
        return (weights * out.e_xc.reshape(-1)).sum()

    @staticmethod
    def backward(ctx, e_bar: torch.Tensor):
        weights, v_xc = ctx.saved_tensors
        return e_bar * weights * v_xc, None, None


class ChebyshevFilter(torch.autograd.Function):
    """The fused filter ``p(A) X`` with the exact transpose as its backward pass."""

    @staticmethod
    def forward(ctx, block: torch.Tensor, hamiltonian, degree: int, lower: float, upper: float,
                spectrum_min: float) -> torch.Tensor:
        from .eigen import chebyshev_filter

        ctx.args = (hamiltonian, degree, lower, upper, spectrum_min)
        return chebyshev_filter(hamiltonian, block, degree, lower, upper, spectrum_min)

    @staticmethod
    def backward(ctx, y_bar: torch.Tensor):
        from .eigen import chebyshev_filter

        hamiltonian, degree, lower, upper, spectrum_min = ctx.args
        d = hamiltonian._inverse_weight
        x = chebyshev_filter(hamiltonian, (d * y_bar).contiguous(), degree, lower, upper, spectrum_min)
        return x / d, None, None, None, None, None


# --------------------------------------------------------------------- external perturbation
def seeded_gaussians(seed: int = 2024, count: int = 8, half_extent: float = 3.0):
    """Centres U[-half_extent, half_extent]^3, widths U[0.5, 1.5] bohr, amplitudes N(0, 1e-3) Ha."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(-half_extent, half_extent, size=(count, 3))
    widths = rng.uniform(0.5, 1.5, size=count)
    amplitudes = rng.normal(0.0, 1.0e-3, size=count)
    return centres, widths, amplitudes


def gaussian_values(points: torch.Tensor, centres, widths) -> torch.Tensor:
    """``g_k(r) = exp(-|r - c_k|^2 / (2 w_k^2))`` at ``points (P, 3)``: ``(k, P)``."""
    c = torch.as_tensor(np.asarray(centres), dtype=torch.float64, device=points.device)
    w = torch.as_tensor(np.asarray(widths), dtype=torch.float64, device=points.device)
    d2 = ((points[None, :, :] - c[:, None, :]) ** 2).sum(dim=-1)
    return torch.exp(-d2 / (2.0 * w[:, None] ** 2))


def perturbation_fields(geometry, centres, widths):
    """``(g_node (k, M), g_grid (k, N))`` of the Gaussians at the quadrature nodes and grid points."""
    q = geometry.quadrature
    return gaussian_values(q.points, centres, widths), gaussian_values(geometry.grid.points(), centres, widths)


def effective_perturbation(geometry, g_node: torch.Tensor, g_grid: torch.Tensor) -> torch.Tensor:
    """``quadrature.effective_potential`` (quadrature.py:747-753) of each field: ``(k, N)``."""
    q = geometry.quadrature
    f2_grid = geometry.factor.weight
    out = [q.lumped_weights(g_node[k] * q.f2, g_grid[k] * f2_grid) / q.mass_weights for k in range(g_node.shape[0])]
    return torch.stack(out)


def external_potential_gradient(geometry, density: torch.Tensor, g_node: torch.Tensor,
                                g_grid: torch.Tensor) -> torch.Tensor:
    """``dE/d alpha_k = Q[n g_k]`` at a converged density ``(1, N)`` or ``(N,)``: ``(k,)``."""
    n_grid = density.reshape(-1).to(torch.float64)
    rho = n_grid / geometry.factor.weight
    dv = effective_perturbation(geometry, g_node, g_grid)
    return (dv * (geometry.quadrature.mass_weights * rho)[None, :]).sum(dim=1)


def orbital_potential_gradient(geometry, orbitals: torch.Tensor, occupations: torch.Tensor, g_node: torch.Tensor,
                               g_grid: torch.Tensor) -> torch.Tensor:
    """``dE/d alpha_k = sum_i f_i <psi_i| dv_k |psi_i>`` (measure-normalised orbitals): ``(k,)``.

    For a bare-nucleus problem this is first-order eigenvalue perturbation theory, exact because the
    operator is self-adjoint in the measure.
    """
    rho = (occupations.reshape(-1, 1) * orbitals.to(torch.float64) ** 2).sum(dim=0)
    dv = effective_perturbation(geometry, g_node, g_grid)
    return (dv * (geometry.quadrature.mass_weights * rho)[None, :]).sum(dim=1)


def nuclear_gradient(energy_at, positions, delta: float = 1.0e-4) -> np.ndarray:
    """Central differences ``(E(R + d e) - E(R - d e)) / 2d`` per nucleus and axis.

    ``energy_at(positions)`` returns the converged total energy with the nuclei at ``positions``
    (the grid stays fixed: it is not re-anchored to the nuclei).
    """
    base = np.asarray(positions, dtype=float)
    grad = np.zeros_like(base)
    for a in range(base.shape[0]):
        for d in range(3):
            plus, minus = base.copy(), base.copy()
            plus[a, d] += delta
            minus[a, d] -= delta
            grad[a, d] = (energy_at(plus) - energy_at(minus)) / (2.0 * delta)
    return grad


# ------------------------------------------------------------------------ nuclear gradient


def fixed_orbital_energy(geometry, orbitals: torch.Tensor, occupations: torch.Tensor, eigenvalues: torch.Tensor,
                         functional: str | None = None, n_electrons: float | None = None) -> float:
    """The Kohn--Sham Lagrangian at fixed transformed orbitals ``phi`` on ``geometry``:

        L = sum_i f_i <phi_i, A_bare phi_i>_q + E_H[n] + E_xc[n] + E_ion - sum_i f_i eps_i (<phi_i, phi_i>_q - 1)

    with ``n = f^2 sum_i f_i phi_i^2`` and every geometric quantity (face weights, ``h^3/omega``,
    ``W~/omega``, the measure ``q``, the cusp factor, the quadrature) that of ``geometry``. At the
    geometry the orbitals were solved on, L is the total energy (``band - double counting + E_H +
    E_xc + E_ion``, ``src/cdft/scf/step.py:398-439``); ``functional=None`` is the bare-nucleus energy
    (band + E_ion, ``src/cdft/scf/noninteracting.py``).
    """
    from .operators import CuspFactoredHamiltonian
    from .scf import KohnShamStep, nuclear_repulsion

    phi = orbitals.to(torch.float64).reshape(-1, geometry.grid.n_points)
    occ = occupations.to(device=phi.device, dtype=torch.float64).reshape(-1)
    eps = eigenvalues.to(device=phi.device, dtype=torch.float64).reshape(-1)
    ham = CuspFactoredHamiltonian(geometry.grid, geometry.factor, quadrature=geometry.quadrature)
    q = ham.measure.quadrature
    a_phi = ham.apply(phi)
    form = (q[None] * phi * a_phi).sum(dim=1)
    norm = (q[None] * phi * phi).sum(dim=1)
    value = (occ * (form - eps * (norm - 1.0))).sum()
    total = float(value) + nuclear_repulsion(geometry.charges, geometry.positions)
    if functional is not None:
        rho = (occ[:, None] * phi * phi).sum(dim=0)
        n_grid = (rho * geometry.factor.weight)[None]
        step = KohnShamStep(geometry, functional, float(n_electrons if n_electrons is not None else occ.sum()))
        p = step.potentials(n_grid)
        total += float(p.hartree_energy) + float(p.xc_energy)
    return total


def nuclear_gradient_variational(build, positions, orbitals: torch.Tensor, occupations: torch.Tensor,
                                 eigenvalues: torch.Tensor, functional: str | None = None,
                                 n_electrons: float | None = None, delta: float = 1.0e-4,
                                 components=None) -> np.ndarray:
    """``dE/dR_a`` from the stationarity of the Kohn--Sham Lagrangian (Hellmann--Feynman with the
    Pulay terms of the moving cusp factor, quadrature and measure): ``dE/dR = dL/dR`` at the
    converged orbitals, so no orbital response and no re-solve. The explicit geometry derivative of
    :func:`fixed_orbital_energy` is taken by central differences of the device geometry build
    (``build(positions) -> CuspGeometry``, 6 builds per nucleus), at fixed orbitals, multipliers and
    grid (the grid is not re-anchored to the moved nuclei).

    Exact for a bare-nucleus problem (the eigenvalue derivative of an operator self-adjoint in the
    measure). For the self-consistent energy it carries the first-order error of the discrete
    Hartree potential's non-stationarity noted in the module docstring, which vanishes as the grid
    refines. ``components`` (pairs ``(nucleus, axis)``) limits the work to those entries; the
    others are returned as zero.
    """
    base = np.asarray(positions, dtype=float)
    grad = np.zeros_like(base)
    todo = components if components is not None else [(a, d) for a in range(base.shape[0]) for d in range(3)]
    for a, d in todo:
        values = []
        for sign in (+1.0, -1.0):
            moved = base.copy()
            moved[a, d] += sign * delta
            geo = build([tuple(p) for p in moved])
            values.append(fixed_orbital_energy(geo, orbitals, occupations, eigenvalues, functional, n_electrons))
        grad[a, d] = (values[0] - values[1]) / (2.0 * delta)
    return grad
