"""The Kohn--Sham step, the SCF driver and the non-interacting solve on the device.

Host mirror of ``src/cdft/scf/step.py`` (KohnShamStep: potentials, hamiltonian, diagonalise,
occupy, output_density, energy_terms), ``src/cdft/scf/loop.py`` (initial_density,
BoundReusePolicy, solve_self_consistent with its fallback ladder), ``src/cdft/scf/mixing.py``
(LinearMixer, PulayMixer) and ``src/cdft/scf/noninteracting.py`` for the cusp-factorised,
spin-restricted path. The same control flow and the same stop tests as the reference; every
field operation is a library kernel (potentials: Hartree split, Poisson, interpolant fused with the
functional at the nodes, lift, grid assembly; energies: deterministic row sums), and the host reads
a handful of scalars once per eigensolver iteration and once per SCF iteration, as the reference does.
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, stream_handle
from .eigen import (BOUND_REUSE_RITZ_FRACTION, ChebyshevFilteredSubspace, EigenConfig, EigenResult,
                    GraphedChebyshevFilter, SpectralBoundsHint)
from .geometry import CuspGeometry, _hptr, _host, gradient, partial_derivative, row_sums
from .operators import CuspFactoredHamiltonian, measure_cross
from .poisson import CoulombCutoffPoisson
from .rng import SeededStream
from .xc import functional_by_name

FILTER_STEPS_PER_ITERATION = 4
LANCZOS_REUSE_BACKSTOP = 8
LANCZOS_REUSE_MAX_WIDENING = 0.05


def aufbau_occupations(n_states: int, n_electrons: float) -> np.ndarray:
    """Restricted aufbau filling, capacity 2 (``src/cdft/scf/occupations.py:16-48``)."""
    occ = np.zeros((1, n_states))
    remaining = float(n_electrons)
    for i in range(n_states):
        if remaining <= 1e-14:
            break
        take = min(2.0, remaining)
        occ[0, i] = take
        remaining -= take
    if remaining > 1e-10:
        raise ValueError(f"{n_electrons} electrons do not fit in {n_states} states of capacity 2")
    return occ


def nuclear_repulsion(charges, positions) -> float:
    """(``src/cdft/structure.py:127-144``)"""
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    total = 0.0
    for a in range(len(charges)):
        for b in range(a + 1, len(charges)):
            total += charges[a] * charges[b] / float(np.sqrt(((pos[a] - pos[b]) ** 2).sum()))
    return total


@dataclass
class Potentials:
    """``src/cdft/scf/step.py:62-108``: the lumped effective potential and 0-d device energies."""

    v_hartree: torch.Tensor
    v_xc: torch.Tensor
    effective: torch.Tensor
    hartree_energy: torch.Tensor
    xc_energy: torch.Tensor
    xc_double_counting: torch.Tensor
    hartree_coefficients: torch.Tensor


class KohnShamStep:
    """The pure KS map on the device (``src/cdft/scf/step.py:168-481``)."""

    def __init__(self, geometry: CuspGeometry, functional: str, n_electrons: float, eigen: EigenConfig | None = None,
                 *, seed: int = 0, pad_factor: float = 2.5, filter_precision: torch.dtype = torch.float64,
                 n_states: int | None = None, external_potential: torch.Tensor | None = None,
                 graphs: bool = False) -> None:
        # graphs: run every Chebyshev filter of the solve through one GraphedChebyshevFilter (its
        # record lands in the outcome's measurements["cuda_graphs"])
        # external_potential: an extra diagonal term of the operator (an external perturbation in the
        # form quadrature.effective_potential gives it). It enters the Hamiltonian and so the band
        # energy, but not the Hartree/XC double counting, so the total energy gains Q[n dv].
        self.external = None if external_potential is None else external_potential.to(torch.float64).contiguous()
        self.geometry = geometry
        self.grid = geometry.grid
        self.factor = geometry.factor
        self.quadrature = geometry.quadrature
        self.functional = functional_by_name(functional)
        self.n_electrons = float(n_electrons)
        needed = max(1, int(-(-self.n_electrons // 2.0)))
        self.n_states = max(needed, n_states or needed)
        self.n_spin = 1
        from .carriers import eigen_config
        self.eigen = eigen_config(eigen)
        self.seed = seed
        self.ion_ion = nuclear_repulsion(geometry.charges, geometry.positions)
        self.poisson = CoulombCutoffPoisson(self.grid, pad_factor=pad_factor)
        self._bare = CuspFactoredHamiltonian(self.grid, self.factor, quadrature=self.quadrature)
        self.filter_precision = filter_precision
        self._f2_grid = self.factor.weight
        self.filter_engine = GraphedChebyshevFilter(self.grid.device) if graphs else None
        n = self.grid.n_points
        dev = self.grid.device
        self._fields = torch.empty((2, n), dtype=torch.float64, device=dev)
        self._scratch_n = torch.empty(n, dtype=torch.float64, device=dev)
        self._coef = torch.empty(len(geometry.charges), dtype=torch.float64, device=dev)

    # -- potentials (step.py:224-313) --
    def potentials(self, density: torch.Tensor) -> Potentials:
        if density.shape[0] != 1:
            raise NotImplementedError("the self-consistent path is spin-restricted (n_spin = 1)")
        if self.functional.name != "lda_vwn":
            return self._potentials_generic(density)
        g = self.geometry
        q = self.quadrature
        grid = self.grid
        n = grid.n_points
        m = q.n_nodes
        na = len(g.charges)
        dev = grid.device
        stream = stream_handle(dev)
        n_grid = density[0].to(torch.float64).contiguous()
        fields = torch.empty((2, n), dtype=torch.float64, device=dev)  # [rho, v_smooth]
        rho = fields[0]
        n_smooth = self._scratch_n
        call("cdftb_hartree_split_f64", ptr(n_grid), ptr(self._f2_grid), None, None, 0, n, 1, ptr(rho), ptr(n_smooth),
             stream)
        rho_nuc = torch.empty((1, na), dtype=torch.float64, device=dev)
        call("cdftb_quadrature_interpolate_f64", ptr(g.step.nuclei_base), ptr(g.step.nuclei_w1d), na, *grid.shape,
             ptr(rho), 1, n, ptr(rho_nuc), na, stream)
        coef = torch.empty(na, dtype=torch.float64, device=dev)
        call("cdftb_cusp_coefficients_f64", ptr(rho_nuc), ptr(g.step.nucleus_f2), ptr(g.step.overlap), na, 1, ptr(coef),
             stream)
        call("cdftb_hartree_split_f64", ptr(n_grid), ptr(self._f2_grid), ptr(g.step.cusp_grid), ptr(coef), na, n, 1,
             ptr(rho), ptr(n_smooth), stream)
        self.poisson.solve_batch(n_smooth.reshape(1, n), out=fields[1].reshape(1, n))
        node_fields = torch.empty((2, m), dtype=torch.float64, device=dev)
        call("cdftb_quadrature_interpolate_f64", ptr(q.base), ptr(q.w1d), m, *grid.shape, ptr(fields), 2, n,
             ptr(node_fields), m, stream)
        lift_in = torch.empty((2, m), dtype=torch.float64, device=dev)
        e_w = torch.empty(m, dtype=torch.float64, device=dev)
        call("cdftb_potentials_node_lda_f64", ptr(node_fields), m, ptr(q.weights), ptr(q.f2), ptr(g.step.v1s_node),
             ptr(coef), na, 1, ptr(lift_in), ptr(e_w), stream)
        lifted = q._lift_raw(lift_in, 2)
        effective = torch.empty(n, dtype=torch.float64, device=dev)
        v_hartree = torch.empty(n, dtype=torch.float64, device=dev)
        v_xc = torch.empty(n, dtype=torch.float64, device=dev)
        terms = torch.empty((3, n), dtype=torch.float64, device=dev)
        call("cdftb_potentials_grid_lda_f64", ptr(n_grid), ptr(rho), ptr(self._f2_grid), ptr(q.far_weights),
             ptr(q.mass_weights), ptr(fields[1]), ptr(g.step.v1s_grid), ptr(coef), na, ptr(lifted), n, 1,
             ptr(effective), ptr(v_hartree), ptr(terms), ptr(v_xc), stream)
        sums = row_sums(terms)
        node_sum = row_sums(e_w.reshape(1, m))[0]
        return Potentials(v_hartree=v_hartree, v_xc=v_xc[None, :], effective=effective, hartree_energy=0.5 * sums[0],
                          xc_energy=node_sum + sums[2], xc_double_counting=sums[1], hartree_coefficients=coef)

    def _potentials_generic(self, density: torch.Tensor) -> Potentials:
        """Potentials for any native functional (step.py:224-313) through ``functional.evaluate``;
        a GGA adds the gradient term in weak form, by lift and FD transpose (step.py:252-280). The
        spin-restricted VWN LDA takes the fused kernels of :meth:`potentials` instead."""
        gga = self.functional.rung >= 2
        g = self.geometry
        q = self.quadrature
        grid = self.grid
        factor = self.factor
        n = grid.n_points
        m = q.n_nodes
        na = len(g.charges)
        dev = grid.device
        stream = stream_handle(dev)
        f2 = self._f2_grid
        n_grid = density[0].to(torch.float64).contiguous()
        rho = torch.empty(n, dtype=torch.float64, device=dev)
        n_smooth = torch.empty(n, dtype=torch.float64, device=dev)
        call("cdftb_hartree_split_f64", ptr(n_grid), ptr(f2), None, None, 0, n, 1, ptr(rho), ptr(n_smooth), stream)
        rho_nuc = torch.empty((1, na), dtype=torch.float64, device=dev)
        call("cdftb_quadrature_interpolate_f64", ptr(g.step.nuclei_base), ptr(g.step.nuclei_w1d), na, *grid.shape,
             ptr(rho), 1, n, ptr(rho_nuc), na, stream)
        coef = torch.empty(na, dtype=torch.float64, device=dev)
        call("cdftb_cusp_coefficients_f64", ptr(rho_nuc), ptr(g.step.nucleus_f2), ptr(g.step.overlap), na, 1, ptr(coef),
             stream)
        call("cdftb_hartree_split_f64", ptr(n_grid), ptr(f2), ptr(g.step.cusp_grid), ptr(coef), na, n, 1, ptr(rho),
             ptr(n_smooth), stream)
        v_smooth = self.poisson.solve(n_smooth)
        v_h_grid = (coef[:, None] * g.step.v1s_grid).sum(dim=0) + v_smooth
        if not gga:
            node = q.interpolate(torch.cat([rho[None], v_smooth[None]]))
            rho_node, vs_node = node[0], node[1]
            v_h_node = (coef[:, None] * g.step.v1s_node).sum(dim=0) + vs_node
            n_node = q.f2 * rho_node
            out_grid = self.functional.evaluate(n_grid[None, :])
            out_node = self.functional.evaluate(n_node[None, :])
            e_n_node, e_n_grid = out_node.v_xc[0], out_grid.v_xc[0]
            lift_in = torch.cat([(q.weights * (q.f2 * v_h_node))[None], (q.weights * (q.f2 * e_n_node))[None]])
            lifted = q.lift(lift_in.contiguous())
            hartree_w = lifted[0] + q.far_weights * (f2 * v_h_grid)
            xc_w = lifted[1] + q.far_weights * (f2 * e_n_grid)
            hartree_energy = 0.5 * row_sums((hartree_w * rho)[None])[0]
            xc_energy = q.integrate(out_node.e_xc, out_grid.e_xc)
            xc_dc = row_sums((xc_w * rho)[None])[0]
            effective = (hartree_w + xc_w) / q.mass_weights
            return Potentials(v_hartree=v_h_grid, v_xc=e_n_grid[None, :].clone(), effective=effective,
                              hartree_energy=hartree_energy, xc_energy=xc_energy, xc_double_counting=xc_dc,
                              hartree_coefficients=coef)
        grad_rho = gradient(grid, rho)
        node = q.interpolate(torch.cat([rho[None], grad_rho, v_smooth[None]]))
        rho_node, grad_rho_node, vs_node = node[0], node[1:4], node[4]
        v_h_node = (coef[:, None] * g.step.v1s_node).sum(dim=0) + vs_node
        n_node = q.f2 * rho_node
        grad_n_node = q.f2[None, :] * (grad_rho_node - 2.0 * rho_node[None, :] * q.grad_u)
        grad_n_grid = f2[None, :] * (grad_rho - 2.0 * rho[None, :] * factor.grad_u)
        sigma_grid = (grad_n_grid * grad_n_grid).sum(dim=0)
        sigma_node = (grad_n_node * grad_n_node).sum(dim=0)
        out_grid = self.functional.evaluate(n_grid[None, :], sigma_grid[None, :])
        out_node = self.functional.evaluate(n_node[None, :], sigma_node[None, :])
        e_n_node, e_n_grid = out_node.v_xc[0], out_grid.v_xc[0]
        e_s_node, e_s_grid = out_node.v_sigma[0], out_grid.v_sigma[0]
        flux_node = 2.0 * e_s_node[None, :] * q.f2[None, :] * grad_n_node
        flux_grid = 2.0 * e_s_grid[None, :] * f2[None, :] * grad_n_grid
        cross_node = -2.0 * (flux_node * q.grad_u).sum(dim=0)
        cross_grid = -2.0 * (flux_grid * factor.grad_u).sum(dim=0)
        lift_in = torch.cat([(q.weights * (q.f2 * v_h_node))[None], (q.weights * (q.f2 * e_n_node))[None],
                             q.weights[None, :] * flux_node, (q.weights * cross_node)[None]]).contiguous()
        lifted = q.lift(lift_in)
        hartree_w = lifted[0] + q.far_weights * (f2 * v_h_grid)
        xc_w = lifted[1] + q.far_weights * (f2 * e_n_grid)
        # lumped_gradient_weights: -sum_d D_d [L^T(w flux_d) + h^3 far flux_grid_d]
        pre = lifted[2:5] + grid.volume_element * (q.far[None, :] * flux_grid)
        div = torch.zeros(n, dtype=torch.float64, device=dev)
        for d in range(3):
            partial_derivative(grid, pre[d], d, out=div, accumulate=True, sign=-1.0)
        xc_w = xc_w + div
        xc_w = xc_w + (lifted[5] + q.far_weights * cross_grid)
        hartree_energy = 0.5 * row_sums((hartree_w * rho)[None])[0]
        xc_energy = q.integrate(out_node.e_xc, out_grid.e_xc)
        xc_dc = row_sums((xc_w * rho)[None])[0]
        effective = (hartree_w + xc_w) / q.mass_weights
        return Potentials(v_hartree=v_h_grid, v_xc=e_n_grid[None, :], effective=effective, hartree_energy=hartree_energy,
                          xc_energy=xc_energy, xc_double_counting=xc_dc, hartree_coefficients=coef)

    def hamiltonian(self, potentials: Potentials, *, dtype: torch.dtype = torch.float64) -> CuspFactoredHamiltonian:
        extra = potentials.effective if self.external is None else potentials.effective + self.external
        return CuspFactoredHamiltonian(self.grid, self.factor, extra_potential=extra, quadrature=self.quadrature,
                                       dtype=dtype)

    #: A float-filtered full diagonalisation switches to the float64 filter below this residual.
    FLOAT_FILTER_SWITCH_RESIDUAL = 1.0e-4

    def diagonalise(self, hamiltonian, initial=None, max_iterations=None, *, bounds=None, filter_hamiltonian=None):
        """(``src/cdft/scf/step.py:321-355``); ``ritz_stop=False`` inside the SCF.

        With a float ``filter_hamiltonian``, a full diagonalisation (no iteration cap) filters in
        float until its residual is below :attr:`FLOAT_FILTER_SWITCH_RESIDUAL`, then in float64; a
        capped one (the warm-started SCF iterations) filters in float throughout.
        """
        # a freshly seeded generator per call, as step.py:338; its draws are cached on the device
        generator = SeededStream(self.seed, self.grid.device)
        cfg = self.eigen
        if max_iterations is not None:
            cfg = EigenConfig(**{**cfg.__dict__, "max_iterations": max_iterations})
        switch = self.FLOAT_FILTER_SWITCH_RESIDUAL if max_iterations is None else None
        solver = ChebyshevFilteredSubspace(self.grid, cfg, ritz_stop=False, filter_hamiltonian=filter_hamiltonian,
                                           switch_residual=switch, filter_engine=self.filter_engine)
        result = solver.solve(hamiltonian, self.n_states, initial=initial, generator=generator, bounds=bounds)
        info = {"eigen_stop_reason": solver.stop_reason, "eigen_eigenvalue_drift": solver.eigenvalue_drift,
                "eigen_spectral_bounds": list(solver.spectral_bounds or ()), "eigen_bounds_source": solver.bounds_source,
                "eigen_bounds_shift": solver.bounds_shift, "eigen_top_ritz_fraction": solver.top_ritz_fraction}
        return result, info

    def occupy(self, eigenvalues: torch.Tensor) -> torch.Tensor:
        return torch.from_numpy(aufbau_occupations(eigenvalues.shape[-1], self.n_electrons)).to(self.grid.device)

    def output_density(self, eigen: EigenResult, occupations: torch.Tensor):
        phi = eigen.eigenvectors.to(torch.float64)
        rho_out = (occupations[0][:, None] * phi.pow(2)).sum(dim=0)
        return (rho_out * self._f2_grid)[None, :], rho_out

    ENERGY_TERMS = ("total", "kinetic", "external", "hartree", "xc", "harris_foulkes", "band", "external_direct",
                    "kinetic_plus_external")

    def energy_terms(self, eigen, occupations, rho_out, p_in: Potentials, p_out: Potentials | None):
        """(``src/cdft/scf/step.py:398-439``) as 0-d device tensors."""
        band = (occupations[0] * eigen.eigenvalues).sum()
        ham = self._bare
        phi = eigen.eigenvectors.to(torch.float64)
        kinetic = ham.kinetic_energy_tensor(phi, occupations[0])
        dc_out = row_sums((p_in.effective * self.quadrature.mass_weights * rho_out)[None])[0]
        kinetic_plus_external = band - dc_out
        external_direct = ham.external_energy_direct_tensor(rho_out)
        harris = band - p_in.hartree_energy - p_in.xc_double_counting + p_in.xc_energy + self.ion_ion
        if p_out is None:
            total = harris
            hartree, xc = p_in.hartree_energy, p_in.xc_energy
        else:
            hartree, xc = p_out.hartree_energy, p_out.xc_energy
            total = kinetic_plus_external + hartree + xc + self.ion_ion
        external = total - kinetic - hartree - xc - self.ion_ion
        values = {"total": total, "kinetic": kinetic, "external": external, "hartree": hartree, "xc": xc,
                  "harris_foulkes": harris, "band": band, "external_direct": external_direct,
                  "kinetic_plus_external": kinetic_plus_external}
        return {k: values[k] for k in self.ENERGY_TERMS}


def initial_density(step: KohnShamStep, kind: str = "hydrogenic") -> torch.Tensor:
    """(``src/cdft/scf/loop.py:173-193``) on the device; one host read of the charge."""
    scale = {"hydrogenic": 1.0, "diffuse": 0.5, "compact": 2.0}[kind]
    g = step.geometry
    grid = step.grid
    n = grid.n_points
    total = torch.empty(n, dtype=torch.float64, device=grid.device)
    terms = torch.empty(n, dtype=torch.float64, device=grid.device)
    ch, ps = _host(g.charges), _host(g.positions)
    call("cdftb_geometry_initial_density", len(g.charges), _hptr(ch), _hptr(ps), *grid.shape, *grid.origin, grid.spacing,
         scale, ptr(step._f2_grid), ptr(step.quadrature.mass_weights), ptr(total), ptr(terms), stream_handle(grid.device))
    charge_now = float(row_sums(terms[None])[0])
    call("cdftb_scale_f64", ptr(total), n, step.n_electrons / charge_now, stream_handle(grid.device))
    return total[None, :].clone()


class KerkerPreconditioner:
    """``F(q) q^2 / (q^2 + q0^2)`` on the box (``src/cdft/scf/mixing.py:35-56``), one library call
    (``cdftb_kerker_precondition_f64``) for every spin row of a ``(n_spin, N)`` residual."""

    def __init__(self, grid, q0: float) -> None:
        self.grid = grid
        self.q0 = float(q0)

    def __call__(self, residual: torch.Tensor) -> torch.Tensor:
        _lib.require_cuda(residual, "residual")
        x = residual.to(torch.float64).contiguous()
        rows = x.numel() // self.grid.n_points
        nbytes = _lib.library().cdftb_kerker_work_bytes(*self.grid.shape, rows)
        work = torch.empty(nbytes, dtype=torch.uint8, device=x.device)
        out = torch.empty_like(x)
        call("cdftb_kerker_precondition_f64", ptr(x), rows, *self.grid.shape, self.grid.spacing, self.q0, ptr(out),
             ptr(work), nbytes, stream_handle(x.device))
        return out


class LinearMixer:
    """(``src/cdft/scf/mixing.py:59-83``)"""

    def __init__(self, alpha: float, preconditioner=None):
        if not 0.0 < alpha <= 1.0:
            raise ValueError("mixing alpha must lie in (0, 1]")
        self.alpha = alpha
        self.preconditioner = preconditioner
        self.name = f"linear mixing, alpha {alpha:g}"
        self.last_event = "damped step"

    def mix(self, n_in, n_out, iteration):
        residual = n_out - n_in
        if self.preconditioner is not None:
            residual = self.preconditioner(residual)
        return n_in + self.alpha * residual


class PulayMixer:
    """Periodic Pulay / DIIS (``src/cdft/scf/mixing.py:86-162``); residual products on the device."""

    def __init__(self, alpha: float, history: int, period: int, inner_weights: torch.Tensor, preconditioner=None):
        if history < 2:
            raise ValueError("a Pulay history holds at least 2 pairs")
        if period < 1:
            raise ValueError("the Pulay period is at least 1")
        self.alpha, self.history, self.period = alpha, history, period
        self.inner_weights = inner_weights
        self.preconditioner = preconditioner
        self._inputs, self._residuals = [], []
        self.name = (f"DIIS every {period} iterations, alpha {alpha:g}, {history} pairs" if period > 1
                     else f"DIIS, alpha {alpha:g}, {history} pairs")
        self.last_event = ""

    def mix(self, n_in, n_out, iteration):
        residual = n_out - n_in
        if self.preconditioner is not None:
            residual = self.preconditioner(residual)
        self._inputs.append(n_in.clone())
        self._residuals.append(residual.clone())
        if len(self._inputs) > self.history:
            self._inputs.pop(0)
            self._residuals.pop(0)
        m = len(self._inputs)
        if m < 2 or iteration % self.period != 0:
            self.last_event = "damped step"
            return n_in + self.alpha * residual
        stack = torch.stack([r.reshape(-1) for r in self._residuals])
        gram = measure_cross(stack, stack, self.inner_weights)[0].cpu().numpy()
        scale = float(gram.diagonal().max()) or 1.0
        gram = gram + 1.0e-12 * scale * np.eye(m)
        system = np.zeros((m + 1, m + 1))
        system[:m, :m] = gram
        system[:m, m] = -1.0
        system[m, :m] = 1.0
        rhs = np.zeros(m + 1)
        rhs[m] = 1.0
        coefficients = np.linalg.solve(system, rhs)[:m]
        self.last_event = f"DIIS combination of {m} pairs"
        mixed = torch.zeros_like(n_in)
        for c, stored_in, stored_res in zip(coefficients, self._inputs, self._residuals):
            mixed = mixed + float(c) * (stored_in + self.alpha * stored_res)
        return mixed


@dataclass
class MixingConfig:
    """``contract.MixingConfig`` (contract.py:466-474)."""

    scheme: str = "periodic_pulay"  # linear | anderson | pulay | periodic_pulay | kerker
    alpha: float = 0.30
    history: int = 8
    pulay_period: int = 3
    kerker: bool = False
    kerker_q0: float = 1.5


@dataclass
class SCFConfig:
    """``contract.SCFConfig`` (contract.py:475-490)."""

    energy_tol: float = 1.0e-8
    density_tol: float = 1.0e-6
    max_iterations: int = 200
    min_iterations: int = 3
    fallback_ladder: bool = True


def make_mixer(cfg: MixingConfig, alpha: float, inner_weights, scheme: str | None = None, grid=None):
    """The mixer a mixing configuration asks for (``src/cdft/scf/mixing.py:160-177``): ``kerker``
    as a scheme is periodic Pulay with the Kerker preconditioner; ``kerker=True`` adds the
    preconditioner to any scheme; ``anderson`` and ``pulay`` are Pulay with period 1."""
    scheme = str(getattr(scheme or cfg.scheme, "value", scheme or cfg.scheme)).lower()
    if scheme not in ("linear", "anderson", "pulay", "periodic_pulay", "kerker"):
        raise ValueError(f"unknown mixing scheme {scheme!r}")
    kerker = cfg.kerker or scheme == "kerker"
    if kerker and grid is None:
        raise ValueError("the Kerker preconditioner needs the grid")
    pre = KerkerPreconditioner(grid, cfg.kerker_q0) if kerker else None
    if scheme == "linear":
        return LinearMixer(alpha, pre)
    period = cfg.pulay_period if scheme in ("periodic_pulay", "kerker") else 1
    return PulayMixer(alpha, cfg.history, period, inner_weights, pre)


class BoundReusePolicy:
    """(``src/cdft/scf/loop.py:94-170``)"""

    def __init__(self, enabled: bool = True) -> None:
        self.enabled = enabled
        self.bounds = None
        self.since_estimate = 0
        self.widening = 0.0
        self.top_fraction = float("nan")
        self.history: list[str] = []
        self.reestimates = 0
        self.reuses = 0

    def decide(self, *, residual_rose: bool, rung_changed: bool, level_shift: bool):
        if not self.enabled:
            return "carrying bounds is switched off"
        if self.bounds is None:
            return "nothing carried yet"
        if level_shift:
            return "the operator is level-shifted"
        if rung_changed:
            return "the mixer was just replaced"
        if residual_rose:
            return "the density residual grew"
        if self.since_estimate >= LANCZOS_REUSE_BACKSTOP:
            return f"{LANCZOS_REUSE_BACKSTOP} iterations since the last estimate"
        low, high = self.bounds
        if self.widening > LANCZOS_REUSE_MAX_WIDENING * (high - low):
            return "the carried interval has widened too far"
        if not self.top_fraction < BOUND_REUSE_RITZ_FRACTION:
            return "the top Ritz value came close to the upper bound"
        return None

    def hint(self, shift):
        return SpectralBoundsHint(self.bounds[0], self.bounds[1], shift)

    def observe(self, reason, info):
        b = info.get("eigen_spectral_bounds") or None
        self.bounds = (float(b[0]), float(b[1])) if b else None
        self.top_fraction = float(info.get("eigen_top_ritz_fraction", float("nan")))
        if str(info.get("eigen_bounds_source", "lanczos")) == "reused":
            self.reuses += 1
            self.since_estimate += 1
            self.widening += float(info.get("eigen_bounds_shift", 0.0))
            self.history.append("reused")
        else:
            self.reestimates += 1
            self.since_estimate = 0
            self.widening = 0.0
            self.history.append(f"lanczos: {reason}")


class _LevelShifted:
    """``H + Delta (1 - P_occ)`` (``src/cdft/scf/loop.py:553-589``)."""

    uses_divergence_form = True

    def __init__(self, inner, eigen, occupations, shift):
        self.inner = inner
        self.measure = inner.measure
        self.grid = inner.grid
        self.shift = shift
        occupied = None
        if eigen is not None and occupations is not None:
            mask = occupations.sum(dim=0) > 1e-12
            occupied = eigen.eigenvectors[mask].to(torch.float64) if bool(mask.any()) else None
        self.occupied = occupied
        self.apply_count = 0

    def note_applications(self, count):
        self.apply_count += int(count)

    def apply(self, phi):
        self.apply_count += 1
        out = self.inner.apply(phi)
        if self.occupied is None:
            return out
        coefficients = self.measure.cross(phi, self.occupied)
        return out + self.shift * (phi - coefficients @ self.occupied)

    def spectral_bounds(self, **kwargs):
        lo, hi = self.inner.spectral_bounds(**kwargs)
        return lo, hi + self.shift


@dataclass
class SCFOutcome:
    energies: dict
    eigenvalues: list
    scf_iterations: int
    converged: bool
    applications: float
    energy_history: list = field(default_factory=list)
    residual_history: list = field(default_factory=list)
    density: torch.Tensor | None = None
    measurements: dict = field(default_factory=dict)


def solve_self_consistent(step: KohnShamStep, mixing: MixingConfig | None = None, scf: SCFConfig | None = None, *,
                          initial_guess: str = "hydrogenic", max_iterations: int | None = None,
                          refine_in_float64: bool = True,
                          initial_density_override: torch.Tensor | None = None) -> SCFOutcome:
    """(``src/cdft/scf/loop.py:255-550``) on the device.

    With ``step.filter_precision == torch.float32`` the Chebyshev filter runs in float (the
    mixed-precision form); Rayleigh--Ritz, residuals, Lanczos and every energy stay float64. Once the
    float-filtered iteration meets the convergence test, the FP64 refinement sweep takes over: the
    loop continues with the float64 filter until the same test passes again, and the final full
    diagonalisation filters in float64, so the converged density carries no float32 noise.
    """
    from .carriers import mixing_config, scf_config
    started = time.perf_counter()
    mixing = mixing_config(mixing)
    scf = scf_config(scf)
    q = step.quadrature
    mass = q.mass_weights
    f2 = step._f2_grid
    inner_weights = (mass / f2 ** 2).contiguous()

    def norm_l1(delta):
        return row_sums((mass * (delta.sum(dim=0).abs() / f2))[None])[0]

    if initial_density_override is not None:
        n_in = initial_density_override.to(device=step.grid.device, dtype=torch.float64).reshape(1, -1).clone()
    else:
        n_in = initial_density(step, initial_guess)
    mixer = make_mixer(mixing, mixing.alpha, inner_weights, grid=step.grid)
    ladder = [
        ("pulay", lambda: make_mixer(mixing, mixing.alpha, inner_weights, grid=step.grid)),
        ("damped pulay", lambda: make_mixer(mixing, 0.5 * mixing.alpha, inner_weights, grid=step.grid)),
        ("linear", lambda: LinearMixer(0.5 * mixing.alpha)),
        ("linear, level shift 0.5 Ha", lambda: LinearMixer(0.5 * mixing.alpha)),
    ]
    rung, level_shift, worsened = 0, 0.0, 0
    previous_residual = float("inf")
    initial_block = None
    eigen = None
    occupations = None
    energies, harris, residuals, changes = [], [], [], []
    applications: list[int] = []
    policy = BoundReusePolicy()
    previous_effective = None
    rung_changed = False
    converged = False
    fallback_events: list[str] = []
    limit = scf.max_iterations if max_iterations is None else max_iterations
    mixed = step.filter_precision == torch.float32
    refinement_from = None
    iteration = 0
    p_in = None
    for iteration in range(1, limit + 1):
        p_in = step.potentials(n_in)
        hamiltonian = step.hamiltonian(p_in)
        filter_h = step.hamiltonian(p_in, dtype=torch.float32) if mixed else None
        if level_shift:
            hamiltonian = _LevelShifted(hamiltonian, eigen, occupations, level_shift)
            filter_h = None
        steps = None if initial_block is None else FILTER_STEPS_PER_ITERATION
        reason = policy.decide(residual_rose=worsened > 0, rung_changed=rung_changed, level_shift=bool(level_shift))
        hint = None
        if reason is None and previous_effective is not None:
            hint = policy.hint((p_in.effective - previous_effective).abs().max())
        elif reason is None:
            reason = "no previous potential"
        eigen, info = step.diagonalise(hamiltonian, initial=initial_block, max_iterations=steps, bounds=hint,
                                       filter_hamiltonian=filter_h)
        policy.observe(reason, info)
        previous_effective = p_in.effective
        rung_changed = False
        applications.append(int(hamiltonian.apply_count))
        initial_block = eigen.eigenvectors
        occupations = step.occupy(eigen.eigenvalues)
        n_out, rho_out = step.output_density(eigen, occupations)
        p_out = step.potentials(n_out)
        terms = step.energy_terms(eigen, occupations, rho_out, p_in, p_out)
        residual = n_out - n_in
        res_norm_d = norm_l1(residual)
        n_next = mixer.mix(n_in, n_out, iteration)
        change_d = norm_l1(n_next - n_in)
        host = torch.stack([*terms.values(), res_norm_d, change_d]).tolist()
        _lib.check_device_status(f"SCF iteration {iteration}")
        nt = len(terms)
        values = dict(zip(terms, host[:nt]))
        res_norm, change = host[nt], host[nt + 1]
        energies.append(values["total"])
        harris.append(values["harris_foulkes"])
        residuals.append(res_norm)
        changes.append(change)
        de = abs(energies[-1] - energies[-2]) if len(energies) > 1 else float("inf")
        if iteration >= scf.min_iterations and de < scf.energy_tol and res_norm < scf.density_tol:
            if mixed:
                # the float-filtered fixed point is reached: refine in float64 from here
                mixed = False
                refinement_from = iteration + 1
            else:
                converged = True
                break
        worsened = worsened + 1 if res_norm > previous_residual else 0
        previous_residual = res_norm
        if scf.fallback_ladder and worsened >= 3 and rung + 1 < len(ladder):
            rung += 1
            name, factory = ladder[rung]
            mixer = factory()
            if "level shift" in name:
                level_shift = 0.5
            fallback_events.append(f"iteration {iteration}: residual grew three times, stepping down to {name}")
            worsened = 0
            rung_changed = True
            n_next = n_in + 0.5 * mixing.alpha * residual
        n_in = n_next
    # final full diagonalisation at the last input potential, fresh Lanczos, float64 filter
    final_h = step.hamiltonian(p_in)
    float_final = step.filter_precision == torch.float32 and not refine_in_float64
    eigen, info = step.diagonalise(final_h, initial=eigen.eigenvectors,
                                   filter_hamiltonian=step.hamiltonian(p_in, dtype=torch.float32) if float_final else None)
    occupations = step.occupy(eigen.eigenvalues)
    n_out, rho_out = step.output_density(eigen, occupations)
    p_out = step.potentials(n_out)
    terms = step.energy_terms(eigen, occupations, rho_out, p_in, p_out)
    charge = row_sums((mass * rho_out)[None])[0]
    host = torch.stack([*terms.values(), charge, *eigen.eigenvalues]).tolist()
    _lib.check_device_status("final diagonalisation")
    nt = len(terms)
    final = dict(zip(terms, host[:nt]))
    measurements = {
        "scf_hamiltonian_applications": applications,
        "hamiltonian_applications": float(sum(applications) + final_h.apply_count),
        "scf_fallbacks": fallback_events,
        "mixer": mixer.name,
        "charge_error": abs(host[nt] - step.n_electrons),
        "eigen_stop_reason": info["eigen_stop_reason"],
        "lanczos_reestimates": policy.reestimates,
        "lanczos_reuses": policy.reuses,
        "filter_precision": "float32" if step.filter_precision == torch.float32 else "float64",
        "fp64_refinement_from_iteration": refinement_from,
        "fused_kernels": {"tier": "native-sm100a", "library": _lib.LIBRARY_PATH.name},
        "wall_s": time.perf_counter() - started,
    }
    if step.filter_engine is not None:
        measurements["cuda_graphs"] = step.filter_engine.record()
    return SCFOutcome(energies=final, eigenvalues=host[nt + 1:], scf_iterations=iteration,
                      converged=converged and eigen.converged, applications=measurements["hamiltonian_applications"],
                      energy_history=energies, residual_history=residuals, density=n_out, measurements=measurements)


def lobpcg_cross_check(hamiltonian, eigenvalues: torch.Tensor, n_states: int, eigen: EigenConfig, seed: int) -> dict:
    """The two-solver check of gate G2.5 (``src/cdft/scf/noninteracting.py:182-189``): LOBPCG on the
    same operator from a start seeded with ``seed + 1``, against the Chebyshev eigenvalues."""
    from .eigen import LOBPCG

    grid = hamiltonian.grid
    second = LOBPCG(grid, eigen).solve(hamiltonian, n_states, generator=SeededStream(seed + 1, grid.device))
    delta = (eigenvalues.to(torch.float64) - second.eigenvalues).abs()
    return {"two_solver_max_delta": float(delta.max()), "two_solver_converged": bool(second.converged),
            "lobpcg_iterations": float(second.n_iterations),
            "lobpcg_eigenvalues": second.eigenvalues.tolist()}


def solve_noninteracting(geometry: CuspGeometry, n_electrons: float, *, seed: int = 0,
                         eigen: EigenConfig | None = None, external_potential: torch.Tensor | None = None,
                         cross_check: bool | None = None, graphs: bool = False) -> dict:
    """(``src/cdft/scf/noninteracting.py:118-330``) for the cusp-factorised path, ``ritz_stop=True``.

    ``external_potential`` adds a diagonal term to the operator (an external perturbation in the
    form quadrature.effective_potential gives it). The result also holds the occupied orbitals and
    their occupations (``"orbitals"``, ``"occupations"``), normalised in the measure.
    """
    from .carriers import eigen_config
    eigen = eigen_config(eigen)
    cross_check = eigen.cross_check if cross_check is None else cross_check
    grid = geometry.grid
    ham = CuspFactoredHamiltonian(grid, geometry.factor, extra_potential=external_potential,
                                  quadrature=geometry.quadrature)
    n_states = max(1, int(-(-float(n_electrons) // 2.0)))
    generator = SeededStream(seed, grid.device)
    engine = GraphedChebyshevFilter(grid.device) if graphs else None
    solver = ChebyshevFilteredSubspace(grid, eigen, ritz_stop=True, filter_engine=engine)
    result = solver.solve(ham, n_states, generator=generator)
    occ = torch.from_numpy(aufbau_occupations(n_states, float(n_electrons))).to(grid.device)
    kinetic = ham.kinetic_energy_tensor(result.eigenvectors, occ[0])
    band = (occ[0] * result.eigenvalues).sum()
    vals = torch.stack([kinetic, band, *result.eigenvalues]).tolist()
    kinetic, band = vals[0], vals[1]
    ion_ion = nuclear_repulsion(geometry.charges, geometry.positions)
    external = band - kinetic
    out = {"total": kinetic + external + ion_ion, "kinetic": kinetic, "eigenvalues": vals[2:],
           "iterations": result.n_iterations, "converged": result.converged, "applications": float(ham.apply_count),
           "stop_reason": solver.stop_reason, "orbitals": result.eigenvectors, "occupations": occ[0]}
    if engine is not None:
        out["cuda_graphs"] = engine.record()
    if cross_check:
        out.update(lobpcg_cross_check(ham, result.eigenvalues, n_states, eigen, seed))
    return out
