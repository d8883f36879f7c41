"""Kohn--Sham step, SCF driver and the non-interacting solve (oracle).

Restates ``src/cdft/scf/step.py`` (KohnShamStep.potentials/energy_terms/diagonalise),
``src/cdft/scf/loop.py`` (BoundReusePolicy, initial_density, solve_self_consistent),
``src/cdft/scf/mixing.py`` (LinearMixer, PulayMixer), ``src/cdft/scf/occupations.py`` and
``src/cdft/scf/noninteracting.py`` for the cusp-factorised, spin-restricted path.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import xc as xc_mod
from .eigen import BOUND_REUSE_RITZ_FRACTION, ChebyshevFilteredSubspace
from .geometry import CuspFactor, CuspQuadrature, StepGeometry
from .grid import Grid
from .operators import CoulombCutoffPoisson, CuspHamiltonian
from .rng import make_generator

FILTER_STEPS_PER_ITERATION = 4
LANCZOS_REUSE_BACKSTOP = 8
LANCZOS_REUSE_MAX_WIDENING = 0.05


@dataclass
class System:
    """One all-electron system: nuclei, electrons, box, spacing and solver settings."""

    charges: tuple
    positions: tuple
    n_electrons: float
    box_lengths: tuple
    spacing: float
    anchor: tuple | None = None
    functional: str = "none"
    ion_charge: float = 0.0
    chebyshev_degree: int = 20
    n_extra_states: int = 4
    residual_tol: float = 1e-8
    max_eigen_iterations: int = 300
    mixing: str = "linear"
    alpha: float = 0.3
    history: int = 8
    pulay_period: int = 3
    energy_tol: float = 1e-8
    density_tol: float = 1e-6
    max_scf_iterations: int = 200
    min_scf_iterations: int = 3
    seed: int = 0
    pad_factor: float = 2.5


def nuclear_repulsion(charges, positions) -> float:
    """(``src/cdft/structure.py:127-144``)"""
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
    total = 0.0
    for a in range(len(charges)):
        for b in range(a + 1, len(charges)):
            total += charges[a] * charges[b] / float(np.sqrt(((pos[a] - pos[b]) ** 2).sum()))
    return total


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
        raise ValueError("electrons do not fit in the states")
    return occ


def build_geometry(system: System):
    grid = Grid.box(system.box_lengths, system.spacing, anchor=system.anchor)
    factor = CuspFactor(grid, system.charges, system.positions)
    quadrature = CuspQuadrature(grid, factor)
    return grid, factor, quadrature


class KohnShamStep:
    """The pure KS map (``src/cdft/scf/step.py:168-481``)."""

    def __init__(self, system: System, grid: Grid, factor: CuspFactor, quadrature: CuspQuadrature):
        self.system = system
        self.grid = grid
        self.factor = factor
        self.quadrature = quadrature
        self.functional = system.functional
        self.n_electrons = system.n_electrons
        self.n_states = max(1, int(-(-system.n_electrons // 2.0)))
        self.ion_ion = nuclear_repulsion(system.charges, system.positions)
        self.poisson = CoulombCutoffPoisson(grid, system.pad_factor)
        self.bare = quadrature.bare_operator_terms()
        self.bare_hamiltonian = CuspHamiltonian(grid, factor, quadrature, bare=self.bare)
        self.geometry = StepGeometry(grid, quadrature, system.charges, system.positions)
        self.f2 = factor.weight

    def potentials(self, density):
        """(``src/cdft/scf/step.py:224-313``)"""
        q = self.quadrature
        f2 = self.f2
        g = self.geometry
        n_grid = density.sum(axis=0)
        rho = n_grid / f2
        rho_at_nuclei = q.interpolate_at(g.positions, rho)
        n_at_nuclei = g.nucleus_f2 * rho_at_nuclei
        coefficients = np.linalg.solve(g.overlap, n_at_nuclei)
        n_cusp = (coefficients[:, None] * g.cusp_grid).sum(axis=0)
        n_smooth = n_grid - n_cusp
        v_smooth = self.poisson.solve(n_smooth)
        v_h_grid = (coefficients[:, None] * g.v1s_grid).sum(axis=0) + v_smooth
        v_h_node = (coefficients[:, None] * g.v1s_node).sum(axis=0) + q.interpolate(v_smooth)
        n_node, grad_n_node = q.density_gradient_at_nodes(rho)
        hartree_weights = q.lumped_weights(q.f2 * v_h_node, f2 * v_h_grid)
        hartree_energy = 0.5 * (hartree_weights * rho).sum()
        gga = xc_mod.RUNG[self.functional] >= 2
        grad_n_grid = q.density_gradient_on_grid(rho) if gga else None
        sigma_grid = (grad_n_grid * grad_n_grid).sum(axis=0) if gga else None
        sigma_node = (grad_n_node * grad_n_node).sum(axis=0) if gga else None
        e_grid, vn_grid, vs_grid = xc_mod.evaluate(self.functional, n_grid, sigma_grid)
        e_node, vn_node, vs_node = xc_mod.evaluate(self.functional, n_node, sigma_node)
        xc_energy = q.integrate(e_node, e_grid)
        xc_weights = q.lumped_weights(q.f2 * vn_node, f2 * vn_grid)
        if gga:
            flux_node = 2.0 * vs_node[None, :] * q.f2[None, :] * grad_n_node
            flux_grid = 2.0 * vs_grid[None, :] * f2[None, :] * grad_n_grid
            xc_weights = xc_weights + q.lumped_gradient_weights(flux_node, flux_grid)
            cross_node = -2.0 * (flux_node * q.grad_u).sum(axis=0)
            cross_grid = -2.0 * (flux_grid * self.factor.grad_u).sum(axis=0)
            xc_weights = xc_weights + q.lumped_weights(cross_node, cross_grid)
        xc_double_counting = (xc_weights * rho).sum()
        effective = (hartree_weights + xc_weights) / q.mass_weights
        return {
            "effective": effective, "hartree_energy": hartree_energy, "xc_energy": xc_energy,
            "xc_double_counting": xc_double_counting, "v_hartree": v_h_grid, "coefficients": coefficients,
            "v_xc": vn_grid,
        }

    def hamiltonian(self, effective):
        return CuspHamiltonian(self.grid, self.factor, self.quadrature, extra_potential=effective, bare=self.bare)

    def diagonalise(self, hamiltonian, initial=None, max_iterations=None, bounds=None):
        """(``src/cdft/scf/step.py:321-355``), ``ritz_stop=False``"""
        s = self.system
        generator = make_generator(s.seed)
        solver = ChebyshevFilteredSubspace(
            self.grid.n_points, degree=s.chebyshev_degree, n_extra_states=s.n_extra_states,
            max_iterations=max_iterations if max_iterations is not None else s.max_eigen_iterations,
            residual_tol=s.residual_tol, ritz_stop=False)
        result = solver.solve(hamiltonian, self.n_states, initial=initial, generator=generator, bounds=bounds)
        info = {"bounds": solver.spectral_bounds, "source": solver.bounds_source, "shift": solver.bounds_shift,
                "top_fraction": solver.top_ritz_fraction, "stop_reason": solver.stop_reason}
        return result, info

    def occupy(self, eigenvalues):
        return aufbau_occupations(eigenvalues.shape[0], self.n_electrons)

    def output_density(self, eigen, occupations):
        phi = eigen.eigenvectors
        rho_out = (occupations[0][:, None] * phi ** 2).sum(axis=0)[None, :]
        return rho_out * self.f2, rho_out.sum(axis=0)

    def energy_terms(self, eigen, occupations, rho_out, p_in, p_out):
        """(``src/cdft/scf/step.py:398-439``)"""
        band = (occupations * eigen.eigenvalues[None, :]).sum()
        ham = self.bare_hamiltonian
        kinetic = ham.kinetic_energy(eigen.eigenvectors, occupations[0])
        dc_out = (p_in["effective"] * self.quadrature.mass_weights * rho_out).sum()
        kinetic_plus_external = band - dc_out
        external_direct = ham.external_energy_direct(rho_out)
        harris = band - p_in["hartree_energy"] - p_in["xc_double_counting"] + p_in["xc_energy"] + self.ion_ion
        if p_out is None:
            total = harris
            hartree, xc = p_in["hartree_energy"], p_in["xc_energy"]
        else:
            hartree, xc = p_out["hartree_energy"], p_out["xc_energy"]
            total = kinetic_plus_external + hartree + xc + self.ion_ion
        external = total - kinetic - hartree - xc - self.ion_ion
        return {"total": float(total), "kinetic": float(kinetic), "external": float(external),
                "hartree": float(hartree), "xc": float(xc), "harris_foulkes": float(harris), "band": float(band),
                "external_direct": float(external_direct)}


def initial_density(step: KohnShamStep):
    """Hydrogenic superposition normalised in the cusp-aware measure (``src/cdft/scf/loop.py:173-193``)."""
    points = step.grid.points()
    total = np.zeros(step.grid.n_points)
    for atom, z in enumerate(step.system.charges):
        d = np.sqrt(((points - step.geometry.positions[atom]) ** 2).sum(axis=-1))
        total = total + (z ** 3 / math.pi) * np.exp(-2.0 * z * d)
    rho = total / step.f2
    charge_now = float((step.quadrature.mass_weights * rho).sum())
    total = total * (step.n_electrons / charge_now)
    return total[None, :].copy()


class KerkerPreconditioner:
    """``F(q) q^2 / (q^2 + q0^2)`` by a periodic FFT of the box (``src/cdft/scf/mixing.py:35-56``)."""

    def __init__(self, shape, spacing: float, q0: float) -> None:
        self.shape = tuple(int(n) for n in shape)
        two_pi = 2.0 * math.pi
        kx = two_pi * np.fft.fftfreq(self.shape[0], d=spacing)
        ky = two_pi * np.fft.fftfreq(self.shape[1], d=spacing)
        kz = two_pi * np.fft.rfftfreq(self.shape[2], d=spacing)
        q2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
        self.filter = q2 / (q2 + q0 * q0)

    def __call__(self, residual):
        rows = np.atleast_2d(residual)
        out = np.empty_like(rows)
        for s, row in enumerate(rows):
            box = row.reshape(self.shape)
            out[s] = np.fft.irfftn(np.fft.rfftn(box) * self.filter, s=self.shape).reshape(-1)
        return out.reshape(np.shape(residual))


class LinearMixer:
    """(``src/cdft/scf/mixing.py:59-83``)"""

    def __init__(self, alpha):
        self.alpha = alpha

    def mix(self, n_in, n_out, iteration):
        return n_in + self.alpha * (n_out - n_in)


class PulayMixer:
    """(``src/cdft/scf/mixing.py:86-162``)"""

    def __init__(self, alpha, history, period, inner):
        self.alpha, self.history, self.period, self.inner = alpha, history, period, inner
        self.inputs, self.residuals = [], []

    def mix(self, n_in, n_out, iteration):
        residual = n_out - n_in
        self.inputs.append(n_in.copy())
        self.residuals.append(residual.copy())
        if len(self.inputs) > self.history:
            self.inputs.pop(0)
            self.residuals.pop(0)
        m = len(self.inputs)
        if m < 2 or iteration % self.period != 0:
            return n_in + self.alpha * residual
        gram = np.zeros((m, m))
        for i in range(m):
            for j in range(i, m):
                gram[i, j] = gram[j, i] = float(self.inner(self.residuals[i].reshape(-1), self.residuals[j].reshape(-1)))
        scale = float(gram.diagonal().max()) or 1.0
        gram = gram + 1.0e-12 * scale * np.eye(m)
        system = np.zeros((m + 1, m + 1))
        system[:m, :m] = gram
        system[:m, m] = -1.0
        system[m, :m] = 1.0
        rhs = np.zeros(m + 1)
        rhs[m] = 1.0
        coefficients = np.linalg.solve(system, rhs)[:m]
        mixed = np.zeros_like(n_in)
        for c, stored_in, stored_res in zip(coefficients, self.inputs, self.residuals):
            mixed = mixed + float(c) * (stored_in + self.alpha * stored_res)
        return mixed


def _make_mixer(system: System, alpha: float, inner, scheme: str):
    if scheme == "linear":
        return LinearMixer(alpha)
    period = system.pulay_period if scheme == "periodic_pulay" else 1
    return PulayMixer(alpha, system.history, period, inner)


class BoundReusePolicy:
    """(``src/cdft/scf/loop.py:94-170``)"""

    def __init__(self):
        self.bounds = None
        self.since_estimate = 0
        self.widening = 0.0
        self.top_fraction = float("nan")

    def decide(self, residual_rose, rung_changed, level_shift):
        if self.bounds is None:
            return "no carried interval"
        if level_shift:
            return "level shift"
        if rung_changed:
            return "rung changed"
        if residual_rose:
            return "residual rose"
        if self.since_estimate >= LANCZOS_REUSE_BACKSTOP:
            return "backstop"
        low, high = self.bounds
        if self.widening > LANCZOS_REUSE_MAX_WIDENING * (high - low):
            return "widening"
        if not self.top_fraction < BOUND_REUSE_RITZ_FRACTION:
            return "top fraction"
        return None

    def observe(self, info):
        b = info["bounds"]
        self.bounds = (float(b[0]), float(b[1])) if b else None
        self.top_fraction = float(info["top_fraction"])
        if info["source"] == "reused":
            self.since_estimate += 1
            self.widening += float(info["shift"])
        else:
            self.since_estimate = 0
            self.widening = 0.0


class _LevelShifted:
    """``H + Delta (1 - P_occ)`` (``src/cdft/scf/loop.py:553-589``)."""

    def __init__(self, inner, eigen, occupations, shift):
        self.inner = inner
        self.measure = inner.measure
        self.grid = inner.grid
        self.uses_divergence_form = True
        self.shift = shift
        mask = occupations.sum(axis=0) > 1e-12 if occupations is not None else None
        self.occupied = eigen.eigenvectors[mask] if (eigen is not None and mask is not None and mask.any()) else None
        self.apply_count = 0

    def apply(self, phi):
        self.apply_count += 1
        out = self.inner.apply(phi)
        if self.occupied is None:
            return out
        c = self.measure.cross(phi, self.occupied)
        return out + self.shift * (phi - c @ self.occupied)

    def spectral_bounds(self, **kw):
        lo, hi = self.inner.spectral_bounds(**kw)
        return lo, hi + self.shift


def solve_self_consistent(system: System, geometry=None, max_iterations=None, record_iterations=False):
    """(``src/cdft/scf/loop.py:255-550``); returns a dict of energies, eigenvalues and counters."""
    grid, factor, quadrature = geometry if geometry is not None else build_geometry(system)
    step = KohnShamStep(system, grid, factor, quadrature)
    mass = quadrature.mass_weights
    f2 = step.f2

    def norm_l1(delta):
        return float((mass * (np.abs(delta.sum(axis=0)) / f2)).sum())

    inner_weights = mass / f2 ** 2

    def inner(a, b):
        return (inner_weights * a * b).sum()

    n_in = initial_density(step)
    scheme = system.mixing
    mixer = _make_mixer(system, system.alpha, inner, scheme)
    ladder = [
        lambda: _make_mixer(system, system.alpha, inner, scheme),
        lambda: _make_mixer(system, 0.5 * system.alpha, inner, scheme),
        lambda: LinearMixer(0.5 * system.alpha),
        lambda: LinearMixer(0.5 * system.alpha),
    ]
    rung, level_shift, worsened = 0, 0.0, 0
    previous_residual = float("inf")
    initial_block = None
    eigen = None
    occupations = None
    energies, residuals, applications = [], [], []
    policy = BoundReusePolicy()
    previous_effective = None
    rung_changed = False
    converged = False
    limit = system.max_scf_iterations if max_iterations is None else max_iterations
    iteration = 0
    for iteration in range(1, limit + 1):
        p_in = step.potentials(n_in)
        hamiltonian = step.hamiltonian(p_in["effective"])
        if level_shift:
            hamiltonian = _LevelShifted(hamiltonian, eigen, occupations, level_shift)
        steps = None if initial_block is None else FILTER_STEPS_PER_ITERATION
        reason = policy.decide(worsened > 0, rung_changed, bool(level_shift))
        hint = None
        if reason is None and previous_effective is not None:
            hint = (policy.bounds[0], policy.bounds[1], float(np.abs(p_in["effective"] - previous_effective).max()))
        eigen, info = step.diagonalise(hamiltonian, initial=initial_block, max_iterations=steps, bounds=hint)
        policy.observe(info)
        previous_effective = p_in["effective"]
        rung_changed = False
        applications.append(hamiltonian.apply_count)
        initial_block = eigen.eigenvectors
        occupations = step.occupy(eigen.eigenvalues)
        n_out, rho_out = step.output_density(eigen, occupations)
        p_out = step.potentials(n_out)
        terms = step.energy_terms(eigen, occupations, rho_out, p_in, p_out)
        residual = n_out - n_in
        res_norm = norm_l1(residual)
        n_next = mixer.mix(n_in, n_out, iteration)
        energies.append(terms["total"])
        residuals.append(res_norm)
        de = abs(energies[-1] - energies[-2]) if len(energies) > 1 else float("inf")
        if iteration >= system.min_scf_iterations and de < system.energy_tol and res_norm < system.density_tol:
            converged = True
            break
        worsened = worsened + 1 if res_norm > previous_residual else 0
        previous_residual = res_norm
        if worsened >= 3 and rung + 1 < len(ladder):
            rung += 1
            mixer = ladder[rung]()
            if rung == 3:
                level_shift = 0.5
            worsened = 0
            rung_changed = True
            n_next = n_in + 0.5 * system.alpha * residual
        n_in = n_next
    final_h = step.hamiltonian(p_in["effective"])
    eigen, _ = step.diagonalise(final_h, initial=eigen.eigenvectors)
    occupations = step.occupy(eigen.eigenvalues)
    n_out, rho_out = step.output_density(eigen, occupations)
    p_out = step.potentials(n_out)
    terms = step.energy_terms(eigen, occupations, rho_out, p_in, p_out)
    return {
        "energies": terms, "eigenvalues": eigen.eigenvalues.copy(), "scf_iterations": iteration,
        "converged": converged and eigen.converged, "applications": float(sum(applications) + final_h.apply_count),
        "energy_history": energies, "residual_history": residuals, "density": n_out,
        "charge": float((mass * rho_out).sum()),
    }


def solve_noninteracting(system: System, geometry=None):
    """(``src/cdft/scf/noninteracting.py:118-330``) for the cusp-factorised path."""
    grid, factor, quadrature = geometry if geometry is not None else build_geometry(system)
    ham = CuspHamiltonian(grid, factor, quadrature)
    n_states = max(1, int(-(-system.n_electrons // 2.0)))
    generator = make_generator(system.seed)
    solver = ChebyshevFilteredSubspace(grid.n_points, degree=system.chebyshev_degree, n_extra_states=system.n_extra_states,
                                       max_iterations=system.max_eigen_iterations, residual_tol=system.residual_tol,
                                       ritz_stop=True)
    result = solver.solve(ham, n_states, generator=generator)
    occ = aufbau_occupations(n_states, system.n_electrons)
    kinetic = float(ham.kinetic_energy(result.eigenvectors, occ[0]))
    band = float((occ[0] * result.eigenvalues).sum())
    ion_ion = nuclear_repulsion(system.charges, system.positions)
    external = band - kinetic
    return {"total": kinetic + external + ion_ion, "kinetic": kinetic, "eigenvalues": result.eigenvalues.copy(),
            "iterations": result.n_iterations, "converged": result.converged, "applications": float(ham.apply_count)}


# ---- the benchmark systems ----

def h_atom(points_per_edge: int = 33, half_box: float = 4.0) -> System:
    """Bare H, cubic box ``2 half_box`` with ``points_per_edge`` points (h = 2 half_box / (ppe - 1))."""
    edge = 2.0 * half_box
    return System(charges=(1.0,), positions=((0.0, 0.0, 0.0),), n_electrons=1.0, box_lengths=(edge,) * 3,
                  spacing=edge / (points_per_edge - 1), anchor=(0.0, 0.0, 0.0))


def he_lda(spacing: float = 0.25, edge: float = 16.0, mixing: str = "linear", alpha: float = 0.3) -> System:
    """He, VWN-LDA, cubic box ``edge``, spacing ``spacing`` (65^3 at 0.25 / 16)."""
    return System(charges=(2.0,), positions=((0.0, 0.0, 0.0),), n_electrons=2.0, box_lengths=(edge,) * 3,
                  spacing=spacing, functional="lda_vwn", mixing=mixing, alpha=alpha)


def h2_pbe(bond: float = 1.4, spacing: float = 0.20, box=(16.0, 16.0, 18.0), degree: int = 16,
           mixing: str = "periodic_pulay") -> System:
    """H2 along z, PBE, un-anchored lattice (``derive_grid=False``)."""
    half = bond / 2.0
    return System(charges=(1.0, 1.0), positions=((0.0, 0.0, -half), (0.0, 0.0, half)), n_electrons=2.0,
                  box_lengths=tuple(box), spacing=spacing, functional="pbe", chebyshev_degree=degree, mixing=mixing)


def h2_plus(bond: float = 2.0, spacing: float = 0.25, transverse: float = 12.0) -> System:
    """H2+ along z, bare nuclei, box ``transverse^2 x (bond + 12)``, un-anchored lattice."""
    half = bond / 2.0
    return System(charges=(1.0, 1.0), positions=((0.0, 0.0, -half), (0.0, 0.0, half)), n_electrons=1.0,
                  box_lengths=(transverse, transverse, bond + 12.0), spacing=spacing)
