"""The cusp-factorised Hamiltonian, the measure and the Coulomb-cutoff Poisson solver (oracle).

Restates ``src/cdft/operators/hamiltonian.py`` (CuspFactoredHamiltonian, _lanczos_bounds),
``src/cdft/eigen/measure.py`` (Measure) and ``src/cdft/operators/poisson.py`` (CoulombCutoffPoisson).
"""

from __future__ import annotations

import math

import numpy as np

from .geometry import CuspFactor, CuspQuadrature
from .grid import Grid, weighted_divergence
from .rng import seeded_randn


class Measure:
    """``<a,b> = sum_r q(r) a(r) b(r)`` (``src/cdft/eigen/measure.py:18-82``)."""

    def __init__(self, grid: Grid, quadrature: np.ndarray) -> None:
        self.grid = grid
        self.q = quadrature

    def inner(self, a, b):
        return (a * b * self.q).sum(axis=-1)

    def norm(self, a):
        return np.sqrt(np.maximum(self.inner(a, a), 0.0))

    def gram(self, block):
        flat = block.reshape(-1, self.grid.n_points)
        return (flat * self.q) @ flat.T

    def cross(self, left, right):
        a = left.reshape(-1, self.grid.n_points)
        b = right.reshape(-1, self.grid.n_points)
        return (a * self.q) @ b.T


class CuspHamiltonian:
    """``A = f^-1 H f`` in staggered divergence form (``src/cdft/operators/hamiltonian.py:178-396``)."""

    def __init__(self, grid: Grid, factor: CuspFactor, quadrature: CuspQuadrature, extra_potential=None, bare=None):
        self.grid = grid
        self.factor = factor
        self.quadrature = quadrature
        if bare is None and quadrature is None:
            # No quadrature: W pointwise, measure f^2 h^3 (hamiltonian.py:228-231).
            bare = (factor.transformed_potential, 1.0 / factor.weight, factor.weight * grid.volume_element)
        elif bare is None:
            bare = quadrature.bare_operator_terms()
        self.bare_potential, self.inverse_weight, q = bare
        self.measure = Measure(grid, q)
        self.potential = self.bare_potential if extra_potential is None else self.bare_potential + extra_potential
        self.faces = factor.face_weights(grid.fd_order)
        self.apply_count = 0
        self.uses_divergence_form = True

    def kinetic_apply(self, phi):
        """``(1/2 w) sum_d D_d^T[f^2_face D_d phi]`` (hamiltonian.py:303-318)."""
        box = phi.reshape(*phi.shape[:-1], *self.grid.shape)
        div = weighted_divergence(box, self.faces, self.grid.spacing, self.grid.fd_order)
        return div.reshape(*phi.shape[:-1], self.grid.n_points) * 0.5 * self.inverse_weight

    def apply_with_potential(self, phi, potential):
        return self.kinetic_apply(phi) + phi * potential

    def apply(self, phi):
        self.apply_count += 1
        return self.apply_with_potential(phi, self.potential)

    def spectral_bounds(self, steps=12, safety=1.02, generator=None):
        start = seeded_randn(self.grid.n_points, generator)
        return lanczos_bounds(self.apply, start, self.measure.inner, self.measure.norm, steps, safety)

    def external_energy_parts(self, rho):
        """``((1/2)Q[f^2 grad rho.grad u], Q[f^2 rho W])`` (hamiltonian.py:360-378)."""
        q = self.quadrature
        rho_node = q.interpolate(rho)
        grad_rho_node = q.interpolate_gradient(rho)
        cross_node = q.f2 * (grad_rho_node * q.grad_u).sum(axis=0)
        cross_grid = self.factor.weight * (self.grid.gradient(rho) * self.factor.grad_u).sum(axis=0)
        cross = 0.5 * q.integrate(cross_node, cross_grid)
        potential = q.integrate(q.f2 * rho_node * q.transformed_potential,
                                self.factor.weight * rho * self.factor.transformed_potential)
        return cross, potential

    def kinetic_energy(self, phi, occupations):
        """(hamiltonian.py:331-358)"""
        kinetic_form = self.measure.inner(phi, self.kinetic_apply(phi))
        first = (occupations * kinetic_form).sum()
        rho = (occupations[..., None] * phi ** 2).sum(axis=-2)
        cross, potential = self.external_energy_parts(rho)
        return first - cross - potential

    def external_energy_direct(self, rho):
        cross, potential = self.external_energy_parts(rho)
        return cross + 2.0 * potential


def lanczos_bounds(apply, start, inner, norm, steps, safety):
    """Rigorous Lanczos enclosure (``src/cdft/operators/hamiltonian.py:29-89``)."""
    v = start / norm(start)
    alphas, betas = [], []
    v_prev = np.zeros_like(v)
    beta = 0.0
    for _ in range(steps):
        w = apply(v)
        alpha = inner(v, w)
        w = w - alpha * v - beta * v_prev
        w = w - inner(w, v) * v - inner(w, v_prev) * v_prev
        beta = norm(w)
        alphas.append(float(alpha))
        betas.append(float(beta))
        v_prev, v = v, w / beta
    for index, value in enumerate(betas):
        if value < 1e-12:
            del alphas[index + 1:], betas[index + 1:]
            break
    size = len(alphas)
    tri = np.zeros((size, size))
    for i in range(size):
        tri[i, i] = alphas[i]
        if i + 1 < size:
            tri[i, i + 1] = tri[i + 1, i] = betas[i]
    ritz = np.linalg.eigvalsh(tri)
    residual = betas[-1] if betas else 0.0
    lo = float(ritz[0]) - residual
    hi = float(ritz[-1]) + residual
    centre = 0.5 * (hi + lo)
    half = 0.5 * (hi - lo) * safety
    return centre - half, centre + half


def fft_friendly(n: int) -> int:
    """Next 2,3,5-smooth integer (``src/cdft/operators/poisson.py:110-120``)."""
    candidate = n
    while True:
        residue = candidate
        for prime in (2, 3, 5):
            while residue % prime == 0:
                residue //= prime
        if residue == 1:
            return candidate
        candidate += 1


class CoulombCutoffPoisson:
    """Zero-padded FFT with the truncated kernel (``src/cdft/operators/poisson.py:21-107``)."""

    def __init__(self, grid: Grid, pad_factor: float = 2.5) -> None:
        self.grid = grid
        self.padded_shape = tuple(fft_friendly(int(math.ceil(pad_factor * n))) for n in grid.shape)
        self.cutoff_radius = 0.5 * min(n * grid.spacing for n in self.padded_shape)
        h = grid.spacing
        n0, n1, n2 = self.padded_shape
        kx = 2.0 * math.pi * np.fft.fftfreq(n0, d=h)
        ky = 2.0 * math.pi * np.fft.fftfreq(n1, d=h)
        kz = 2.0 * math.pi * np.fft.rfftfreq(n2, d=h)
        g_sq = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
        g = np.sqrt(g_sq)
        radius = self.cutoff_radius
        with np.errstate(divide="ignore", invalid="ignore"):
            kernel = np.where(g_sq > 0.0, 4.0 * math.pi * (1.0 - np.cos(g * radius)) / np.maximum(g_sq, 1e-300),
                              2.0 * math.pi * radius ** 2)
        self.kernel = kernel
        #: None: numpy's FFT (the checker's default). A thread count: scipy's multithreaded FFT of the
        #: same transforms, used only to time the CPU path on all host threads.
        self.fft_workers = None

    def solve(self, density):
        if density.ndim != 1:
            raise ValueError("expected a total density of shape (n_points,)")
        box = density.reshape(self.grid.shape)
        padded = np.zeros(self.padded_shape)
        padded[: box.shape[0], : box.shape[1], : box.shape[2]] = box
        if self.fft_workers:
            import scipy.fft as sfft

            transformed = sfft.rfftn(padded, s=self.padded_shape, workers=self.fft_workers)
            potential = sfft.irfftn(transformed * self.kernel, s=self.padded_shape, workers=self.fft_workers)
        else:
            transformed = np.fft.rfftn(padded, s=self.padded_shape)
            potential = np.fft.irfftn(transformed * self.kernel, s=self.padded_shape)
        return potential[: box.shape[0], : box.shape[1], : box.shape[2]].reshape(-1).copy()


def analytic_gaussian_potential(radius, sigma: float, charge: float = 1.0):
    """``Q erf(r/(sqrt2 sigma))/r`` (``src/cdft/operators/poisson.py:123-130``)."""
    from scipy.special import erf
    scaled = radius / (math.sqrt(2.0) * sigma)
    limit = charge * math.sqrt(2.0 / math.pi) / sigma
    return np.where(radius > 1e-12, charge * erf(scaled) / np.maximum(radius, 1e-30), limit)
