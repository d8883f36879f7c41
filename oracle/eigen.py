"""Rayleigh--Ritz, residuals and the Chebyshev-filtered subspace iteration (oracle).

Restates ``src/cdft/eigen/rayleigh_ritz.py`` and ``src/cdft/eigen/chefsi.py``.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg

from .rng import seeded_randn

BOUND_REUSE_RITZ_FRACTION = 0.9


def orthonormalise(block, measure):
    """Cholesky (eigh fallback) orthonormalisation (``src/cdft/eigen/rayleigh_ritz.py:51-72``)."""
    flat = block.reshape(-1, measure.grid.n_points)
    gram = measure.gram(flat)
    try:
        chol = np.linalg.cholesky(gram)
    except np.linalg.LinAlgError:
        evals, evecs = np.linalg.eigh(0.5 * (gram + gram.T))
        keep = evals > evals[-1] * 1e-14
        if not keep.any():
            raise ValueError("the orbital block collapsed to rank zero") from None
        scaled = evecs[:, keep] / np.sqrt(evals[keep])
        return scaled.T @ flat
    return scipy.linalg.solve_triangular(chol, flat, lower=True)


def rayleigh_ritz(hamiltonian, block, measure):
    """(``src/cdft/eigen/rayleigh_ritz.py:75-102``) -> (evals, vectors, orth_error)"""
    basis = orthonormalise(block, measure)
    subspace = measure.cross(basis, hamiltonian.apply(basis))
    subspace = 0.5 * (subspace + subspace.T)
    evals, rotation = np.linalg.eigh(subspace)
    vectors = rotation.T @ basis
    gram = measure.gram(vectors)
    error = float(np.abs(gram - np.eye(gram.shape[0])).max())
    return evals, vectors, error


def residual_norms(hamiltonian, evals, vectors, measure):
    """(``src/cdft/eigen/rayleigh_ritz.py:105-115``)"""
    applied = hamiltonian.apply(vectors)
    return measure.norm(applied - evals[:, None] * vectors)


def chebyshev_coefficients(degree, lower, upper, spectrum_min):
    """Rows ``(c, a_k, b_k)`` of the scaled recurrence (``src/cdft/eigen/chefsi.py:116-136``)."""
    if upper <= lower:
        raise ValueError(f"filter interval is empty: lower={lower}, upper={upper}")
    e = 0.5 * (upper - lower)
    c = 0.5 * (upper + lower)
    sigma = e / (spectrum_min - c)
    sigma1 = sigma
    rows = [(c, sigma1 / e, 0.0)]
    for _ in range(2, degree + 1):
        sigma2 = 1.0 / (2.0 / sigma1 - sigma)
        rows.append((c, 2.0 * sigma2 / e, sigma * sigma2))
        sigma = sigma2
    return rows


def chebyshev_filter(hamiltonian, block, degree, lower, upper, spectrum_min):
    """The scaled three-term Chebyshev filter (``src/cdft/eigen/chefsi.py:81-113``)."""
    if upper <= lower:
        raise ValueError(f"filter interval is empty: lower={lower}, upper={upper}")
    e = 0.5 * (upper - lower)
    c = 0.5 * (upper + lower)
    sigma = e / (spectrum_min - c)
    sigma1 = sigma
    applied = hamiltonian.apply(block)
    y = (applied - c * block) * (sigma1 / e)
    previous = block
    for _ in range(2, degree + 1):
        sigma2 = 1.0 / (2.0 / sigma1 - sigma)
        applied = hamiltonian.apply(y)
        y_new = (applied - c * y) * (2.0 * sigma2 / e) - (sigma * sigma2) * previous
        previous, y = y, y_new
        sigma = sigma2
    return y


class EigenResult:
    def __init__(self, eigenvalues, eigenvectors, residuals, n_iterations, converged):
        self.eigenvalues = eigenvalues
        self.eigenvectors = eigenvectors
        self.residuals = residuals
        self.n_iterations = n_iterations
        self.converged = converged


def _fraction(value, low, high):
    width = high - low
    return (value - low) / width if width > 0.0 else float("inf")


class ChebyshevFilteredSubspace:
    """CheFSI (``src/cdft/eigen/chefsi.py:408-585``)."""

    def __init__(self, n_points, *, degree, n_extra_states, extra_states_fraction=0.2, lanczos_steps=12,
                 bound_safety=1.02, max_iterations=300, residual_tol=1e-8, cross_check_tol=1e-8, ritz_stop=True):
        self.n_points = n_points
        self.degree = degree
        self.n_extra_states = n_extra_states
        self.extra_states_fraction = extra_states_fraction
        self.lanczos_steps = lanczos_steps
        self.bound_safety = bound_safety
        self.max_iterations = max_iterations
        self.residual_tol = residual_tol
        self.cross_check_tol = cross_check_tol
        self.ritz_stop = ritz_stop
        self.history = []
        self.spectral_bounds = None
        self.bounds_source = "unset"
        self.bounds_shift = 0.0
        self.top_ritz_fraction = float("nan")

    def solve(self, hamiltonian, n_states, initial=None, generator=None, bounds=None):
        measure = hamiltonian.measure
        extra = max(self.n_extra_states, int(self.extra_states_fraction * n_states))
        m = min(n_states + extra, self.n_points)
        if initial is None:
            block = seeded_randn((m, self.n_points), generator)
        else:
            block = initial.reshape(-1, self.n_points)
            if block.shape[0] < m:
                pad = seeded_randn((m - block.shape[0], self.n_points), generator)
                block = np.concatenate([block, pad], axis=0)

        def lanczos():
            return hamiltonian.spectral_bounds(steps=self.lanczos_steps, safety=self.bound_safety, generator=generator)

        if bounds is None:
            spectrum_min, spectrum_max = lanczos()
            self.bounds_source = "lanczos"
            self.bounds_shift = 0.0
        evals, vectors, _ = rayleigh_ritz(hamiltonian, block, measure)
        converged = False
        iteration = 0
        residual = residual_norms(hamiltonian, evals, vectors, measure)
        previous = evals.copy()
        stable = 0
        self.eigenvalue_drift = float("inf")
        self.stop_reason = "iteration limit"
        weak_form = self.ritz_stop and bool(getattr(hamiltonian, "uses_divergence_form", False))
        eigenvalue_tol = 0.1 * self.cross_check_tol
        next_lower = float(evals[min(m, evals.shape[0]) - 1])
        if bounds is not None:
            shift = float(bounds[2])
            spectrum_min, spectrum_max = bounds[0] - shift, bounds[1] + shift
            self.bounds_source = "reused"
            self.bounds_shift = shift
        top_fraction = float("-inf")
        for iteration in range(1, self.max_iterations + 1):
            lower = next_lower
            fraction = _fraction(lower, spectrum_min, spectrum_max)
            if self.bounds_source == "reused" and not fraction < BOUND_REUSE_RITZ_FRACTION:
                spectrum_min, spectrum_max = lanczos()
                self.bounds_source = "lanczos (reuse rejected)"
                fraction = _fraction(lower, spectrum_min, spectrum_max)
            top_fraction = max(top_fraction, fraction)
            lower = min(max(lower, spectrum_min + 1e-8), spectrum_max - 1e-8)
            filtered = chebyshev_filter(hamiltonian, vectors, self.degree, lower, spectrum_max, spectrum_min)
            evals, vectors, orth = rayleigh_ritz(hamiltonian, filtered, measure)
            residual = residual_norms(hamiltonian, evals, vectors, measure)
            worst = float(residual[:n_states].max())
            drift = float(np.abs(evals[:n_states] - previous[:n_states]).max())
            next_lower = float(evals[min(m, evals.shape[0]) - 1])
            previous = evals.copy()
            self.eigenvalue_drift = drift
            self.history.append({"iteration": iteration, "residual": worst, "orthonormality": orth, "drift": drift})
            if worst < self.residual_tol:
                converged = True
                self.stop_reason = "residual below residual_tol"
                break
            stable = stable + 1 if (weak_form and drift < eigenvalue_tol) else 0
            if stable >= 2:
                converged = True
                self.stop_reason = "Ritz values stable on the weak-form path"
                break
        self.spectral_bounds = (spectrum_min, spectrum_max)
        self.top_ritz_fraction = top_fraction
        return EigenResult(evals[:n_states], vectors[:n_states], residual[:n_states], iteration, converged)
