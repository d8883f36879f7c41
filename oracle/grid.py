"""Uniform grid, finite-difference weights and the staggered divergence stencil (oracle).

Restates ``src/cdft/grid.py`` (box construction, flat<->box maps, gradient),
``src/cdft/operators/laplacian.py`` (central weights) and ``src/cdft/operators/divergence.py``
(staggered weights and the eager weighted divergence).
"""

from __future__ import annotations

import math
from fractions import Fraction
from functools import lru_cache

import numpy as np


def _solve_rational(matrix: list[list[Fraction]], rhs: list[Fraction]) -> list[Fraction]:
    """Gauss-Jordan elimination in exact rational arithmetic."""
    size = len(rhs)
    matrix = [row[:] for row in matrix]
    rhs = rhs[:]
    for col in range(size):
        pivot = next(r for r in range(col, size) if matrix[r][col] != 0)
        matrix[col], matrix[pivot] = matrix[pivot], matrix[col]
        rhs[col], rhs[pivot] = rhs[pivot], rhs[col]
        inv = matrix[col][col]
        matrix[col] = [v / inv for v in matrix[col]]
        rhs[col] = rhs[col] / inv
        for row in range(size):
            if row == col or matrix[row][col] == 0:
                continue
            factor = matrix[row][col]
            matrix[row] = [a - factor * b for a, b in zip(matrix[row], matrix[col])]
            rhs[row] = rhs[row] - factor * rhs[col]
    return rhs


@lru_cache(maxsize=None)
def fd_coefficients(derivative: int, accuracy: int) -> tuple[float, ...]:
    """Central weights for d^n/dx^n, offsets -hw..hw (``src/cdft/operators/laplacian.py:36-75``)."""
    hw = accuracy // 2 + (derivative - 1) // 2
    offsets = list(range(-hw, hw + 1))
    matrix = [[Fraction(o) ** m for o in offsets] for m in range(len(offsets))]
    rhs = [Fraction(0)] * len(offsets)
    rhs[derivative] = Fraction(math.factorial(derivative))
    return tuple(float(v) for v in _solve_rational(matrix, rhs))


@lru_cache(maxsize=None)
def staggered_coefficients(accuracy: int) -> tuple[float, ...]:
    """Face-derivative weights, k = -p..p-1 (``src/cdft/operators/divergence.py:31-74``)."""
    half = accuracy // 2
    positions = [Fraction(2 * k + 1, 2) for k in range(-half, half)]
    matrix = [[p ** m for p in positions] for m in range(len(positions))]
    rhs = [Fraction(0)] * len(positions)
    rhs[1] = Fraction(1)
    return tuple(float(v) for v in _solve_rational(matrix, rhs))


@lru_cache(maxsize=None)
def gauss_legendre(order: int) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Legendre nodes/weights on [-1, 1] (the rule of ``src/cdft/operators/gauss_legendre.py``).

    Newton iteration on the Legendre recurrence from the Tricomi initial guess, then the same
    symmetrisation and normalisation as the reference; agrees with it to the last bit or two.
    """
    n = int(order)
    nodes = np.cos(np.pi * (np.arange(1, n + 1) - 0.25) / (n + 0.5))
    for _ in range(100):
        p0 = np.ones_like(nodes)
        p1 = nodes.copy()
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * nodes * p1 - (k - 1) * p0) / k
        if n == 1:
            p0, p1 = np.ones_like(nodes), nodes.copy()
        dp = n * (nodes * p1 - p0) / (nodes * nodes - 1.0)
        step = p1 / dp
        nodes = nodes - step
        if np.max(np.abs(step)) < 1e-17:
            break
    p0 = np.ones_like(nodes)
    p1 = nodes.copy()
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * nodes * p1 - (k - 1) * p0) / k
    if n == 1:
        p0, p1 = np.ones_like(nodes), nodes.copy()
    dp = n * (nodes * p1 - p0) / (nodes * nodes - 1.0)
    weights = 2.0 / ((1.0 - nodes * nodes) * dp * dp)
    order_idx = np.argsort(nodes)
    nodes, weights = nodes[order_idx], weights[order_idx]
    weights = (weights + weights[::-1]) / 2.0
    nodes = (nodes - nodes[::-1]) / 2.0
    weights = weights * (2.0 / weights.sum())
    return nodes, weights


class Grid:
    """A full-box uniform grid with a zero (Dirichlet) halo (``src/cdft/grid.py:480-760``)."""

    def __init__(self, shape, spacing: float, origin, fd_order: int = 8, gradient_order: int = 8):
        self.shape = tuple(int(n) for n in shape)
        self.spacing = float(spacing)
        self.origin = tuple(float(o) for o in origin)
        self.fd_order = fd_order
        self.gradient_order = gradient_order
        self.n_points = self.shape[0] * self.shape[1] * self.shape[2]

    @classmethod
    def box(cls, lengths, spacing: float, anchor=None, fd_order: int = 8) -> "Grid":
        """``UniformGrid.from_config`` for ``DomainMode.BOX`` / ``BoundaryMode.ZERO`` (grid.py:580-605)."""
        h = float(spacing)
        counts = tuple(max(int(round(length / h)) + 1, 1) for length in lengths)
        h = lengths[0] / (counts[0] - 1) if counts[0] > 1 else h
        if anchor is None:
            origin = tuple(-h * round(0.5 * length / h) for length in lengths)
        else:
            origin = tuple(float(a) - h * round((float(a) + 0.5 * length) / h) for a, length in zip(anchor, lengths))
        return cls(counts, h, origin, fd_order=fd_order)

    @property
    def volume_element(self) -> float:
        return self.spacing ** 3

    def axes(self):
        return [self.origin[d] + np.arange(self.shape[d], dtype=np.float64) * self.spacing for d in range(3)]

    def points(self) -> np.ndarray:
        """(N, 3) coordinates in C order, ``origin + index * h`` (grid.py:656-659)."""
        idx = np.indices(self.shape).reshape(3, -1).T.astype(np.float64)
        return np.asarray(self.origin) + idx * self.spacing

    def box_of(self, field: np.ndarray) -> np.ndarray:
        return field.reshape(*field.shape[:-1], *self.shape)

    def integrate(self, field: np.ndarray):
        return (field * self.volume_element).sum(axis=-1)

    def _padded(self, field: np.ndarray, pad: int) -> np.ndarray:
        box = self.box_of(field)
        out = np.zeros((*box.shape[:-3], *(n + 2 * pad for n in self.shape)))
        out[..., pad:pad + self.shape[0], pad:pad + self.shape[1], pad:pad + self.shape[2]] = box
        return out

    def partial_derivative(self, field: np.ndarray, axis: int) -> np.ndarray:
        """One first-derivative component, zero halo (laplacian.py:111-130, grid.py:745-758)."""
        coeffs = fd_coefficients(1, self.gradient_order)
        hw = len(coeffs) // 2
        pad = max(self.fd_order // 2, self.gradient_order // 2)
        padded = self._padded(field, pad)
        scale = 1.0 / self.spacing
        acc = None
        for index, c in enumerate(coeffs):
            if c == 0.0:
                continue
            sl = [slice(pad, pad + n) for n in self.shape]
            sl[axis] = slice(pad + index - hw, pad + index - hw + self.shape[axis])
            term = padded[(Ellipsis, *sl)]
            acc = term * (c * scale) if acc is None else acc + term * (c * scale)
        return acc.reshape(*field.shape[:-1], self.n_points)

    def gradient(self, field: np.ndarray) -> np.ndarray:
        """``(..., 3, N)`` gradient (grid.py:740-743)."""
        return np.stack([self.partial_derivative(field, d) for d in range(3)], axis=-2)


def _pad_axis(box: np.ndarray, axis: int, width: int) -> np.ndarray:
    shape = list(box.shape)
    shape[box.ndim - 3 + axis] += 2 * width
    out = np.zeros(shape)
    index = [slice(None)] * 3
    index[axis] = slice(width, width + box.shape[box.ndim - 3 + axis])
    out[(Ellipsis, *index)] = box
    return out


def _slice_along(t: np.ndarray, axis: int, start: int, length: int) -> np.ndarray:
    index = [slice(None)] * 3
    index[axis] = slice(start, start + length)
    return t[(Ellipsis, *index)]


def weighted_divergence(box: np.ndarray, face_weights, spacing: float, accuracy: int) -> np.ndarray:
    """``sum_d D_d^T [w_d D_d phi]`` on a box (``src/cdft/operators/divergence.py:99-197``).

    ``box`` is ``(..., nx, ny, nz)``; ``face_weights[d]`` has the box shape extended by
    ``accuracy`` along axis ``d`` and is indexed from face ``-accuracy/2``.
    """
    half = accuracy // 2
    coeffs = staggered_coefficients(accuracy)
    scale = 1.0 / spacing
    shape = box.shape[-3:]
    out = None
    for axis in range(3):
        padded = _pad_axis(box, axis, accuracy)
        faces = None
        for index, c in enumerate(coeffs):
            start = accuracy - half + 1 + (index - half)
            term = _slice_along(padded, axis, start, shape[axis] + accuracy)
            faces = term * (c * scale) if faces is None else faces + term * (c * scale)
        faces = faces * face_weights[axis]
        term_sum = None
        for index, c in enumerate(coeffs):
            start = half - 1 - (index - half)
            term = _slice_along(faces, axis, start, shape[axis])
            term_sum = term * (c * scale) if term_sum is None else term_sum + term * (c * scale)
        out = term_sum if out is None else out + term_sum
    return out
