"""Cusp factor, cusp-aware quadrature and the Hartree-split geometry (oracle).

Restates ``src/cdft/operators/cusp.py`` (CuspFactor), ``src/cdft/operators/quadrature.py``
(CuspQuadrature, lagrange_weights, sphere rules, partition, far weights, the CSR interpolant and
its transpose) and ``src/cdft/scf/step.py:111-165`` (StepGeometry).
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sparse
from scipy.special import erfc

from .grid import Grid, gauss_legendre


class CuspFactor:
    """``f = exp(-sum_a Z_a |r - R_a|)`` on a grid (``src/cdft/operators/cusp.py:33-214``)."""

    average_radius_cells = 2.0
    average_quadrature = 4

    def __init__(self, grid: Grid, charges, positions) -> None:
        self.grid = grid
        self.charges = tuple(float(z) for z in charges)
        self.positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        self.is_identity = len(self.charges) == 0
        n = grid.n_points
        points = grid.points()
        u = np.zeros(n)
        grad_u = np.zeros((3, n))
        for index, z in enumerate(self.charges):
            delta = points - self.positions[index]
            distance = np.sqrt((delta * delta).sum(axis=-1))
            u += z * distance
            safe = np.maximum(distance, 1.0e-30)
            on = distance <= 1.0e-12
            unit = np.where((~on)[:, None], delta / safe[:, None], 0.0)
            grad_u += z * unit.T
        self.u = u
        self.grad_u = grad_u
        self.weight = np.exp(-2.0 * u)
        self.transformed_potential = self._build_potential()
        self._faces = {}

    def _build_potential(self) -> np.ndarray:
        """``W = -|grad u|^2/2``, 4^3 Gauss--Legendre cell average within 2h (cusp.py:94-145)."""
        potential = -0.5 * (self.grad_u * self.grad_u).sum(axis=0)
        if self.is_identity:
            return potential
        grid = self.grid
        points = grid.points()
        h = grid.spacing
        reach = self.average_radius_cells * h
        near = np.zeros(grid.n_points, dtype=bool)
        for atom in range(len(self.charges)):
            d = points - self.positions[atom]
            near |= np.sqrt((d * d).sum(axis=-1)) <= reach
        count = int(near.sum())
        if count == 0:
            return potential
        gl_nodes, gl_weights = gauss_legendre(self.average_quadrature)
        offsets = [float(x) * 0.5 * h for x in gl_nodes]
        weights = [float(w) * 0.5 for w in gl_weights]
        selected = points[near]
        mean_square = np.zeros(count)
        mean_vector = np.zeros((count, 3))
        total = 0.0
        for ix, wx in zip(offsets, weights):
            for iy, wy in zip(offsets, weights):
                for iz, wz in zip(offsets, weights):
                    weight = float(wx * wy * wz)
                    total += weight
                    shift = np.array([ix, iy, iz])
                    gradient = np.zeros_like(selected)
                    for atom, z in enumerate(self.charges):
                        delta = (selected + shift) - self.positions[atom]
                        distance = np.maximum(np.sqrt((delta * delta).sum(axis=-1, keepdims=True)), 1.0e-300)
                        gradient = gradient + z * delta / distance
                    mean_square = mean_square + weight * (gradient * gradient).sum(axis=-1)
                    mean_vector = mean_vector + weight * gradient
        potential = potential.copy()
        potential[near] = -0.5 * mean_square / total
        self.grad_u = self.grad_u.copy()
        self.grad_u[:, near] = (mean_vector / total).T
        self.n_cell_averaged = count
        return potential

    def face_weights(self, accuracy: int):
        """``f^2`` at the staggered faces of each axis, from face ``-p`` (cusp.py:168-214)."""
        if accuracy in self._faces:
            return self._faces[accuracy]
        grid = self.grid
        half = accuracy // 2
        h = grid.spacing
        out = []
        for axis in range(3):
            sizes = list(grid.shape)
            sizes[axis] += accuracy
            coords = []
            for d in range(3):
                index = np.arange(sizes[d], dtype=np.float64)
                if d == axis:
                    index = index - half + 0.5
                coords.append(grid.origin[d] + index * h)
            mesh = np.meshgrid(*coords, indexing="ij")
            u = np.zeros(sizes)
            for atom, z in enumerate(self.charges):
                squared = 0
                for d in range(3):
                    squared = squared + (mesh[d] - self.positions[atom, d]) ** 2
                u = u + z * np.sqrt(squared)
            if float(u.max()) > 354.0:
                raise ValueError("the cusp weight exp(-2u) underflows float64 on this domain")
            out.append(np.exp(-2.0 * u))
        self._faces[accuracy] = tuple(out)
        return self._faces[accuracy]

    def density(self, phi: np.ndarray, occupations: np.ndarray) -> np.ndarray:
        """``n = sum_i f_i f^2 phi_i^2`` (cusp.py:325-331)."""
        return (occupations[..., None] * phi ** 2).sum(axis=-2) * self.weight


def lagrange_weights(t: np.ndarray, degree: int) -> np.ndarray:
    """Degree-``degree`` Lagrange basis at offset ``t`` (``src/cdft/operators/quadrature.py:56-93``)."""
    half = degree // 2
    offsets = np.arange(-half, -half + degree + 1, dtype=np.float64)
    x = t[:, None] - offsets[None, :]
    weights = np.ones_like(x)
    for j in range(degree + 1):
        for m in range(degree + 1):
            if m == j:
                continue
            weights[:, j] = weights[:, j] * x[:, m] / float(j - m)
    return weights


def sphere_rule(centre, radius_sphere: float, spacing: float, radial_order: int, node_spacing: float):
    """Composite GL radius x product angular rule (``src/cdft/operators/quadrature.py:123-182``)."""
    n_panels = max(2, int(math.ceil(radius_sphere / spacing)))
    edges = np.linspace(0.0, radius_sphere, n_panels + 1)
    gl_nodes, gl_weights = gauss_legendre(radial_order)
    points, weights = [], []
    n_radial = 0
    for lo, hi in zip(edges[:-1], edges[1:]):
        mid, halfw = 0.5 * (hi + lo), 0.5 * (hi - lo)
        for node, weight in zip(gl_nodes, gl_weights):
            r = mid + halfw * node
            wr = halfw * weight * r * r
            n_theta = max(4, int(math.ceil(math.sqrt(2.0 * math.pi) * r / (node_spacing * spacing))))
            n_phi = 2 * n_theta
            cos_nodes, cos_weights = gauss_legendre(n_theta)
            phis = 2.0 * math.pi * (np.arange(n_phi) + 0.5) / n_phi
            sin_theta = np.sqrt(np.clip(1.0 - cos_nodes ** 2, 0.0, 1.0))
            directions = np.stack(
                [np.outer(sin_theta, np.cos(phis)).ravel(), np.outer(sin_theta, np.sin(phis)).ravel(),
                 np.repeat(cos_nodes, n_phi)], axis=1)
            w_ang = np.repeat(cos_weights, n_phi) * (2.0 * math.pi / n_phi)
            points.append(r * directions)
            weights.append(wr * w_ang)
            n_radial += 1
    return np.concatenate(points) + np.asarray(centre), np.concatenate(weights), n_radial


class CuspQuadrature:
    """The cusp-aware quadrature (``src/cdft/operators/quadrature.py:188-773``)."""

    degree = 7
    taper_width_in_spacings = 1.3
    taper_margin = 4.5
    min_centre_in_spacings = 3.5
    max_radius_in_spacings = 11.5
    radial_order = 6
    node_spacing = 1.0
    node_spacing_overlapping = 0.7
    far_refine = 2
    far_edge_margin_in_spacings = 6.0
    far_edge_width_in_spacings = 1.5
    cell_width_in_spacings = 1.0

    def __init__(self, grid: Grid, factor: CuspFactor) -> None:
        self.grid = grid
        self.factor = factor
        h = grid.spacing
        positions = factor.positions
        charges = factor.charges
        n_atoms = len(charges)
        origin = np.asarray(grid.origin)
        upper = origin + np.array([(n - 1) * h for n in grid.shape])
        half = self.degree // 2
        margin = (half + 1.5) * h
        self.taper, self.overlapping, self.spheres = [], [], []
        pts, owner, base = [], [], []
        for atom in range(n_atoms):
            centre = positions[atom]
            edge_distance = float(np.minimum(centre - origin, upper - centre).min())
            radius_sphere = min(edge_distance - margin, self.max_radius_in_spacings * h)
            if radius_sphere <= 2.0 * h:
                raise ValueError(f"nucleus {atom} is too close to the box edge for the cusp quadrature")
            width = self.taper_width_in_spacings * h
            taper_centre = radius_sphere - self.taper_margin * width
            if taper_centre < self.min_centre_in_spacings * h:
                scale = radius_sphere / ((self.min_centre_in_spacings + self.taper_margin * self.taper_width_in_spacings) * h)
                width = self.taper_width_in_spacings * h * scale
                taper_centre = self.min_centre_in_spacings * h * scale
            self.taper.append((taper_centre, width))
            overlapping = False
            if n_atoms > 1:
                others = np.concatenate([positions[:atom], positions[atom + 1:]])
                nearest = float(np.sqrt(((others - centre) ** 2).sum(axis=-1)).min())
                overlapping = nearest < 2.0 * radius_sphere
            self.overlapping.append(overlapping)
            p, w, n_radial = sphere_rule(centre, radius_sphere, h, self.radial_order,
                                         self.node_spacing_overlapping if overlapping else self.node_spacing)
            self.spheres.append((centre.copy(), radius_sphere))
            pts.append(p)
            base.append(w)
            owner.append(np.full(p.shape[0], atom))
        self.points = np.concatenate(pts)
        self.owner = np.concatenate(owner)
        base_weights = np.concatenate(base)
        self.n_nodes = self.points.shape[0]
        self.partition = self._partition_weights(self.points, self.owner)
        self.weights = base_weights * self.partition
        u = np.zeros(self.n_nodes)
        grad_u = np.zeros((3, self.n_nodes))
        for atom, z in enumerate(charges):
            delta = self.points - positions[atom]
            distance = np.maximum(np.sqrt((delta * delta).sum(axis=-1)), 1.0e-300)
            u = u + z * distance
            grad_u = grad_u + z * (delta / distance[:, None]).T
        self.f2 = np.exp(-2.0 * u)
        self.grad_u = grad_u
        self.transformed_potential = -0.5 * (grad_u * grad_u).sum(axis=0)
        self._build_stencils()
        self.far = self._far_factor(grid.points())
        self.far_weights = grid.volume_element * self.far
        self.plain_far = self.far_weights * factor.weight
        self.far_lumped = any(self.overlapping)
        self.lumped_far = self._lumped_far_weights() if self.far_lumped else self.plain_far
        self.mass_weights = self.lift(self.weights * self.f2) + self.lumped_far
        if (self.mass_weights <= 0.0).any():
            raise ValueError("the cusp-aware mass weights are not all positive")

    # --- partition (quadrature.py:360-504) ---
    def _bump(self, points, atom):
        centre, radius = self.spheres[atom]
        tc, width = self.taper[atom]
        s = np.sqrt(((points - centre) ** 2).sum(axis=-1))
        value = 0.5 * erfc((s - tc) / width)
        return np.where(s < radius, value, 0.0)

    def _far_factor(self, points):
        far = np.ones(points.shape[0])
        for atom in range(len(self.spheres)):
            far = far * (1.0 - self._bump(points, atom))
        return far

    def _becke_cells(self, points):
        n_atoms = len(self.spheres)
        if n_atoms == 1:
            return np.ones((1, points.shape[0]))
        distances = np.stack([np.sqrt(((points - c) ** 2).sum(axis=-1)) for c, _ in self.spheres])
        width = self.cell_width_in_spacings * self.grid.spacing * math.sqrt(2.0)
        cells = np.ones((n_atoms, points.shape[0]))
        for a in range(n_atoms):
            for b in range(n_atoms):
                if a != b:
                    cells[a] = cells[a] * 0.5 * erfc((distances[a] - distances[b]) / width)
        return cells / np.maximum(cells.sum(axis=0, keepdims=True), 1.0e-300)

    def _partition_weights(self, points, owner):
        near = 1.0 - self._far_factor(points)
        cells = self._becke_cells(points)
        result = np.zeros(points.shape[0])
        for atom in range(len(self.spheres)):
            mask = owner == atom
            share = cells[atom]
            for other in range(len(self.spheres)):
                if other == atom:
                    continue
                c, radius = self.spheres[other]
                outside = np.sqrt(((points - c) ** 2).sum(axis=-1)) >= radius
                share = share + cells[other] * outside
            result[mask] = (share * near)[mask]
        return result

    def _lumped_far_weights(self):
        """``Q_far[f^2 ell_i]`` on the twice-refined lattice (quadrature.py:421-497)."""
        grid = self.grid
        h = grid.spacing
        refine = int(self.far_refine)
        shape = grid.shape
        positions = self.factor.positions
        charges = self.factor.charges
        k = self.degree + 1
        half = self.degree // 2
        matrices, fine_axes = [], []
        for axis in range(3):
            n = shape[axis]
            n_fine = n * refine
            fine = grid.origin[axis] - 0.5 * h + h * (np.arange(n_fine, dtype=np.float64) + 0.5) / refine
            fine_axes.append(fine)
            fractional = (fine - grid.origin[axis]) / h
            first = np.clip(np.floor(fractional).astype(np.int64) - half, 0, n - k)
            t = fractional - first.astype(np.float64)
            x = t[:, None] - np.arange(k, dtype=np.float64)[None, :]
            weights = np.ones_like(x)
            for j in range(k):
                for m in range(k):
                    if m != j:
                        weights[:, j] = weights[:, j] * x[:, m] / float(j - m)
            matrix = np.zeros((n, n_fine))
            rows = (first[:, None] + np.arange(k)[None, :]).reshape(-1)
            cols = np.repeat(np.arange(n_fine), k)
            np.add.at(matrix, (rows, cols), weights.reshape(-1))
            matrices.append(matrix)
        n_x, n_y, n_z = (shape[0] * refine, shape[1] * refine, shape[2] * refine)
        xs, ys = np.meshgrid(fine_axes[0], fine_axes[1], indexing="ij")
        plane_xy = np.stack([xs.reshape(-1), ys.reshape(-1)], axis=1)
        collapsed = np.zeros((n_x, n_y, shape[2]))
        volume = (h / refine) ** 3
        for iz in range(n_z):
            points = np.concatenate([plane_xy, np.full((plane_xy.shape[0], 1), fine_axes[2][iz])], axis=1)
            far = np.ones(points.shape[0])
            u = np.zeros(points.shape[0])
            for atom, ((centre, radius), (tc, width)) in enumerate(zip(self.spheres, self.taper)):
                s = np.sqrt(((points - centre) ** 2).sum(axis=-1))
                bump = np.where(s < radius, 0.5 * erfc((s - tc) / width), 0.0)
                far = far * (1.0 - bump)
                u = u + charges[atom] * s
            values = (volume * far * np.exp(-2.0 * u)).reshape(n_x, n_y)
            collapsed = collapsed + values[:, :, None] * matrices[2][:, iz][None, None, :]
        lumped = np.einsum("ax,by,xyc->abc", matrices[0], matrices[1], collapsed).reshape(-1)
        points = grid.points()
        origin = np.asarray(grid.origin)
        upper = origin + np.array([(n - 1) * h for n in shape])
        face = np.minimum((points - origin).min(axis=1), (upper - points).min(axis=1))
        margin = self.far_edge_margin_in_spacings * h
        width = self.far_edge_width_in_spacings * h
        interior = 0.5 * erfc((margin - face) / width)
        return self.plain_far + interior * (lumped - self.plain_far)

    # --- interpolation operator (quadrature.py:506-650) ---
    def _build_stencils(self):
        grid = self.grid
        h = grid.spacing
        origin = np.asarray(grid.origin)
        fractional = (self.points - origin) / h
        base = np.floor(fractional)
        t = fractional - base
        half = self.degree // 2
        k = self.degree + 1
        w1, i1 = [], []
        for axis in range(3):
            w1.append(lagrange_weights(t[:, axis], self.degree))
            index = base[:, axis].astype(np.int64)[:, None] + np.arange(-half, -half + k)[None, :]
            if (index < 0).any() or (index >= grid.shape[axis]).any():
                raise ValueError("an interpolation stencil reaches outside the grid")
            i1.append(index)
        self.base = base.astype(np.int64)
        self.t = t
        self.lagrange = w1
        sx, sy, sz = grid.shape[1] * grid.shape[2], grid.shape[2], 1
        wx, wy, wz = w1
        ix, iy, iz = i1
        columns = (ix[:, :, None, None] * sx + iy[:, None, :, None] * sy + iz[:, None, None, :] * sz).reshape(-1)
        values = (wx[:, :, None, None] * wy[:, None, :, None] * wz[:, None, None, :]).reshape(-1)
        indptr = np.arange(0, self.n_nodes * k ** 3 + 1, k ** 3)
        self.L = sparse.csr_matrix((values, columns, indptr), shape=(self.n_nodes, grid.n_points))
        self.LT = self.L.tocsc().T.tocsr()

    def interpolate(self, field):
        """``L field`` at the nodes (quadrature.py:613-620)."""
        if field.ndim == 1:
            return self.L @ field
        return (self.L @ field.reshape(-1, self.grid.n_points).T).T.reshape(*field.shape[:-1], self.n_nodes)

    def interpolate_gradient(self, field):
        """Interpolated order-8 grid gradient, ``(3, M)`` (quadrature.py:622-626)."""
        return self.interpolate(self.grid.gradient(field))

    def lift(self, node_values):
        """``L^T x`` (quadrature.py:628-638)."""
        if node_values.ndim == 1:
            return self.LT @ node_values
        return (self.LT @ node_values.reshape(-1, self.n_nodes).T).T.reshape(*node_values.shape[:-1], self.grid.n_points)

    def lift_gradient(self, node_vectors):
        """``-div_FD (L^T X)`` (quadrature.py:640-650)."""
        lifted = self.lift(node_vectors)
        div = np.zeros(self.grid.n_points)
        for d in range(3):
            div = div + self.grid.partial_derivative(lifted[d], d)
        return -div

    def interpolate_at(self, points, field):
        """Degree-7 interpolation at arbitrary points (quadrature.py:652-697)."""
        grid = self.grid
        h = grid.spacing
        fractional = (np.asarray(points, dtype=np.float64) - np.asarray(grid.origin)) / h
        base = np.floor(fractional)
        t = fractional - base
        half = self.degree // 2
        k = self.degree + 1
        ws, idx = [], []
        for axis in range(3):
            ws.append(lagrange_weights(t[:, axis], self.degree))
            idx.append(base[:, axis].astype(np.int64)[:, None] + np.arange(-half, -half + k)[None, :])
        sx, sy, sz = grid.shape[1] * grid.shape[2], grid.shape[2], 1
        flat = idx[0][:, :, None, None] * sx + idx[1][:, None, :, None] * sy + idx[2][:, None, None, :] * sz
        w3 = ws[0][:, :, None, None] * ws[1][:, None, :, None] * ws[2][:, None, None, :]
        return (field[flat] * w3).sum(axis=(-3, -2, -1))

    def integrate(self, node_values, grid_values):
        near = (self.weights * node_values).sum(axis=-1) if self.n_nodes else 0.0
        return near + (self.far_weights * grid_values).sum(axis=-1)

    def lumped_weights(self, node_values, grid_values):
        return self.lift(self.weights * node_values) + self.far_weights * grid_values

    def lumped_gradient_weights(self, node_vectors, grid_vectors):
        """(quadrature.py:718-729)"""
        near = self.lift_gradient(self.weights * node_vectors)
        weighted = self.far[None, :] * grid_vectors
        div = np.zeros(self.grid.n_points)
        for d in range(3):
            div = div + self.grid.gradient(weighted[d])[d]
        return near - self.grid.volume_element * div

    def effective_potential(self, node_values, grid_values):
        """``omega~/omega`` (quadrature.py:747-753)."""
        tilde = self.lumped_weights(node_values * self.f2, grid_values * self.factor.weight)
        return tilde / self.mass_weights

    def bare_operator_terms(self):
        """``(W~/omega, h^3/omega, q)`` (quadrature.py:731-745)."""
        potential = self.effective_potential(self.transformed_potential, self.factor.transformed_potential)
        h3 = self.grid.volume_element
        inverse_weight = h3 / self.mass_weights
        quadrature = (self.mass_weights / h3) * h3
        return potential, inverse_weight, quadrature

    def density_gradient_at_nodes(self, rho):
        rho_node = self.interpolate(rho)
        grad_rho = self.interpolate_gradient(rho)
        n = self.f2 * rho_node
        grad_n = self.f2[None, :] * (grad_rho - 2.0 * rho_node[None, :] * self.grad_u)
        return n, grad_n

    def density_gradient_on_grid(self, rho):
        grad_rho = self.grid.gradient(rho)
        return self.factor.weight[None, :] * (grad_rho - 2.0 * rho[None, :] * self.factor.grad_u)


def hydrogenic_1s_potential(charge: float, distance: np.ndarray) -> np.ndarray:
    """Potential of ``exp(-2 Z s)`` (``src/cdft/operators/quadrature.py:805-820``)."""
    z = float(charge)
    x = z * distance
    small = x < 1.0e-3
    safe = np.maximum(distance, 1.0e-300)
    full = (math.pi / z ** 3) * (1.0 - np.exp(-2.0 * x) * (1.0 + x)) / safe
    series = (math.pi / z ** 2) * (1.0 - (2.0 / 3.0) * x ** 2 + (2.0 / 3.0) * x ** 3 - 0.4 * x ** 4 + (8.0 / 45.0) * x ** 5)
    return np.where(small, series, full)


class StepGeometry:
    """Hartree-split geometry (``src/cdft/scf/step.py:111-165``)."""

    def __init__(self, grid: Grid, quadrature: CuspQuadrature, charges, positions) -> None:
        positions = np.asarray(positions, dtype=np.float64).reshape(-1, 3)
        n_atoms = len(charges)
        dist = [[float(np.sqrt(((positions[a] - positions[b]) ** 2).sum())) for b in range(n_atoms)] for a in range(n_atoms)]
        self.positions = positions
        self.overlap = np.array([[math.exp(-2.0 * zb * dist[a][b]) for b, zb in enumerate(charges)] for a in range(n_atoms)])
        pts = grid.points()
        r_grid = [np.sqrt(((pts - positions[a]) ** 2).sum(axis=-1)) for a in range(n_atoms)]
        r_node = [np.sqrt(((quadrature.points - positions[a]) ** 2).sum(axis=-1)) for a in range(n_atoms)]
        self.cusp_grid = np.stack([np.exp(-2.0 * z * r_grid[a]) for a, z in enumerate(charges)])
        self.v1s_grid = np.stack([hydrogenic_1s_potential(z, r_grid[a]) for a, z in enumerate(charges)])
        self.v1s_node = np.stack([hydrogenic_1s_potential(z, r_node[a]) for a, z in enumerate(charges)])
        self.nucleus_f2 = np.array([
            math.exp(-2.0 * sum(zb * dist[a][b] for b, zb in enumerate(charges) if b != a)) for a in range(n_atoms)])
