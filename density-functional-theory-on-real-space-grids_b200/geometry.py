"""Geometry of the cusp-factorised path, built on the device.

Host mirror of ``src/cdft/operators/cusp.py`` (CuspFactor), ``src/cdft/operators/quadrature.py``
(CuspQuadrature) and ``src/cdft/scf/step.py:111-165`` (StepGeometry). The only host-side work is the
node *plan* -- sphere radii, tapers and the list of sphere-rule node positions and bare weights
(Gauss--Legendre radius x product angular rule, ``quadrature.py:123-182, 252-288``), plus the three
one-dimensional interpolation matrices of the lumped far weights. Every grid- and node-sized field
(u, grad u, f^2, the cell-averaged W, face weights, partition weights, the interpolant's stencils,
the CSR of its transpose, far factors, mass weights and the bare operator terms) is computed by the
library's kernels.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from fractions import Fraction
from functools import lru_cache

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr, stream_handle
from .grid import UniformGrid
from .operators import Measure

MAX_ATOMS = 8


@lru_cache(maxsize=None)
def gauss_legendre(order: int) -> tuple[np.ndarray, np.ndarray]:
    """Gauss--Legendre nodes and weights on [-1, 1] (the rule of ``src/cdft/operators/gauss_legendre.py``).

    Newton on the three-term recurrence, then the reference's symmetrisation and normalisation.
    """
    n = int(order)
    x = np.cos(np.pi * (np.arange(1, n + 1) - 0.25) / (n + 0.5))

    def legendre(x):
        p0, p1 = np.ones_like(x), x.copy()
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
        if n == 1:
            p0, p1 = np.ones_like(x), x.copy()
        return p1, n * (x * p1 - p0) / (x * x - 1.0)

    for _ in range(100):
        p, dp = legendre(x)
        step = p / dp
        x = x - step
        if np.max(np.abs(step)) < 1e-17:
            break
    _, dp = legendre(x)
    w = 2.0 / ((1.0 - x * x) * dp * dp)
    order_idx = np.argsort(x)
    x, w = x[order_idx], w[order_idx]
    w = (w + w[::-1]) / 2.0
    x = (x - x[::-1]) / 2.0
    return x, w * (2.0 / w.sum())


@lru_cache(maxsize=None)
def first_derivative_weights(accuracy: int) -> tuple[float, ...]:
    """Central first-derivative weights, offsets -p..p (``src/cdft/operators/laplacian.py:36-75``)."""
    hw = accuracy // 2
    offsets = list(range(-hw, hw + 1))
    size = len(offsets)
    a = [[Fraction(o) ** m for o in offsets] for m in range(size)]
    b = [Fraction(0)] * size
    b[1] = Fraction(1)
    for col in range(size):
        piv = next(r for r in range(col, size) if a[r][col] != 0)
        a[col], a[piv] = a[piv], a[col]
        b[col], b[piv] = b[piv], b[col]
        inv = a[col][col]
        a[col] = [v / inv for v in a[col]]
        b[col] = b[col] / inv
        for r in range(size):
            if r != col and a[r][col] != 0:
                f = a[r][col]
                a[r] = [x - f * y for x, y in zip(a[r], a[col])]
                b[r] = b[r] - f * b[col]
    return tuple(float(v) for v in b)


def _flag(device) -> torch.Tensor:
    return torch.zeros(1, dtype=torch.int32, device=device)


def _host(values, dtype=np.float64) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(values, dtype=dtype))


def _hptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class CuspFactor:
    """Kato factor fields on the device (``src/cdft/operators/cusp.py:33-214``)."""

    average_quadrature = 4

    def __init__(self, grid: UniformGrid, charges, positions) -> None:
        self.grid = grid
        self.charges = tuple(float(z) for z in charges)
        self.positions = _host(positions).reshape(-1, 3)
        if not 1 <= len(self.charges) <= MAX_ATOMS:
            raise ValueError(f"between 1 and {MAX_ATOMS} nuclei are supported, got {len(self.charges)}")
        self.is_identity = False
        dev = grid.device
        n = grid.n_points
        f = dict(dtype=torch.float64, device=dev)
        self.u = torch.empty(n, **f)
        self.grad_u = torch.empty((3, n), **f)
        self.weight = torch.empty(n, **f)
        self.transformed_potential = torch.empty(n, **f)
        nodes, weights = gauss_legendre(self.average_quadrature)
        h = grid.spacing
        gl4 = torch.tensor([float(x) * 0.5 * h for x in nodes] + [float(w) * 0.5 for w in weights], **f)
        count = _flag(dev)
        self._charges_h = _host(self.charges)
        self._positions_h = _host(self.positions)
        call("cdftb_geometry_cusp_fields", len(self.charges), _hptr(self._charges_h), _hptr(self._positions_h),
             *grid.shape, *grid.origin, h, ptr(gl4), ptr(self.u), ptr(self.grad_u), ptr(self.weight),
             ptr(self.transformed_potential), ptr(count), stream_handle(dev))
        self.n_cell_averaged = int(count.item())
        self._faces: dict[int, tuple] = {}

    def face_weights(self, accuracy: int):
        """``f^2`` at the staggered faces (cusp.py:168-214); raises on float64 underflow."""
        if accuracy in self._faces:
            return self._faces[accuracy]
        grid = self.grid
        shapes = []
        for axis in range(3):
            s = list(grid.shape)
            s[axis] += accuracy
            shapes.append(s)
        out = tuple(torch.empty(s, dtype=torch.float64, device=grid.device) for s in shapes)
        flag = _flag(grid.device)
        call("cdftb_geometry_face_weights", len(self.charges), _hptr(self._charges_h), _hptr(self._positions_h),
             *grid.shape, *grid.origin, grid.spacing, int(accuracy), ptr(out[0]), ptr(out[1]), ptr(out[2]), ptr(flag),
             stream_handle(grid.device))
        if int(flag.item()):
            raise ValueError("the cusp weight exp(-2u) underflows float64 on this domain (max u > 354); "
                             "reduce the box or the nuclear charge")
        self._faces[accuracy] = out
        return out


def sphere_rule(centre: np.ndarray, radius_sphere: float, spacing: float, radial_order: int, node_spacing: float):
    """Node positions and bare weights ``r^2 dr dOmega`` of one sphere (``quadrature.py:123-182``)."""
    n_panels = max(2, int(math.ceil(radius_sphere / spacing)))
    edges = np.linspace(0.0, radius_sphere, n_panels + 1)
    gl_nodes, gl_weights = gauss_legendre(radial_order)
    points, weights = [], []
    for lo, hi in zip(edges[:-1], edges[1:]):
        mid, half = 0.5 * (hi + lo), 0.5 * (hi - lo)
        for node, weight in zip(gl_nodes, gl_weights):
            r = mid + half * node
            wr = half * weight * r * r
            n_theta = max(4, int(math.ceil(math.sqrt(2.0 * math.pi) * r / (node_spacing * spacing))))
            n_phi = 2 * n_theta
            cos_nodes, cos_weights = gauss_legendre(n_theta)
            phis = 2.0 * math.pi * (np.arange(n_phi) + 0.5) / n_phi
            sin_theta = np.sqrt(np.clip(1.0 - cos_nodes ** 2, 0.0, 1.0))
            directions = np.stack([np.outer(sin_theta, np.cos(phis)).ravel(), np.outer(sin_theta, np.sin(phis)).ravel(),
                                   np.repeat(cos_nodes, n_phi)], axis=1)
            points.append(r * directions)
            weights.append(wr * (np.repeat(cos_weights, n_phi) * (2.0 * math.pi / n_phi)))
    return np.concatenate(points) + centre, np.concatenate(weights)


def _interp_matrix(n: int, refine: int, origin: float, h: float, degree: int = 7):
    """The transposed 1-D interpolation matrix coarse x fine of ``quadrature.py:449-467`` and its bands."""
    k = degree + 1
    half = degree // 2
    n_fine = n * refine
    fine = origin - 0.5 * h + h * (np.arange(n_fine, dtype=np.float64) + 0.5) / refine
    fractional = (fine - origin) / h
    first = np.clip(np.floor(fractional).astype(np.int64) - half, 0, n - k)
    t = fractional - first.astype(np.float64)
    x = t[:, None] - np.arange(k, dtype=np.float64)[None, :]
    w = np.ones_like(x)
    for j in range(k):
        for m in range(k):
            if m != j:
                w[:, j] = w[:, j] * x[:, m] / float(j - m)
    matrix = np.zeros((n, n_fine))
    rows = (first[:, None] + np.arange(k)[None, :]).reshape(-1)
    cols = np.repeat(np.arange(n_fine), k)
    np.add.at(matrix, (rows, cols), w.reshape(-1))
    lo = np.zeros(n, dtype=np.int32)
    hi = np.zeros(n, dtype=np.int32)
    for c in range(n):
        nz = np.nonzero((first <= c) & (c < first + k))[0]
        lo[c], hi[c] = (nz.min(), nz.max() + 1) if nz.size else (0, 0)
    return fine, matrix, lo, hi


class CuspQuadrature:
    """The cusp-aware quadrature on the device (``src/cdft/operators/quadrature.py:188-773``)."""

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

    def __init__(self, grid: UniformGrid, factor: CuspFactor) -> None:
        self.grid = grid
        self.factor = factor
        dev = grid.device
        h = grid.spacing
        positions = factor.positions
        charges = factor.charges
        n_atoms = len(charges)
        origin = np.asarray(grid.origin)
        upper = origin + np.array([(n - 1) * h for n in grid.shape])
        margin = (self.degree // 2 + 1.5) * h
        self.taper, self.overlapping, spheres, pts, owner, base = [], [], [], [], [], []
        for atom in range(n_atoms):
            centre = positions[atom]
            edge_distance = float(np.minimum(centre - origin, upper - centre).min())
            radius = min(edge_distance - margin, self.max_radius_in_spacings * h)
            if radius <= 2.0 * h:
                raise ValueError(f"nucleus {atom} is {edge_distance:.3g} bohr from the box edge; the cusp quadrature "
                                 f"needs at least {2.0 * h + margin:.3g} bohr. Enlarge the box.")
            width = self.taper_width_in_spacings * h
            taper_centre = radius - self.taper_margin * width
            if taper_centre < self.min_centre_in_spacings * h:
                scale = radius / ((self.min_centre_in_spacings + self.taper_margin * self.taper_width_in_spacings) * h)
                width = self.taper_width_in_spacings * h * scale
                taper_centre = self.min_centre_in_spacings * h * scale
            self.taper.append((taper_centre, width))
            overlapping = False
            if n_atoms > 1:
                others = np.concatenate([positions[:atom], positions[atom + 1:]])
                overlapping = float(np.sqrt(((others - centre) ** 2).sum(axis=-1)).min()) < 2.0 * radius
            self.overlapping.append(overlapping)
            p, w = sphere_rule(centre, radius, h, self.radial_order,
                               self.node_spacing_overlapping if overlapping else self.node_spacing)
            spheres.append([*centre, radius, taper_centre, width])
            pts.append(p)
            base.append(w)
            owner.append(np.full(p.shape[0], atom, dtype=np.int32))
        self.sphere_rows = _host(spheres)
        self.n_nodes = int(sum(p.shape[0] for p in pts))
        m = self.n_nodes
        f = dict(dtype=torch.float64, device=dev)
        self.points = torch.from_numpy(np.ascontiguousarray(np.concatenate(pts))).to(dev)
        owner_d = torch.from_numpy(np.concatenate(owner)).to(dev)
        base_d = torch.from_numpy(np.ascontiguousarray(np.concatenate(base))).to(dev)
        self.partition = torch.empty(m, **f)
        self.weights = torch.empty(m, **f)
        self.f2 = torch.empty(m, **f)
        self.grad_u = torch.empty((3, m), **f)
        self.transformed_potential = torch.empty(m, **f)
        stream = stream_handle(dev)
        cell_width = self.cell_width_in_spacings * h * math.sqrt(2.0)
        call("cdftb_geometry_node_fields", n_atoms, _hptr(factor._charges_h), _hptr(factor._positions_h),
             _hptr(self.sphere_rows), cell_width, ptr(self.points), ptr(owner_d), ptr(base_d), m, ptr(self.partition),
             ptr(self.weights), ptr(self.f2), ptr(self.grad_u), ptr(self.transformed_potential), stream)
        # interpolant stencils and the CSR of its transpose
        self.base = torch.empty((m, 3), dtype=torch.int32, device=dev)
        self.w1d = torch.empty((m, 24), **f)
        bad = _flag(dev)
        call("cdftb_quadrature_stencils", ptr(self.points), m, *grid.shape, *grid.origin, h, ptr(self.base),
             ptr(self.w1d), ptr(bad), stream)
        if int(bad.item()):
            raise ValueError("an interpolation stencil reaches outside the grid; the sphere radius bound is wrong")
        n = grid.n_points
        self.row_ptr = torch.empty(n + 1, dtype=torch.int64, device=dev)
        self.col = torch.empty(m * 512, dtype=torch.int32, device=dev)
        nbytes = _lib.library().cdftb_lift_plan_scratch_bytes(m, n)
        scratch = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=dev)
        call("cdftb_lift_plan_build", ptr(self.base), m, *grid.shape, ptr(self.row_ptr), ptr(self.col), ptr(scratch),
             scratch.numel(), stream)
        del scratch
        # the weight of every entry of L^T, formed once (the lifts then stream (col, value) pairs)
        self.lift_values = torch.empty(m * 512, dtype=torch.float64, device=dev)
        call("cdftb_lift_plan_values_f64", ptr(self.base), ptr(self.w1d), ptr(self.row_ptr), ptr(self.col),
             *grid.shape, ptr(self.lift_values), stream)
        # the rows of L^T cut into segments of at most 256 entries (the many-field lift's work units)
        lib = _lib.library()
        self.seg_capacity = lib.cdftb_lift_segments_capacity(m, n)
        self.seg_ptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
        self.seg_row = torch.empty(self.seg_capacity, dtype=torch.int32, device=dev)
        seg_scratch = torch.empty(lib.cdftb_lift_segments_scratch_bytes(n), dtype=torch.uint8, device=dev)
        call("cdftb_lift_plan_segments", ptr(self.row_ptr), *grid.shape, ptr(self.seg_ptr), ptr(self.seg_row),
             self.seg_capacity, ptr(seg_scratch), seg_scratch.numel(), stream)
        del seg_scratch
        # the nodes grouped by base cell (nodes of a group read the same 8^3 box): the many-field
        # interpolant reads each box once per group instead of once per node
        key = (self.base[:, 0].to(torch.int64) * grid.shape[1] + self.base[:, 1]) * grid.shape[2] + self.base[:, 2]
        key, order = torch.sort(key, stable=True)
        _, counts = torch.unique_consecutive(key, return_counts=True)
        self.group_nodes = order.to(torch.int32).contiguous()
        # work items of at most GROUP_BATCH nodes of one cell (a cell near a nucleus holds up to ~80
        # nodes): one warp each, so that a crowded cell does not hold up the launch
        starts = torch.cumsum(counts, 0) - counts
        items = (counts + self.GROUP_BATCH - 1) // self.GROUP_BATCH
        first = torch.repeat_interleave(starts, items)
        k = torch.arange(int(items.sum()), device=dev) - torch.repeat_interleave(torch.cumsum(items, 0) - items, items)
        item_start = first + k * self.GROUP_BATCH
        self.group_ptr = torch.cat([item_start, counts.sum().reshape(1)]).to(torch.int32).contiguous()
        self.n_groups = int(item_start.numel())
        # far factor, plain and lumped far mass weights
        self.far = torch.empty(n, **f)
        self.far_weights = torch.empty(n, **f)
        self.plain_far = torch.empty(n, **f)
        call("cdftb_geometry_grid_far", n_atoms, _hptr(factor._charges_h), _hptr(factor._positions_h),
             _hptr(self.sphere_rows), *grid.shape, *grid.origin, h, ptr(factor.weight), ptr(self.far),
             ptr(self.far_weights), ptr(self.plain_far), stream)
        self.far_lumped = any(self.overlapping)
        self.lumped_far = self._lumped_far_weights() if self.far_lumped else self.plain_far
        # mass weights and the bare operator terms
        lift_in = torch.stack([self.weights * self.f2, self.weights * (self.transformed_potential * self.f2)])
        lifted = self._lift_raw(lift_in.contiguous(), 2)
        self.mass_weights = torch.empty(n, **f)
        self._bare_potential = torch.empty(n, **f)
        self._inverse_weight = torch.empty(n, **f)
        self._quadrature = torch.empty(n, **f)
        nonpos = _flag(dev)
        call("cdftb_geometry_bare_terms", ptr(lifted), ptr(self.lumped_far), ptr(self.far_weights),
             ptr(factor.transformed_potential), ptr(factor.weight), n, h, ptr(self.mass_weights),
             ptr(self._bare_potential), ptr(self._inverse_weight), ptr(self._quadrature), ptr(nonpos), stream)
        if int(nonpos.item()):
            raise ValueError("the cusp-aware mass weights are not all positive (Z h > 1?); refine the grid")
        self._measure = Measure(grid, self._quadrature)

    def _lumped_far_weights(self) -> torch.Tensor:
        grid = self.grid
        dev = grid.device
        h = grid.spacing
        refine = self.far_refine
        axes = [_interp_matrix(n, refine, o, h, self.degree) for n, o in zip(grid.shape, grid.origin)]
        t = [torch.from_numpy(np.ascontiguousarray(a[0])).to(dev) for a in axes]
        mats = [torch.from_numpy(np.ascontiguousarray(a[1])).to(dev) for a in axes]
        los = [torch.from_numpy(a[2]).to(dev) for a in axes]
        his = [torch.from_numpy(a[3]).to(dev) for a in axes]
        nx, ny, nz = grid.shape
        work = torch.empty(nx * refine * ny * refine * nz + nx * ny * refine * nz, dtype=torch.float64, device=dev)
        out = torch.empty(grid.n_points, dtype=torch.float64, device=dev)
        f = self.factor
        call("cdftb_geometry_lumped_far", len(f.charges), _hptr(f._charges_h), _hptr(f._positions_h),
             _hptr(self.sphere_rows), *grid.shape, *grid.origin, h, refine, ptr(t[0]), ptr(t[1]), ptr(t[2]),
             ptr(mats[0]), ptr(los[0]), ptr(his[0]), ptr(mats[1]), ptr(los[1]), ptr(his[1]), ptr(mats[2]), ptr(los[2]),
             ptr(his[2]), ptr(self.plain_far), self.far_edge_margin_in_spacings * h, self.far_edge_width_in_spacings * h,
             ptr(work), ptr(out), stream_handle(dev))
        return out

    # --- interpolation and its transpose (quadrature.py:613-650) ---
    #: From this many fields on, L and L^T run one pass per 32 fields (the batched systems).
    MANY_FIELDS = 8
    #: Nodes of one cell per warp of the grouped interpolant (GROUP_BATCH in csrc/quadrature.cu).
    GROUP_BATCH = 4

    def _many_scratch(self, device) -> torch.Tensor:
        nbytes = _lib.library().cdftb_quadrature_many_scratch_bytes(self.n_nodes, self.grid.n_points)
        return torch.empty(nbytes, dtype=torch.uint8, device=device)

    def _interp_raw(self, fields: torch.Tensor, nf: int) -> torch.Tensor:
        n = self.grid.n_points
        out = torch.empty((nf, self.n_nodes), dtype=torch.float64, device=fields.device)
        if nf >= self.MANY_FIELDS:
            scratch = self._many_scratch(fields.device)
            call("cdftb_quadrature_interpolate_grouped_f64", ptr(self.base), ptr(self.w1d), self.n_nodes,
                 *self.grid.shape, ptr(self.group_nodes), ptr(self.group_ptr), self.n_groups, ptr(fields), nf, n,
                 ptr(out), self.n_nodes, ptr(scratch), scratch.numel(), stream_handle(fields.device))
            return out
        call("cdftb_quadrature_interpolate_f64", ptr(self.base), ptr(self.w1d), self.n_nodes, *self.grid.shape,
             ptr(fields), nf, n, ptr(out), self.n_nodes, stream_handle(fields.device))
        return out

    def _lift_raw(self, x: torch.Tensor, nf: int) -> torch.Tensor:
        n = self.grid.n_points
        out = torch.empty((nf, n), dtype=torch.float64, device=x.device)
        if nf >= self.MANY_FIELDS:
            scratch = self._many_scratch(x.device)
            call("cdftb_quadrature_lift_many_f64", ptr(self.row_ptr), ptr(self.col), ptr(self.lift_values),
                 ptr(self.seg_ptr), ptr(self.seg_row), self.seg_capacity, *self.grid.shape, self.n_nodes, ptr(x), nf,
                 self.n_nodes, ptr(out), n, ptr(scratch), scratch.numel(), stream_handle(x.device))
            return out
        call("cdftb_quadrature_lift_f64", ptr(self.base), ptr(self.w1d), ptr(self.row_ptr), ptr(self.col),
             ptr(self.lift_values), *self.grid.shape, ptr(x), nf, self.n_nodes, ptr(out), n, stream_handle(x.device))
        return out

    def interpolate(self, field: torch.Tensor) -> torch.Tensor:
        """``L field`` at the nodes, ``(..., m)``."""
        n = self.grid.n_points
        flat = field.to(torch.float64).reshape(-1, n).contiguous()
        return self._interp_raw(flat, flat.shape[0]).reshape(*field.shape[:-1], self.n_nodes)

    def interpolate_gradient(self, field: torch.Tensor) -> torch.Tensor:
        return self.interpolate(gradient(self.grid, field))

    def lift(self, node_values: torch.Tensor) -> torch.Tensor:
        """``L^T x`` on the grid, ``(..., N)``."""
        flat = node_values.to(torch.float64).reshape(-1, self.n_nodes).contiguous()
        return self._lift_raw(flat, flat.shape[0]).reshape(*node_values.shape[:-1], self.grid.n_points)

    def interpolate_at(self, points: torch.Tensor, field: torch.Tensor) -> torch.Tensor:
        """Degree-7 interpolation at arbitrary points (quadrature.py:652-697)."""
        pts = points.to(torch.float64).reshape(-1, 3).contiguous()
        k = pts.shape[0]
        base = torch.empty((k, 3), dtype=torch.int32, device=pts.device)
        w1d = torch.empty((k, 24), dtype=torch.float64, device=pts.device)
        bad = _flag(pts.device)
        call("cdftb_quadrature_stencils", ptr(pts), k, *self.grid.shape, *self.grid.origin, self.grid.spacing, ptr(base),
             ptr(w1d), ptr(bad), stream_handle(pts.device))
        out = torch.empty((1, k), dtype=torch.float64, device=pts.device)
        call("cdftb_quadrature_interpolate_f64", ptr(base), ptr(w1d), k, *self.grid.shape,
             ptr(field.to(torch.float64).contiguous()), 1, self.grid.n_points, ptr(out), k, stream_handle(pts.device))
        return out[0]

    # --- integrals and lumped weights (quadrature.py:701-753) ---
    def integrate(self, node_values: torch.Tensor, grid_values: torch.Tensor) -> torch.Tensor:
        return row_sums(self.weights * node_values) + row_sums(self.far_weights * grid_values)

    def lumped_weights(self, node_values: torch.Tensor, grid_values: torch.Tensor) -> torch.Tensor:
        return self.lift(self.weights * node_values) + self.far_weights * grid_values

    def bare_operator_terms(self):
        """``(W~/omega, h^3/omega, Measure)``, built once on the device."""
        return self._bare_potential, self._inverse_weight, self._measure

    def density_gradient_at_nodes(self, rho: torch.Tensor):
        both = self.interpolate(torch.cat([rho.reshape(1, -1), gradient(self.grid, rho).reshape(3, -1)]))
        rho_node, grad_rho = both[0], both[1:]
        n = self.f2 * rho_node
        grad_n = self.f2[None, :] * (grad_rho - 2.0 * rho_node[None, :] * self.grad_u)
        return n, grad_n

    def external_energy_parts(self, rho: torch.Tensor, factor: CuspFactor):
        """``((1/2) Q[f^2 grad rho . grad u], Q[f^2 rho W])`` (hamiltonian.py:360-378)."""
        grad_rho = gradient(self.grid, rho)
        both = self.interpolate(torch.cat([rho.reshape(1, -1), grad_rho]))
        rho_node, grad_rho_node = both[0], both[1:]
        cross_node = self.f2 * (grad_rho_node * self.grad_u).sum(dim=0)
        cross_grid = factor.weight * (grad_rho * factor.grad_u).sum(dim=0)
        cross = 0.5 * self.integrate(cross_node, cross_grid)
        potential = self.integrate(self.f2 * rho_node * self.transformed_potential,
                                   factor.weight * rho * factor.transformed_potential)
        return cross, potential


def row_sums(a: torch.Tensor) -> torch.Tensor:
    """Deterministic sum over the last axis (float64), shape ``a.shape[:-1]``."""
    x = a.to(torch.float64).contiguous()
    length = x.shape[-1]
    rows = x.numel() // length
    out = torch.empty(rows, dtype=torch.float64, device=x.device)
    nbytes = _lib.library().cdftb_row_sums_scratch_bytes(rows, length)
    scratch = torch.empty(max(nbytes, 8), dtype=torch.uint8, device=x.device)
    call("cdftb_row_sums_f64", ptr(x), rows, length, ptr(out), ptr(scratch), scratch.numel(), stream_handle(x.device))
    return out.reshape(a.shape[:-1])


_FD_TABLE: dict = {}


def _fd_table(accuracy: int, device) -> torch.Tensor:
    key = (accuracy, str(device))
    if key not in _FD_TABLE:
        _FD_TABLE[key] = torch.tensor(first_derivative_weights(accuracy), dtype=torch.float64, device=device)
    return _FD_TABLE[key]


def partial_derivative(grid: UniformGrid, field: torch.Tensor, axis: int, out: torch.Tensor | None = None,
                       accumulate: bool = False, sign: float = 1.0) -> torch.Tensor:
    """One order-``gradient_order`` central derivative, zero halo (``src/cdft/grid.py:745-758``)."""
    x = field.to(torch.float64).contiguous()
    batch = x.numel() // grid.n_points
    if out is None:
        out = torch.empty_like(x)
    call("cdftb_fd_derivative_f64", ptr(x), ptr(out), *grid.shape, int(axis), grid.gradient_order,
         ptr(_fd_table(grid.gradient_order, x.device)), grid.spacing, batch, 1 if accumulate else 0, float(sign),
         stream_handle(x.device))
    return out


def gradient(grid: UniformGrid, field: torch.Tensor) -> torch.Tensor:
    """``(..., 3, N)`` gradient (``src/cdft/grid.py:740-743``): the three derivatives of
    :func:`partial_derivative` in one pass, bit for bit."""
    x = field.to(torch.float64).contiguous()
    n = grid.n_points
    batch = x.numel() // n
    out = torch.empty((*x.shape[:-1], 3, n), dtype=torch.float64, device=x.device)
    call("cdftb_gradient_f64", ptr(x), ptr(out), *grid.shape, grid.gradient_order,
         ptr(_fd_table(grid.gradient_order, x.device)), grid.spacing, batch, stream_handle(x.device))
    return out


class StepGeometry:
    """The Hartree-split tensors (``src/cdft/scf/step.py:111-165``) on the device."""

    def __init__(self, grid: UniformGrid, quadrature: CuspQuadrature, charges, positions) -> None:
        dev = grid.device
        positions = _host(positions).reshape(-1, 3)
        n_atoms = len(charges)
        dist = [[float(np.sqrt(((positions[a] - positions[b]) ** 2).sum())) for b in range(n_atoms)]
                for a in range(n_atoms)]
        overlap = np.array([[math.exp(-2.0 * zb * dist[a][b]) for b, zb in enumerate(charges)] for a in range(n_atoms)])
        np.linalg.solve(overlap, np.ones(n_atoms))  # validated once, as the reference does (step.py:152)
        self.overlap = torch.from_numpy(overlap).to(dev)
        self.nucleus_f2 = torch.tensor([math.exp(-2.0 * sum(zb * dist[a][b] for b, zb in enumerate(charges) if b != a))
                                        for a in range(n_atoms)], dtype=torch.float64, device=dev)
        self.positions = torch.from_numpy(positions.copy()).to(dev)
        n, m = grid.n_points, quadrature.n_nodes
        self.cusp_grid = torch.empty((n_atoms, n), dtype=torch.float64, device=dev)
        self.v1s_grid = torch.empty((n_atoms, n), dtype=torch.float64, device=dev)
        self.v1s_node = torch.empty((n_atoms, m), dtype=torch.float64, device=dev)
        ch = _host(charges)
        ps = _host(positions)
        call("cdftb_geometry_step_fields", n_atoms, _hptr(ch), _hptr(ps), *grid.shape, *grid.origin, grid.spacing,
             ptr(quadrature.points), m, ptr(self.cusp_grid), ptr(self.v1s_grid), ptr(self.v1s_node), stream_handle(dev))
        # stencil of the nuclei themselves, for rho(R_a)
        self.nuclei_base = torch.empty((n_atoms, 3), dtype=torch.int32, device=dev)
        self.nuclei_w1d = torch.empty((n_atoms, 24), dtype=torch.float64, device=dev)
        bad = _flag(dev)
        call("cdftb_quadrature_stencils", ptr(self.positions), n_atoms, *grid.shape, *grid.origin, grid.spacing,
             ptr(self.nuclei_base), ptr(self.nuclei_w1d), ptr(bad), stream_handle(dev))
        if int(bad.item()):
            raise ValueError("interpolation point too close to the box edge for the stencil")


@dataclass
class CuspGeometry:
    """Everything geometry-only that one system's solve reads, built once."""

    grid: UniformGrid
    charges: tuple
    positions: np.ndarray
    factor: CuspFactor
    quadrature: CuspQuadrature
    step: StepGeometry
    extra: dict = field(default_factory=dict)


def build_cusp_geometry(grid: UniformGrid, charges, positions) -> CuspGeometry:
    """Factor, quadrature and Hartree-split geometry of one system on ``grid.device``."""
    factor = CuspFactor(grid, charges, positions)
    factor.face_weights(grid.fd_order)
    quadrature = CuspQuadrature(grid, factor)
    step = StepGeometry(grid, quadrature, factor.charges, factor.positions)
    return CuspGeometry(grid, factor.charges, factor.positions, factor, quadrature, step)
