"""The measure and the cusp-factorised Hamiltonian on the device, through the cdftb kernels.

Host mirror of ``src/cdft/eigen/measure.py`` (Measure), ``src/cdft/operators/hamiltonian.py``
(CuspFactoredHamiltonian, _lanczos_bounds) and ``src/cdft/operators/divergence.py:153``
(weighted_divergence): same names, argument meaning and error behaviour; every product, apply and
reduction runs in ``libcdftb.so``.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import F32, F64, call, ptr, stream_handle
from .grid import UniformGrid


def _scratch(nbytes: int, device) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 8), dtype=torch.uint8, device=device)


def apply_workspace(op, batch: int, device: torch.device) -> torch.Tensor:
    """Device scratch of the one-launch apply (``cdftb_cusp_apply_work_bytes``), as bytes."""
    nbytes = _lib.library().cdftb_cusp_apply_work_bytes(ctypes.byref(op), batch)
    return torch.empty(max(nbytes, 16), dtype=torch.uint8, device=device)


def measure_cross(a: torch.Tensor, b: torch.Tensor, q: torch.Tensor | None, groups: int = 1) -> torch.Tensor:
    """``out[g] = (a[g] * q) @ b[g].T`` for ``groups`` stacked blocks (float64, deterministic).

    ``q`` is one measure ``(N,)`` for every group, or one per group ``(groups, N)``.
    """
    n = a.shape[-1]
    a2 = a.reshape(groups, -1, n)
    b2 = b.reshape(groups, -1, n)
    if a2.dtype != torch.float64 or b2.dtype != torch.float64:
        raise ValueError("measure products take float64 blocks")
    a2 = a2.contiguous()
    b2 = b2.contiguous()
    ma, mb = a2.shape[1], b2.shape[1]
    out = torch.empty((groups, ma, mb), dtype=torch.float64, device=a.device)
    nbytes = _lib.library().cdftb_measure_cross_scratch_bytes(ma, mb, n, groups)
    scratch = _scratch(nbytes, a.device)
    if q is not None and q.dim() == 2:
        if q.shape != (groups, n):
            raise ValueError(f"a per-group measure must be ({groups}, {n}), got {tuple(q.shape)}")
        qc = q.contiguous()
        call("cdftb_measure_cross_grouped_f64", ptr(a2), ma, a2.stride(0), ptr(b2), mb, b2.stride(0), ptr(qc),
             qc.stride(0), n, groups, ptr(out), ptr(scratch), scratch.numel(), stream_handle(a.device))
        return out
    call("cdftb_measure_cross_f64", ptr(a2), ma, a2.stride(0), ptr(b2), mb, b2.stride(0), ptr(q), n, groups, ptr(out),
         ptr(scratch), scratch.numel(), stream_handle(a.device))
    return out


def rowwise_inner(a: torch.Tensor, b: torch.Tensor, q: torch.Tensor | None) -> torch.Tensor:
    """``sum_p q a[i, p] b[i, p]`` per row, float64 ``(...)``."""
    n = a.shape[-1]
    rows = a.numel() // n
    out = measure_cross(a.reshape(rows, 1, n), b.reshape(rows, 1, n), q, groups=rows)
    return out.reshape(a.shape[:-1])


class Measure:
    """``<a,b> = sum_r q(r) a(r) b(r)`` (``src/cdft/eigen/measure.py:18-82``), q = the quadrature weight."""

    def __init__(self, grid: UniformGrid, quadrature: torch.Tensor) -> None:
        if quadrature.shape[-1] != grid.n_points:
            raise ValueError(f"measure weight has {quadrature.shape[-1]} points, grid has {grid.n_points}")
        self.grid = grid
        self.quadrature = quadrature.to(torch.float64).contiguous()

    is_uniform = False

    def inner(self, a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        return rowwise_inner(a.to(torch.float64), b.to(torch.float64), self.quadrature)

    def norm(self, a: torch.Tensor) -> torch.Tensor:
        return self.inner(a, a).clamp_min(0.0).sqrt()

    def gram(self, block: torch.Tensor) -> torch.Tensor:
        flat = block.to(torch.float64).reshape(-1, self.grid.n_points)
        return measure_cross(flat, flat, self.quadrature)[0]

    def cross(self, left: torch.Tensor, right: torch.Tensor) -> torch.Tensor:
        a = left.to(torch.float64).reshape(-1, self.grid.n_points)
        b = right.to(torch.float64).reshape(-1, self.grid.n_points)
        return measure_cross(a, b, self.quadrature)[0]

    @property
    def dynamic_range(self) -> float:
        return float(self.quadrature.max() / self.quadrature.min())


def weighted_divergence(box: torch.Tensor, face_weights, spacing: float, accuracy: int, shape) -> torch.Tensor:
    """``sum_d D_d^T [w_d D_d phi]`` on a CUDA box (``src/cdft/operators/divergence.py:153``)."""
    _lib.require_cuda(box, "box")
    if box.dtype != torch.float64:
        raise ValueError("weighted_divergence takes a float64 box")
    shape = tuple(int(s) for s in shape)
    if tuple(box.shape[-3:]) != shape:
        raise ValueError(f"box shape {tuple(box.shape[-3:])} != {shape}")
    for axis, w in enumerate(face_weights):
        want = list(shape)
        want[axis] += accuracy
        if tuple(w.shape) != tuple(want):
            raise ValueError(f"face weights of axis {axis} have shape {tuple(w.shape)}, expected {tuple(want)}")
    flat = box.contiguous()
    batch = flat.numel() // (shape[0] * shape[1] * shape[2])
    out = torch.empty_like(flat)
    w = [x.to(torch.float64).contiguous() for x in face_weights]
    call("cdftb_weighted_divergence_f64", ptr(flat), ptr(out), batch, *shape, ptr(w[0]), ptr(w[1]), ptr(w[2]),
         float(spacing), int(accuracy), stream_handle(box.device))
    return out


class CuspFactoredHamiltonian:
    """``A = f^-1 H f`` in staggered divergence form (``src/cdft/operators/hamiltonian.py:375``).

    ``factor`` provides ``face_weights(accuracy)``; ``quadrature`` provides
    ``bare_operator_terms() -> (W~/omega, h^3/omega, Measure)``. ``extra_potential`` (N) is added
    to the bare potential. ``dtype=torch.float32`` keeps float copies of the geometry and runs the
    apply in float (the mixed-precision filter); products and the measure stay float64.
    """

    uses_divergence_form = True

    def __init__(self, grid: UniformGrid, factor, extra_potential: torch.Tensor | None = None, quadrature=None,
                 *, dtype: torch.dtype = torch.float64, bare=None) -> None:
        self.grid = grid
        self.factor = factor
        self.quadrature = quadrature
        if bare is None:
            bare = quadrature.bare_operator_terms()
        potential, inverse_weight, measure = bare
        self.measure = measure
        self._bare_potential = potential
        self._inverse_weight = inverse_weight
        if extra_potential is not None:
            if extra_potential.shape[-1] != grid.n_points:
                raise ValueError(f"extra potential has {extra_potential.shape[-1]} points, grid has {grid.n_points}")
            potential = potential + extra_potential
        self._potential = potential.contiguous()
        self._apply_count = 0
        self.dtype = dtype
        faces = factor.face_weights(grid.fd_order)
        if dtype == torch.float64:
            self._faces = tuple(f.contiguous() for f in faces)
            self._inv = inverse_weight.contiguous()
        else:
            # float copies of the geometry, made once per geometry and dtype
            cache = factor.__dict__.setdefault("_cast_cache", {})
            key = (dtype, inverse_weight.data_ptr())
            if key not in cache:
                cache[key] = (tuple(cast(f.contiguous(), dtype) for f in faces), cast(inverse_weight.contiguous(), dtype))
            self._faces, self._inv = cache[key]
        self._pot_cast = self._potential if dtype == torch.float64 else cast(self._potential, dtype)

    # -- the seam --
    @property
    def apply_count(self) -> int:
        return self._apply_count

    def note_applications(self, count: int) -> None:
        self._apply_count += int(count)

    def graph_potential(self) -> torch.Tensor:
        return self._potential

    def graph_geometry_key(self) -> tuple:
        return ("cusp-native", id(self.grid), tuple(f.data_ptr() for f in self._faces), self._inv.data_ptr(),
                self.measure.quadrature.data_ptr())

    def filter_potential(self) -> torch.Tensor:
        """The potential as the filter reads it (in the operator's dtype)."""
        return self._pot_cast

    def local_potential(self) -> torch.Tensor:
        return self._potential

    def operator(self, potential: torch.Tensor | None = None, groups: int = 1, orbitals_per_group: int = 1,
                 dtype: torch.dtype | None = None) -> _lib.Operator:
        """The ``cdftb_operator`` descriptor for this operator (optionally another potential)."""
        dtype = dtype or self.dtype
        if dtype != self.dtype:
            raise ValueError("operator dtype differs from the Hamiltonian's")
        pot = self._pot_cast if potential is None else potential.to(dtype).contiguous()
        op = _lib.Operator()
        op.nx, op.ny, op.nz = self.grid.shape
        op.accuracy = self.grid.fd_order
        op.spacing = self.grid.spacing
        op.dtype = F64 if dtype == torch.float64 else F32
        op.face_weights = (ctypes.c_void_p * 3)(*(f.data_ptr() for f in self._faces))
        op.inverse_weight = self._inv.data_ptr()
        op.potential = pot.data_ptr()
        op.potential_stride = pot.shape[-1] if pot.dim() > 1 else 0
        op.orbitals_per_group = int(orbitals_per_group)
        op.quadrature = self.measure.quadrature.data_ptr()
        op._keep = pot  # keep the potential alive as long as the descriptor
        return op

    def _run(self, phi: torch.Tensor, potential: torch.Tensor | None, kinetic_only: bool) -> torch.Tensor:
        _lib.require_cuda(phi, "phi")
        if phi.shape[-1] != self.grid.n_points:
            raise ValueError(f"orbitals have {phi.shape[-1]} points, grid has {self.grid.n_points}")
        x = phi.contiguous()
        if x.dtype != self.dtype:
            x = cast(x, self.dtype)
        batch = x.numel() // self.grid.n_points
        out = torch.empty_like(x)
        op = self.operator(potential)
        work = apply_workspace(op, batch, x.device)
        call("cdftb_cusp_apply", ctypes.byref(op), ptr(x), _lib.dtype_code(x), ptr(out), _lib.dtype_code(out), batch,
             1 if kinetic_only else 0, ptr(work), work.numel(), stream_handle(phi.device))
        return out

    def apply(self, phi: torch.Tensor) -> torch.Tensor:
        """``A phi`` for ``(..., N)`` orbitals, counted (hamiltonian.py:251-263)."""
        self._apply_count += 1
        return self._run(phi, None, False)

    def apply_with_potential(self, phi: torch.Tensor, potential: torch.Tensor) -> torch.Tensor:
        """(hamiltonian.py:265-276), not counted."""
        return self._run(phi, potential, False)

    def kinetic_apply(self, phi: torch.Tensor) -> torch.Tensor:
        """``(1/2 w) sum_d D_d^T[f^2_face D_d phi]`` (hamiltonian.py:303-318)."""
        return self._run(phi, None, True)

    def spectral_bounds(self, steps: int = 12, safety: float = 1.02, generator: torch.Generator | None = None):
        """Lanczos enclosure in the weighted measure (hamiltonian.py:388-396)."""
        start = seeded_randn(self.grid.n_points, generator, device=self.grid.device)
        return lanczos_bounds(self, start, steps, safety)

    # -- energies (hamiltonian.py:331-390) --
    def kinetic_energy_tensor(self, phi: torch.Tensor, occupations: torch.Tensor) -> torch.Tensor:
        occ = occupations.to(torch.float64)
        kinetic_form = self.measure.inner(phi, self.kinetic_apply(phi))
        first = (occ * kinetic_form).sum()
        rho = (occ[..., None] * phi.to(torch.float64).pow(2)).sum(dim=-2)
        cross, potential = self.quadrature.external_energy_parts(rho, self.factor)
        return first - cross - potential

    def external_energy_direct_tensor(self, rho: torch.Tensor) -> torch.Tensor:
        cross, potential = self.quadrature.external_energy_parts(rho, self.factor)
        return cross + 2.0 * potential


def cast(x: torch.Tensor, dtype: torch.dtype) -> torch.Tensor:
    """Cast a device block between float64 and float32 with the library's cast kernel."""
    if x.dtype == dtype:
        return x
    x = x.contiguous()
    out = torch.empty(x.shape, dtype=dtype, device=x.device)
    call("cdftb_cast", ptr(x), _lib.dtype_code(x), ptr(out), _lib.dtype_code(out), x.numel(), stream_handle(x.device))
    return out


def seeded_randn(shape, generator, *, device, dtype=torch.float64) -> torch.Tensor:
    """Draw on the generator's (CPU) device, then move: ``src/cdft/precision.py:246-263``.

    A :class:`~.rng.SeededStream` serves the same draws from its device cache (read-only tensors).
    """
    if hasattr(generator, "randn") and not isinstance(generator, torch.Generator):
        return generator.randn(shape)
    source = generator.device if generator is not None else torch.device("cpu")
    size = (shape,) if isinstance(shape, int) else tuple(shape)
    return torch.randn(size, device=source, dtype=dtype, generator=generator).to(device)


def lanczos_bounds(hamiltonian: CuspFactoredHamiltonian, start: torch.Tensor, steps: int, safety: float):
    """The rigorous Lanczos enclosure (``src/cdft/operators/hamiltonian.py:29-89``).

    Vectors, products and updates stay on the device (the recurrence scalars are device values
    fed to the update kernel); alpha and beta are read once after the loop and the small
    tridiagonal problem is solved on the host, as in the reference.
    """
    q = hamiltonian.measure.quadrature
    n = start.shape[-1]
    dev = start.device
    stream = stream_handle(dev)
    v = start.to(torch.float64).reshape(1, n).contiguous()
    nrm = rowwise_inner(v, v, q).clamp_min(0.0)
    v = v.clone()
    call("cdftb_lanczos_update_f64", 2, ptr(v), None, None, ptr(nrm.contiguous()), None, n, 1, stream)
    v_prev = torch.zeros_like(v)
    beta_prev = torch.zeros(1, dtype=torch.float64, device=dev)
    alphas, betas = [], []
    for _ in range(steps):
        w = hamiltonian.apply(v)
        alpha = rowwise_inner(v, w, q).contiguous()
        call("cdftb_lanczos_update_f64", 0, ptr(w), ptr(v), ptr(v_prev), ptr(alpha), ptr(beta_prev), n, 1, stream)
        c1 = rowwise_inner(w, v, q).contiguous()
        c2 = rowwise_inner(w, v_prev, q).contiguous()
        call("cdftb_lanczos_update_f64", 1, ptr(w), ptr(v), ptr(v_prev), ptr(c1), ptr(c2), n, 1, stream)
        wsq = rowwise_inner(w, w, q).clamp_min(0.0).contiguous()
        beta = wsq.sqrt()
        alphas.append(alpha)
        betas.append(beta)
        call("cdftb_lanczos_update_f64", 2, ptr(w), None, None, ptr(wsq), None, n, 1, stream)
        v_prev, v = v, w
        beta_prev = beta
    values = torch.cat([*alphas, *betas]).tolist()
    _lib.check_device_status("lanczos_bounds")
    a = values[:steps]
    b = values[steps:]
    for index, value in enumerate(b):
        if value < 1e-12:
            del a[index + 1:], b[index + 1:]
            break
    size = len(a)
    tri = np.zeros((size, size))
    for i in range(size):
        tri[i, i] = a[i]
        if i + 1 < size:
            tri[i, i + 1] = tri[i + 1, i] = b[i]
    ritz = np.linalg.eigvalsh(tri)
    residual = b[-1] if b else 0.0
    lo = float(ritz[0]) - residual
    hi = float(ritz[-1]) + residual
    centre = 0.5 * (hi + lo)
    half = 0.5 * (hi - lo) * safety
    return centre - half, centre + half
