"""Many independent systems in one set of launches: the batched SCF.

B systems that share one geometry (one grid, one set of nuclei; e.g. an ensemble of seeded starts or
perturbed runs) advance in lockstep: every field operation of an SCF iteration is one library call
over all B systems (the stencil launches B x m orbitals with one potential and one Chebyshev
coefficient table per system; the reductions, small dense steps, Poisson passes, interpolant, lift
and assembly kernels all carry a system index), while the control flow -- bounds reuse, eigensolver
stop tests, mixers, fallback ladder, convergence -- is kept per system on the host exactly as in
``src/cdft/scf/loop.py`` and ``src/cdft/eigen/chefsi.py``. A system that has converged leaves the
active set: later launches run on the compacted remainder, so its result is the one a solve of that
system alone gives. The host reads a handful of scalars per system once per eigensolver iteration
and once per SCF iteration, in one transfer for the whole batch.

Spin-restricted, any native functional (the VWN LDA on fused kernels, every other LDA and GGA on the
generic batched path); the level-shift rung of the fallback ladder runs in the single-system driver
(:mod:`.scf`).
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import F32, F64, call, ptr, stream_handle
from .eigen import BOUND_REUSE_RITZ_FRACTION, EigenConfig, chebyshev_coefficients, filter_workspace
from .geometry import CuspGeometry, gradient, partial_derivative, row_sums
from .grid import UniformGrid
from .operators import apply_workspace, cast, measure_cross, rowwise_inner
from .poisson import CoulombCutoffPoisson
from .rng import SeededStream
from .scf import (FILTER_STEPS_PER_ITERATION, BoundReusePolicy, LinearMixer, MixingConfig, SCFConfig,
                  aufbau_occupations, make_mixer, nuclear_repulsion)
from .xc import functional_by_name


class BatchedHamiltonian:
    """``A`` on B systems of one geometry: B diagonal potentials, blocks ``(B, k, N)``."""

    def __init__(self, grid, factor, quadrature, potentials: torch.Tensor, dtype=torch.float64):
        self.grid = grid
        self.quadrature = quadrature
        self.dtype = dtype
        self.potentials = potentials.contiguous()  # (B, N) float64
        faces = factor.face_weights(grid.fd_order)
        inv = quadrature.bare_operator_terms()[1]
        if dtype == torch.float64:
            self._faces = tuple(f.contiguous() for f in faces)
            self._inv = inv
            self._pot = self.potentials
        else:
            cache = factor.__dict__.setdefault("_cast_cache", {})
            key = (dtype, inv.data_ptr())
            if key not in cache:
                cache[key] = (tuple(cast(f.contiguous(), dtype) for f in faces), cast(inv.contiguous(), dtype))
            self._faces, self._inv = cache[key]
            self._pot = cast(self.potentials, dtype)
        self.q = quadrature.bare_operator_terms()[2].quadrature
        self.applications = 0

    @property
    def batch(self) -> int:
        return self.potentials.shape[0]

    def _op(self, k: int) -> _lib.Operator:
        op = _lib.Operator()
        op.nx, op.ny, op.nz = self.grid.shape
        op.accuracy = self.grid.fd_order
        op.spacing = self.grid.spacing
        op.dtype = F64 if self.dtype == torch.float64 else F32
        op.face_weights = (ctypes.c_void_p * 3)(*(f.data_ptr() for f in self._faces))
        op.inverse_weight = self._inv.data_ptr()
        op.potential = self._pot.data_ptr()
        op.potential_stride = self.grid.n_points
        op.orbitals_per_group = int(k)
        op.quadrature = self.q.data_ptr()
        return op

    def apply(self, phi: torch.Tensor, kinetic_only: bool = False) -> torch.Tensor:
        """``A phi`` for ``(B, k, N)`` orbitals (system b uses potential b)."""
        x = phi.contiguous()
        if x.dtype != self.dtype:
            x = cast(x, self.dtype)
        k = x.shape[1]
        out = torch.empty_like(x)
        op = self._op(k)
        work = apply_workspace(op, x.shape[0] * k, x.device)
        call("cdftb_cusp_apply", ctypes.byref(op), ptr(x), _lib.dtype_code(x), ptr(out), _lib.dtype_code(out),
             x.shape[0] * k, 1 if kinetic_only else 0, ptr(work), work.numel(), stream_handle(x.device))
        if not kinetic_only:
            self.applications += 1
        return out

    def filter(self, block: torch.Tensor, table: torch.Tensor, degree: int) -> torch.Tensor:
        """The fused Chebyshev filter on ``(B, k, N)`` float64 blocks, one coefficient table per system."""
        x = block.contiguous()
        b, k, n = x.shape
        out = torch.empty_like(x)
        op = self._op(k)
        work = filter_workspace(op, b * k, x.device)
        call("cdftb_chebyshev_filter", ctypes.byref(op), ptr(x), _lib.dtype_code(x), ptr(out), _lib.dtype_code(out),
             ptr(work), work.numel(), b * k, ptr(table.contiguous()), degree, stream_handle(x.device))
        self.applications += degree
        return out

    def subset(self, index: list[int]) -> "BatchedHamiltonian":
        sub = BatchedHamiltonian.__new__(BatchedHamiltonian)
        sub.__dict__.update(self.__dict__)
        idx = torch.tensor(index, dtype=torch.long, device=self.potentials.device)
        sub.potentials = self.potentials.index_select(0, idx).contiguous()
        sub._pot = sub.potentials if self.dtype == torch.float64 else cast(sub.potentials, self.dtype)
        sub.applications = 0
        return sub


class LevelShiftedBatch:
    """``H + shift (1 - P_occ)`` for every system of a batch (``src/cdft/scf/loop.py:553-589``, the
    fallback ladder's last rung): ``P_occ`` projects, in the measure, onto each system's occupied
    orbitals of the previous iteration. Applies as ``H phi + shift (phi - (phi, o) o)``; the filter is
    the reference's eager scaled recurrence over that apply (one apply launch per step, float64);
    Lanczos bounds are the inner operator's with the upper bound raised by ``shift``."""

    def __init__(self, inner: BatchedHamiltonian, occupied: torch.Tensor, shift: float) -> None:
        self.inner = inner
        self.occupied = occupied.to(torch.float64).contiguous()  # (B, k_occ, N)
        self.shift = float(shift)
        self.grid = inner.grid
        self.q = inner.q
        self.potentials = inner.potentials
        self.dtype = torch.float64
        self.applications = 0

    @property
    def batch(self) -> int:
        return self.inner.batch

    def apply(self, phi: torch.Tensor, kinetic_only: bool = False) -> torch.Tensor:
        if kinetic_only:
            return self.inner.apply(phi, kinetic_only=True)
        x = phi.to(torch.float64).contiguous()
        out = self.inner.apply(x)
        coefficients = measure_cross(x, self.occupied, self.q, x.shape[0])  # (B, k, k_occ)
        self.applications += 1
        return out + self.shift * (x - torch.bmm(coefficients, self.occupied))

    def filter(self, block: torch.Tensor, table: torch.Tensor, degree: int) -> torch.Tensor:
        """``chefsi.py:81-113`` per system with that system's rows ``(c, a_k, b_k)`` of ``table``."""
        rows = table.to(torch.float64)
        c = rows[:, :, 0][:, :, None, None]
        a = rows[:, :, 1][:, :, None, None]
        bk = rows[:, :, 2][:, :, None, None]
        x = block.to(torch.float64)
        y = (self.apply(x) - c[:, 0] * x) * a[:, 0]
        previous = x
        for k in range(1, degree):
            y_new = (self.apply(y) - c[:, k] * y) * a[:, k] - bk[:, k] * previous
            previous, y = y, y_new
        return y

    def subset(self, index: list[int]) -> "LevelShiftedBatch":
        idx = torch.tensor(index, dtype=torch.long, device=self.occupied.device)
        return LevelShiftedBatch(self.inner.subset(index), self.occupied.index_select(0, idx), self.shift)


def _enclosures(sub, starts: torch.Tensor, config: EigenConfig):
    """Lanczos bounds for every system of ``sub`` (a level-shifted batch: its inner operator's, with
    the upper bound raised by the shift, as ``_LevelShifted.spectral_bounds``)."""
    if isinstance(sub, LevelShiftedBatch):
        return [(lo, hi + sub.shift) for lo, hi in batched_lanczos(sub.inner, starts, config.lanczos_steps,
                                                                   config.bound_safety)]
    return batched_lanczos(sub, starts, config.lanczos_steps, config.bound_safety)


class _RitzBuffers:
    def __init__(self):
        self._key = None

    def get(self, b, m, device):
        if self._key != (b, m, str(device)):
            f = dict(dtype=torch.float64, device=device)
            self.lower = torch.empty((b, m, m), **f)
            self.info = torch.empty(b, dtype=torch.int32, device=device)
            self.evals = torch.empty((b, m), **f)
            self.rot = torch.empty((b, m, m), **f)
            self._key = (b, m, str(device))
        return self


_RB = _RitzBuffers()


def _row_inner(a: torch.Tensor, b: torch.Tensor, q: torch.Tensor) -> torch.Tensor:
    """``sum_p q a b`` per row of ``(B, k, N)`` blocks; ``q`` shared ``(N,)`` or per system ``(B, N)``."""
    bsz, k, n = a.shape
    if q.dim() == 1:
        return rowwise_inner(a.reshape(bsz * k, n), b.reshape(bsz * k, n), q).reshape(bsz, k)
    if k == 1:
        return measure_cross(a, b, q, bsz).reshape(bsz, 1)
    return measure_cross(a, b, q, bsz).diagonal(dim1=1, dim2=2).contiguous()


def batched_rayleigh_ritz(h: BatchedHamiltonian, block: torch.Tensor, check_orthonormality: bool = True):
    """Rayleigh--Ritz for every system (``src/cdft/eigen/rayleigh_ritz.py:51-115``), one call per step.

    Returns ``(evals (B, m), vectors (B, m, N), residual norms (B, m), orth error (B), cholesky info (B))``;
    the residual uses ``U^T (A Q)`` (U orthogonal) instead of a second apply. The orthonormality
    error of the Ritz vectors (a diagnostic: the reference only records it, chefsi.py:546-560) costs
    one more measure product; without ``check_orthonormality`` it is not formed and is ``None``.
    """
    b, m, n = block.shape
    dev = block.device
    stream = stream_handle(dev)
    q = h.q
    flat = block.to(torch.float64).contiguous()
    gram = measure_cross(flat, flat, q, b)
    rb = _RB.get(b, m, dev)
    call("cdftb_small_cholesky_f64", ptr(gram), ptr(rb.lower), ptr(rb.info), m, b, stream)
    basis = torch.empty_like(flat)
    call("cdftb_block_trsm_lower_f64", ptr(rb.lower), ptr(flat), m * n, ptr(basis), F64, m * n, m, n, b, stream)
    applied = h.apply(basis)
    sub = measure_cross(basis, applied, q, b)
    call("cdftb_small_eigh_f64", ptr(sub), ptr(rb.evals), ptr(rb.rot), m, b, stream)
    vectors = torch.empty_like(flat)
    evals = rb.evals.clone()
    if m <= 8:
        # the rotations, the residual and its norm in one pass (no rotated A Q or residual block)
        norms_sq = torch.empty((b, m), dtype=torch.float64, device=dev)
        need = _lib.library().cdftb_block_ritz_scratch_bytes(m, n, b)
        scratch = torch.empty(need, dtype=torch.uint8, device=dev)
        q_stride = 0 if q.dim() == 1 else n
        call("cdftb_block_ritz_f64", ptr(rb.rot), ptr(basis), ptr(applied), ptr(evals), ptr(q.contiguous()), q_stride,
             m, n, b, ptr(vectors), ptr(norms_sq), ptr(scratch), need, stream)
        norms = norms_sq.clamp_min(0.0).sqrt()
    else:
        call("cdftb_block_rotate_f64", ptr(rb.rot), ptr(basis), m * n, ptr(vectors), F64, m * n, m, m, n, b, stream)
        rot_applied = torch.empty_like(flat)
        call("cdftb_block_rotate_f64", ptr(rb.rot), ptr(applied), m * n, ptr(rot_applied), F64, m * n, m, m, n, b,
             stream)
        res = torch.empty_like(flat)
        call("cdftb_block_residual_f64", ptr(rot_applied), ptr(vectors), ptr(evals), ptr(res), m, n, b, m * n, stream)
        norms = _row_inner(res, res, q).clamp_min(0.0).sqrt()
    orth = None
    if check_orthonormality:
        g2 = measure_cross(vectors, vectors, q, b)
        eye = torch.eye(m, dtype=torch.float64, device=dev)
        orth = (g2 - eye).abs().amax(dim=(1, 2))
    return evals, vectors, norms, orth, rb.info.clone()


def batched_lanczos(h: BatchedHamiltonian, starts: torch.Tensor, steps: int, safety: float) -> list[tuple[float, float]]:
    """The Lanczos enclosure (``src/cdft/operators/hamiltonian.py:29-89``) for every system at once."""
    b, n = starts.shape
    q = h.q
    dev = starts.device
    stream = stream_handle(dev)
    v = starts.to(torch.float64).clone().contiguous()

    def rowwise_inner(x, y, q):
        return _row_inner(x.reshape(b, 1, n), y.reshape(b, 1, n), q).reshape(b)

    nrm = rowwise_inner(v, v, q).clamp_min(0.0).contiguous()
    call("cdftb_lanczos_update_f64", 2, ptr(v), None, None, ptr(nrm), None, n, b, stream)
    v_prev = torch.zeros_like(v)
    beta_prev = torch.zeros(b, dtype=torch.float64, device=dev)
    alphas, betas = [], []
    for _ in range(steps):
        w = h.apply(v.reshape(b, 1, n)).reshape(b, n).contiguous()
        alpha = rowwise_inner(v, w, q).contiguous()
        call("cdftb_lanczos_update_f64", 0, ptr(w), ptr(v), ptr(v_prev), ptr(alpha), ptr(beta_prev), n, b, stream)
        c1 = rowwise_inner(w, v, q).contiguous()
        c2 = rowwise_inner(w, v_prev, q).contiguous()
        call("cdftb_lanczos_update_f64", 1, ptr(w), ptr(v), ptr(v_prev), ptr(c1), ptr(c2), n, b, stream)
        wsq = rowwise_inner(w, w, q).clamp_min(0.0).contiguous()
        beta = wsq.sqrt()
        alphas.append(alpha)
        betas.append(beta)
        call("cdftb_lanczos_update_f64", 2, ptr(w), None, None, ptr(wsq), None, n, b, stream)
        v_prev, v = v, w
        beta_prev = beta
    values = torch.stack([*alphas, *betas]).cpu().numpy()  # (2 steps, b)
    _lib.check_device_status("batched_lanczos")
    out = []
    for s in range(b):
        a = list(values[:steps, s])
        bt = list(values[steps:, s])
        for index, value in enumerate(bt):
            if value < 1e-12:
                del a[index + 1:], bt[index + 1:]
                break
        size = len(a)
        tri = np.zeros((size, size))
        for i in range(size):
            tri[i, i] = a[i]
            if i + 1 < size:
                tri[i, i + 1] = tri[i + 1, i] = bt[i]
        ritz = np.linalg.eigvalsh(tri)
        residual = bt[-1] if bt else 0.0
        lo, hi = float(ritz[0]) - residual, float(ritz[-1]) + residual
        centre, half = 0.5 * (hi + lo), 0.5 * (hi - lo) * safety
        out.append((centre - half, centre + half))
    return out


@dataclass
class _EigenState:
    spectrum: tuple | None = None
    source: str = "unset"
    shift: float = 0.0
    next_lower: float = 0.0
    previous: np.ndarray | None = None
    top_fraction: float = float("-inf")
    converged: bool = False
    iterations: int = 0
    stop_reason: str = "iteration limit"
    float_filter: bool = False
    stable: int = 0
    applications: int = 0  # block applications of this system's operator (Lanczos, filter, Ritz)


def _stable(state, drift: float, tol: float) -> bool:
    """Count consecutive iterations whose Ritz drift is below ``tol``; true at the second."""
    state.stable = state.stable + 1 if drift < tol else 0
    return state.stable >= 2


def _fraction(value, low, high):
    width = high - low
    return (value - low) / width if width > 0.0 else float("inf")


def batched_chefsi(h: BatchedHamiltonian, h32: BatchedHamiltonian | None, n_states: int, config: EigenConfig,
                   initial: torch.Tensor | None, streams: list[SeededStream], bounds: list, max_iterations: int,
                   switch_residual: float | None, ritz_stop: bool = False, float_mask: list | None = None,
                   stop_at_switch: bool = False):
    """CheFSI for every system of ``h`` (``src/cdft/eigen/chefsi.py:442-585``).

    ``ritz_stop`` adds the weak-form stop of the bare-nucleus path: Ritz values stable (drift below
    a tenth of ``cross_check_tol``) on two iterations in a row.

    ``float_mask[b]`` (default: every system) marks the systems that start in float filtering when
    ``h32`` is given; each leaves it on its own at ``switch_residual``, to go on in float64 or, with
    ``stop_at_switch``, to stop there. A step filters the float systems in one float launch and the
    others in one float64 launch.

    ``bounds[b]`` is ``None`` (run Lanczos) or ``(lower, upper, shift)``. Returns per-system
    eigenvalues ``(B, n_states)``, eigenvectors ``(B, n_states, N)``, residuals ``(B, n_states)``,
    and the per-system states (bounds used, source, iterations, stop reason).
    """
    b = h.batch
    n = h.grid.n_points
    dev = h.potentials.device
    extra = max(config.n_extra_states, int(config.extra_states_fraction * n_states))
    m = min(n_states + extra, n)
    # the start block, written once in place: the carried vectors, then each system's fresh draws
    # (one gather of the b draws and one copy of the carried rows, not a copy per system)
    if initial is None:
        block = torch.stack([streams[s].randn((m, n)) for s in range(b)])
    else:
        carried = initial.reshape(b, -1, n)
        k = min(carried.shape[1], m)
        block = torch.empty((b, m, n), dtype=torch.float64, device=dev)
        block[:, :k] = carried[:, :k]
        if k < m:
            block[:, k:] = torch.stack([streams[s].randn((m - k, n)) for s in range(b)])
    states = [_EigenState(float_filter=h32 is not None and (float_mask is None or bool(float_mask[s])))
              for s in range(b)]
    need = [s for s in range(b) if bounds[s] is None]
    if need:
        starts = torch.stack([streams[s].randn(n) for s in need])
        sub = h if len(need) == b else h.subset(need)
        for s, bb in zip(need, _enclosures(sub, starts, config)):
            states[s].spectrum = bb
            states[s].source = "lanczos"
            states[s].applications += config.lanczos_steps
        h.applications += sub.applications if sub is not h else 0
    evals, vectors, residual, _, _ = batched_rayleigh_ritz(h, block, check_orthonormality=False)
    for st in states:
        st.applications += 1
    top = m - 1
    tops = evals[:, top].tolist()
    for s in range(b):
        st = states[s]
        st.next_lower = tops[s]
        if bounds[s] is not None:
            lo, hi, shift = bounds[s]
            st.spectrum = (lo - shift, hi + shift)
            st.source = "reused"
            st.shift = shift
    previous = evals.clone()
    # results per system, kept for the n_states wanted rows only (the others are never returned)
    out_evals = evals[:, :n_states].clone()
    out_vectors = vectors[:, :n_states].clone()
    out_res = residual[:, :n_states].clone()
    active = list(range(b))
    for iteration in range(1, max_iterations + 1):
        # per-system filter intervals (and a fresh Lanczos where a carried bound is rejected)
        redo = []
        for s in active:
            st = states[s]
            lower = st.next_lower
            lo, hi = st.spectrum
            frac = _fraction(lower, lo, hi)
            if st.source == "reused" and not frac < BOUND_REUSE_RITZ_FRACTION:
                redo.append(s)
        if redo:
            starts = torch.stack([streams[s].randn(n) for s in redo])
            sub = h.subset(redo)
            for s, bb in zip(redo, _enclosures(sub, starts, config)):
                states[s].spectrum = bb
                states[s].source = "lanczos (reuse rejected)"
                states[s].applications += config.lanczos_steps
            h.applications += sub.applications
        rows = []
        use_float = []
        for s in active:
            st = states[s]
            lo, hi = st.spectrum
            lower = st.next_lower
            st.top_fraction = max(st.top_fraction, _fraction(lower, lo, hi))
            lower = min(max(lower, lo + 1e-8), hi - 1e-8)
            rows.append(chebyshev_coefficients(config.chebyshev_degree, lower, hi, lo))
            use_float.append(st.float_filter)
        table = torch.tensor(rows, dtype=torch.float64).pin_memory().to(dev, non_blocking=True)
        full = len(active) == b
        sel = None if full else torch.tensor(active, dtype=torch.long, device=dev)
        hv = h if full else h.subset(active)
        cur = vectors if full else vectors.index_select(0, sel)
        # systems in their float phase filter in float, the others in float64 (one launch each)
        if h32 is not None and all(use_float):
            hf = h32 if full else h32.subset(active)
            filtered = hf.filter(cur, table, config.chebyshev_degree)
        elif h32 is not None and any(use_float):
            fpos = [j for j, u in enumerate(use_float) if u]
            dpos = [j for j, u in enumerate(use_float) if not u]
            filtered = torch.empty_like(cur)
            for pos, ham in ((fpos, h32), (dpos, h)):
                idx = torch.tensor(pos, dtype=torch.long, device=dev)
                part = ham.subset([active[j] for j in pos])
                filtered.index_copy_(0, idx, part.filter(cur.index_select(0, idx), table.index_select(0, idx),
                                                         config.chebyshev_degree))
        else:
            filtered = hv.filter(cur, table, config.chebyshev_degree)
        ev, vec, res, _, info = batched_rayleigh_ritz(hv, filtered, check_orthonormality=False)
        prev = previous if full else previous.index_select(0, sel)
        drift = (ev[:, :n_states] - prev[:, :n_states]).abs().amax(dim=1)
        worst = res[:, :n_states].amax(dim=1)
        host = torch.stack([worst, drift, ev[:, top], info.to(torch.float64)]).cpu().numpy()
        _lib.check_device_status(f"batched CheFSI iteration {iteration}")
        if (host[3] != 0).any():
            raise RuntimeError("a filtered block lost rank (Cholesky failed) in the batched solver; "
                               "solve that system with the single-system driver")
        if full:
            vectors, evals, residual = vec, ev, res
        else:
            vectors.index_copy_(0, sel, vec)
            evals.index_copy_(0, sel, ev)
            residual.index_copy_(0, sel, res)
        previous = evals.clone()
        still = []
        done = []
        for j, s in enumerate(active):
            st = states[s]
            st.iterations = iteration
            st.applications += config.chebyshev_degree + 1  # the filter and the Rayleigh--Ritz apply
            st.next_lower = float(host[2, j])
            if host[0, j] < config.residual_tol:
                st.converged = True
                st.stop_reason = "residual below residual_tol"
                done.append(s)
            elif ritz_stop and _stable(st, host[1, j], 0.1 * config.cross_check_tol):
                st.converged = True
                st.stop_reason = "Ritz values stable on the weak-form path"
                done.append(s)
            else:
                still.append(s)
            if st.float_filter and switch_residual is not None and host[0, j] < switch_residual:
                st.float_filter = False
                if stop_at_switch and not st.converged:
                    st.converged = True
                    st.stop_reason = "residual below the float-filter switch"
                    done.append(s)
                    still.remove(s)
        if done:
            _keep(out_evals, out_vectors, out_res, done, evals, vectors, residual, n_states, dev)
        active = still
        if not active:
            break
    if active:
        _keep(out_evals, out_vectors, out_res, active, evals, vectors, residual, n_states, dev)
    return out_evals, out_vectors, out_res, states


def _keep(out_evals, out_vectors, out_res, systems, evals, vectors, residual, n_states, dev):
    """Copy the wanted rows of these systems' current results into the outputs, in place."""
    if len(systems) == out_vectors.shape[0]:
        out_evals.copy_(evals[:, :n_states])
        out_vectors.copy_(vectors[:, :n_states])
        out_res.copy_(residual[:, :n_states])
        return
    idx = torch.tensor(systems, dtype=torch.long, device=dev)
    out_evals.index_copy_(0, idx, evals[:, :n_states].index_select(0, idx))
    out_vectors.index_copy_(0, idx, vectors[:, :n_states].index_select(0, idx))
    out_res.index_copy_(0, idx, residual[:, :n_states].index_select(0, idx))


@dataclass
class BatchedPotentials:
    effective: torch.Tensor        # (B, N)
    v_hartree: torch.Tensor        # (B, N)
    hartree_energy: torch.Tensor   # (B,)
    xc_energy: torch.Tensor        # (B,)
    xc_double_counting: torch.Tensor  # (B,)
    v_smooth: torch.Tensor | None = None  # (B, N): the Poisson solution of the smooth density
    node: torch.Tensor | None = None      # (2, B, M): rho and v_smooth at the quadrature nodes
    lifted_h: torch.Tensor | None = None  # (B, N): L^T of the Hartree node weights


class BatchedKohnShamStep:
    """The KS map for B systems sharing one geometry (``src/cdft/scf/step.py`` semantics per system)."""

    FLOAT_FILTER_SWITCH_RESIDUAL = 1.0e-4

    def __init__(self, geometry: CuspGeometry, functional: str, n_electrons: float, batch: int,
                 eigen: EigenConfig | None = None, *, seeds=None, pad_factor: float = 2.5,
                 filter_precision: torch.dtype = torch.float64) -> None:
        self.geometry = geometry
        self.grid = geometry.grid
        self.factor = geometry.factor
        self.quadrature = geometry.quadrature
        self.functional = functional_by_name(functional)
        self.batch = int(batch)
        self.n_electrons = float(n_electrons)
        self.n_states = max(1, int(-(-self.n_electrons // 2.0)))
        from .carriers import eigen_config
        self.eigen = eigen_config(eigen)
        self.seeds = list(seeds) if seeds is not None else list(range(self.batch))
        if len(self.seeds) != self.batch:
            raise ValueError("one seed per system")
        self.ion_ion = nuclear_repulsion(geometry.charges, geometry.positions)
        self.poisson = CoulombCutoffPoisson(self.grid, pad_factor=pad_factor, max_batch=self.batch)
        self.filter_precision = filter_precision
        self.f2 = self.factor.weight
        self.bare_potential = self.quadrature.bare_operator_terms()[0]
        self.occ = torch.from_numpy(aufbau_occupations(self.n_states, self.n_electrons)[0]).to(self.grid.device)

    def potentials(self, density: torch.Tensor, v_smooth: torch.Tensor | None = None,
                   node: torch.Tensor | None = None, lifted_h: torch.Tensor | None = None) -> BatchedPotentials:
        """(``src/cdft/scf/step.py:224-313``) for ``(B, N)`` total densities, LDA.

        The smooth density (the total minus the cusp terms, whose coefficients solve a fixed linear
        system), its Poisson solution ``v_smooth``, the node values ``node`` of rho and v_smooth, and
        the lifted Hartree weights ``lifted_h`` are all linear in the density. A caller that already
        holds them for this density -- the same linear combination of earlier results as the density
        is of earlier densities -- passes them, and the Poisson solve, the interpolation and the
        Hartree half of the lift are skipped (the XC half is not linear and is always lifted).
        """
        if self.functional.name != "lda_vwn":
            return self._potentials_generic(density)
        g = self.geometry
        q = self.quadrature
        grid = self.grid
        n = grid.n_points
        m = q.n_nodes
        na = len(g.charges)
        b = density.shape[0]
        dev = grid.device
        stream = stream_handle(dev)
        f = dict(dtype=torch.float64, device=dev)
        n_grid = density.to(torch.float64).contiguous()
        fields = torch.empty((2, b, n), **f)  # [rho | v_smooth]
        rho = fields[0]
        n_smooth = torch.empty((b, n), **f)
        call("cdftb_hartree_split_f64", ptr(n_grid), ptr(self.f2), None, None, 0, n, b, ptr(rho), ptr(n_smooth), stream)
        rho_nuc = torch.empty((b, na), **f)
        call("cdftb_quadrature_interpolate_f64", ptr(g.step.nuclei_base), ptr(g.step.nuclei_w1d), na, *grid.shape,
             ptr(rho), b, n, ptr(rho_nuc), na, stream)
        coef = torch.empty((b, na), **f)
        call("cdftb_cusp_coefficients_f64", ptr(rho_nuc), ptr(g.step.nucleus_f2), ptr(g.step.overlap), na, b,
             ptr(coef), stream)
        if v_smooth is None:
            call("cdftb_hartree_split_f64", ptr(n_grid), ptr(self.f2), ptr(g.step.cusp_grid), ptr(coef), na, n, b,
                 ptr(rho), ptr(n_smooth), stream)
            self.poisson.solve_batch(n_smooth, out=fields[1])
        else:
            fields[1].copy_(v_smooth)
        if node is None:
            node = q._interp_raw(fields.reshape(2 * b, n), 2 * b).reshape(2, b, m)
        else:
            node = node.contiguous()
        lift_in = torch.empty((b, 2, m), **f)
        e_w = torch.empty((b, m), **f)
        call("cdftb_potentials_node_lda_f64", ptr(node), m, ptr(q.weights), ptr(q.f2), ptr(g.step.v1s_node),
             ptr(coef), na, b, ptr(lift_in), ptr(e_w), stream)
        if lifted_h is None:
            lifted = q._lift_raw(lift_in, 2 * b).reshape(b, 2, n)
        else:
            lifted = torch.empty((b, 2, n), **f)
            lifted[:, 0] = lifted_h
            lifted[:, 1] = q._lift_raw(lift_in[:, 1].contiguous(), b)
        effective = torch.empty((b, n), **f)
        v_hartree = torch.empty((b, n), **f)
        terms = torch.empty((b, 3, n), **f)
        call("cdftb_potentials_grid_lda_f64", ptr(n_grid), ptr(rho), ptr(self.f2), ptr(q.far_weights),
             ptr(q.mass_weights), ptr(fields[1]), ptr(g.step.v1s_grid), ptr(coef), na, ptr(lifted), n, b,
             ptr(effective), ptr(v_hartree), ptr(terms), None, stream)
        sums = row_sums(terms)  # (b, 3)
        node_sum = row_sums(e_w)  # (b,)
        return BatchedPotentials(effective=effective, v_hartree=v_hartree, hartree_energy=0.5 * sums[:, 0],
                                 xc_energy=node_sum + sums[:, 2], xc_double_counting=sums[:, 1], v_smooth=fields[1],
                                 node=node, lifted_h=lifted[:, 0])

    def _potentials_generic(self, density: torch.Tensor) -> BatchedPotentials:
        """Potentials for any native functional (``src/cdft/scf/step.py:224-313``) for ``(B, N)``
        densities: the single-system generic path (``scf.KohnShamStep._potentials_generic``) with a
        system axis on every array, the functional evaluated on all systems' points in one call and a
        GGA's gradient term in weak form (lift and FD transpose, step.py:252-280). No linear parts are
        returned, so the driver solves the Poisson problem of every input density."""
        g = self.geometry
        q = self.quadrature
        grid = self.grid
        factor = self.factor
        n = grid.n_points
        m = q.n_nodes
        na = len(g.charges)
        b = density.shape[0]
        dev = grid.device
        stream = stream_handle(dev)
        f = dict(dtype=torch.float64, device=dev)
        gga = self.functional.rung >= 2
        f2 = self.f2
        n_grid = density.to(torch.float64).contiguous()
        rho = torch.empty((b, n), **f)
        n_smooth = torch.empty((b, n), **f)
        call("cdftb_hartree_split_f64", ptr(n_grid), ptr(f2), None, None, 0, n, b, ptr(rho), ptr(n_smooth), stream)
        rho_nuc = torch.empty((b, na), **f)
        call("cdftb_quadrature_interpolate_f64", ptr(g.step.nuclei_base), ptr(g.step.nuclei_w1d), na, *grid.shape,
             ptr(rho), b, n, ptr(rho_nuc), na, stream)
        coef = torch.empty((b, na), **f)
        call("cdftb_cusp_coefficients_f64", ptr(rho_nuc), ptr(g.step.nucleus_f2), ptr(g.step.overlap), na, b,
             ptr(coef), stream)
        call("cdftb_hartree_split_f64", ptr(n_grid), ptr(f2), ptr(g.step.cusp_grid), ptr(coef), na, n, b, ptr(rho),
             ptr(n_smooth), stream)
        v_smooth = self.poisson.solve_batch(n_smooth)
        v_h_grid = (coef[:, :, None] * g.step.v1s_grid[None]).sum(dim=1) + v_smooth
        if gga:
            grad_rho = gradient(grid, rho)  # (B, 3, N)
            node = q.interpolate(torch.cat([rho[:, None], grad_rho, v_smooth[:, None]], dim=1))  # (B, 5, M)
            rho_node, grad_rho_node, vs_node = node[:, 0], node[:, 1:4], node[:, 4]
        else:
            node = q.interpolate(torch.stack([rho, v_smooth], dim=1))  # (B, 2, M)
            rho_node, vs_node = node[:, 0], node[:, 1]
        v_h_node = (coef[:, :, None] * g.step.v1s_node[None]).sum(dim=1) + vs_node
        n_node = q.f2[None] * rho_node
        if gga:
            grad_n_node = q.f2[None, None] * (grad_rho_node - 2.0 * rho_node[:, None] * q.grad_u[None])
            grad_n_grid = f2[None, None] * (grad_rho - 2.0 * rho[:, None] * factor.grad_u[None])
            sigma_grid = (grad_n_grid * grad_n_grid).sum(dim=1)
            sigma_node = (grad_n_node * grad_n_node).sum(dim=1)
            out_grid = self.functional.evaluate(n_grid.reshape(1, b * n), sigma_grid.reshape(1, b * n))
            out_node = self.functional.evaluate(n_node.reshape(1, b * m), sigma_node.reshape(1, b * m))
        else:
            out_grid = self.functional.evaluate(n_grid.reshape(1, b * n))
            out_node = self.functional.evaluate(n_node.reshape(1, b * m))
        e_n_node, e_n_grid = out_node.v_xc.reshape(b, m), out_grid.v_xc.reshape(b, n)
        parts = [(q.weights[None] * (q.f2[None] * v_h_node))[:, None], (q.weights[None] * (q.f2[None] * e_n_node))[:, None]]
        if gga:
            e_s_node, e_s_grid = out_node.v_sigma.reshape(b, m), out_grid.v_sigma.reshape(b, n)
            flux_node = 2.0 * e_s_node[:, None] * q.f2[None, None] * grad_n_node
            flux_grid = 2.0 * e_s_grid[:, None] * f2[None, None] * grad_n_grid
            cross_node = -2.0 * (flux_node * q.grad_u[None]).sum(dim=1)
            cross_grid = -2.0 * (flux_grid * factor.grad_u[None]).sum(dim=1)
            parts += [q.weights[None, None] * flux_node, (q.weights[None] * cross_node)[:, None]]
        lifted = q.lift(torch.cat(parts, dim=1).contiguous())  # (B, 2 or 6, N)
        hartree_w = lifted[:, 0] + q.far_weights[None] * (f2[None] * v_h_grid)
        xc_w = lifted[:, 1] + q.far_weights[None] * (f2[None] * e_n_grid)
        if gga:
            # lumped_gradient_weights: -sum_d D_d [L^T(w flux_d) + h^3 far flux_grid_d]
            pre = lifted[:, 2:5] + grid.volume_element * (q.far[None, None] * flux_grid)
            div = torch.zeros((b, n), **f)
            for d in range(3):
                partial_derivative(grid, pre[:, d].contiguous(), d, out=div, accumulate=True, sign=-1.0)
            xc_w = xc_w + div
            xc_w = xc_w + (lifted[:, 5] + q.far_weights[None] * cross_grid)
        hartree_energy = 0.5 * row_sums(hartree_w * rho)
        xc_energy = row_sums(q.weights[None] * out_node.e_xc.reshape(b, m)) + \
            row_sums(q.far_weights[None] * out_grid.e_xc.reshape(b, n))
        xc_dc = row_sums(xc_w * rho)
        effective = (hartree_w + xc_w) / q.mass_weights[None]
        return BatchedPotentials(effective=effective, v_hartree=v_h_grid, hartree_energy=hartree_energy,
                                 xc_energy=xc_energy, xc_double_counting=xc_dc)

    def hamiltonian(self, effective: torch.Tensor, dtype=torch.float64) -> BatchedHamiltonian:
        return BatchedHamiltonian(self.grid, self.factor, self.quadrature, self.bare_potential[None, :] + effective,
                                  dtype=dtype)

    def output_density(self, vectors: torch.Tensor):
        rho_out = (self.occ[None, :, None] * vectors.pow(2)).sum(dim=1)  # (B, N)
        return rho_out * self.f2[None, :], rho_out

    def output_density_residual(self, vectors: torch.Tensor, n_in: torch.Tensor):
        """:meth:`output_density` and the integrand of the density residual norm in one pass.

        Returns ``(n_out, rho_out, terms)`` with ``terms = mass |n_out - n_in| / f^2`` per point, whose
        row sums are the residual norms (``src/cdft/scf/loop.py:298-301, 375-376``).
        """
        v = vectors.to(torch.float64).contiguous()
        b, k, n = v.shape
        x = n_in.to(torch.float64).contiguous()
        f = dict(dtype=torch.float64, device=v.device)
        rho_out, n_out, terms = torch.empty((b, n), **f), torch.empty((b, n), **f), torch.empty((b, n), **f)
        occ = self.occ.to(torch.float64).contiguous()
        call("cdftb_density_residual_f64", ptr(v), ptr(occ), k, n, b, ptr(self.f2),
             ptr(self.quadrature.mass_weights.contiguous()), ptr(x), ptr(rho_out), ptr(n_out), ptr(terms),
             stream_handle(v.device))
        return n_out, rho_out, terms

    def external_parts(self, rho: torch.Tensor, rho_node: torch.Tensor | None = None):
        """``((1/2)Q[f^2 grad rho . grad u], Q[f^2 rho W])`` per system (hamiltonian.py:360-378).

        ``rho_node`` (B, M): ``L rho`` when the caller already holds it (the output potentials
        interpolate the same density), so that only the gradient is interpolated here.
        """
        q = self.quadrature
        factor = self.factor
        b, n = rho.shape
        grad = gradient(self.grid, rho)  # (B, 3, N)
        if rho_node is None:
            fields = torch.cat([rho[:, None], grad], dim=1).contiguous()  # (B, 4, N)
            node = q.interpolate(fields)  # (B, 4, M)
            rho_node, grad_node = node[:, 0], node[:, 1:]
        else:
            grad_node = q.interpolate(grad.contiguous())  # (B, 3, M)
        cross_node = q.f2[None] * (grad_node * q.grad_u[None]).sum(dim=1)
        # the grid halves of both integrals in one pass: (far_w weight grad rho . grad u, far_w weight rho W)
        grid_terms = torch.empty((b, 2, n), dtype=torch.float64, device=rho.device)
        call("cdftb_external_grid_terms_f64", ptr(grad.contiguous()), ptr(rho.contiguous()),
             ptr(factor.weight.contiguous()), ptr(factor.grad_u.contiguous()),
             ptr(factor.transformed_potential.contiguous()), ptr(q.far_weights.contiguous()), n, b, ptr(grid_terms),
             stream_handle(rho.device))
        grid_sums = row_sums(grid_terms)  # (B, 2)
        cross = 0.5 * (row_sums(q.weights[None] * cross_node) + grid_sums[:, 0])
        pot = row_sums(q.weights[None] * (q.f2[None] * rho_node * q.transformed_potential[None])) + grid_sums[:, 1]
        return cross, pot

    def energy_terms(self, evals, vectors, rho_out, p_in: BatchedPotentials, p_out: BatchedPotentials):
        """(``src/cdft/scf/step.py:398-439``) per system, as (B,) device tensors."""
        q = self.quadrature
        b, k, n = vectors.shape
        band = (self.occ[None] * evals).sum(dim=1)
        h = BatchedHamiltonian(self.grid, self.factor, self.quadrature,
                               self.bare_potential[None].expand(b, n).contiguous())
        kin = h.apply(vectors, kinetic_only=True)
        kinetic_form = rowwise_inner(vectors.reshape(b * k, n), kin.reshape(b * k, n), h.q).reshape(b, k)
        first = (self.occ[None] * kinetic_form).sum(dim=1)
        cross, pot = self.external_parts(rho_out, p_out.node[0] if p_out.node is not None else None)
        kinetic = first - cross - pot
        dc_out = row_sums(p_in.effective * q.mass_weights[None] * rho_out)
        kpe = band - dc_out
        harris = band - p_in.hartree_energy - p_in.xc_double_counting + p_in.xc_energy + self.ion_ion
        total = kpe + p_out.hartree_energy + p_out.xc_energy + self.ion_ion
        external = total - kinetic - p_out.hartree_energy - p_out.xc_energy - self.ion_ion
        return {"total": total, "kinetic": kinetic, "external": external, "hartree": p_out.hartree_energy,
                "xc": p_out.xc_energy, "harris_foulkes": harris, "band": band, "external_direct": cross + 2.0 * pot}

    def initial_density(self) -> torch.Tensor:
        from .scf import KohnShamStep, initial_density

        one = initial_density(_InitialDensityView(self))
        return one.expand(self.batch, -1).contiguous()


class _InitialDensityView:
    """The attributes :func:`scf.initial_density` reads, taken from a batched step."""

    def __init__(self, step: BatchedKohnShamStep):
        self.geometry = step.geometry
        self.grid = step.grid
        self._f2_grid = step.f2
        self.quadrature = step.quadrature
        self.n_electrons = step.n_electrons


@dataclass
class _SystemState:
    mixer: object
    policy: BoundReusePolicy
    rung: int = 0
    worsened: int = 0
    previous_residual: float = float("inf")
    energies: list = field(default_factory=list)
    residuals: list = field(default_factory=list)
    converged: bool = False
    iterations: int = 0
    applications: int = 0
    float_phase: bool = False
    refinement_from: int | None = None
    rung_changed: bool = False
    fallback_events: list = field(default_factory=list)
    level_shift: float = 0.0


@dataclass
class BatchedOutcome:
    energies: list            # per system dict of floats
    eigenvalues: list         # per system list
    scf_iterations: list
    converged: list
    applications: float
    density: torch.Tensor     # (B, N)
    measurements: dict = field(default_factory=dict)


def solve_self_consistent_batch(step: BatchedKohnShamStep, mixing: MixingConfig | None = None,
                                scf: SCFConfig | None = None, *, initial_density: torch.Tensor | None = None,
                                max_iterations: int | None = None) -> BatchedOutcome:
    """``src/cdft/scf/loop.py:255-550`` for B systems at once (see the module docstring).

    With ``step.filter_precision == torch.float32`` each system filters in float until it meets the
    convergence test, then refines in float64 until the test passes again (the FP64 refinement
    sweep); the final full diagonalisation filters in float64.
    """
    started = time.perf_counter()
    from .carriers import mixing_config, scf_config
    mixing = mixing_config(mixing)
    scf = scf_config(scf)
    b = step.batch
    dev = step.grid.device
    q = step.quadrature
    mass, f2 = q.mass_weights, step.f2
    inner_weights = (mass / f2 ** 2).contiguous()
    mixed = step.filter_precision == torch.float32

    def make(alpha, scheme=None):
        return make_mixer(mixing, alpha, inner_weights, scheme, grid=step.grid)

    systems = [_SystemState(mixer=make(mixing.alpha), policy=BoundReusePolicy(), float_phase=mixed) for _ in range(b)]
    n_in = (initial_density if initial_density is not None else step.initial_density()).to(torch.float64).clone()
    if n_in.shape[0] != b:
        n_in = n_in.expand(b, -1).contiguous()
    initial_block = None
    previous_effective = None
    lin_in = None  # (v_smooth, node, lifted_h) of n_in, carried by linearity while every mixer is linear
    limit = scf.max_iterations if max_iterations is None else max_iterations
    active = list(range(b))
    last_p_in = [None] * b
    last_vectors = [None] * b
    p_in_all = None
    for iteration in range(1, limit + 1):
        if not active:
            break
        sel = torch.tensor(active, dtype=torch.long, device=dev)
        full = len(active) == b
        nin = n_in if full else n_in.index_select(0, sel)
        lin = None
        if lin_in is not None:
            lin = lin_in if full else (lin_in[0].index_select(0, sel), lin_in[1].index_select(1, sel),
                                       lin_in[2].index_select(0, sel))
        p_in = step.potentials(nin, *(lin or ()))
        h = step.hamiltonian(p_in.effective)
        float_now = [systems[s].float_phase for s in active]
        h32 = step.hamiltonian(p_in.effective, dtype=torch.float32) if any(float_now) else None
        hints = []
        shifts = None
        if previous_effective is not None:
            prev = previous_effective if full else previous_effective.index_select(0, sel)
            shifts = (p_in.effective - prev).abs().amax(dim=1).tolist()
        for j, s in enumerate(active):
            st = systems[s]
            reason = st.policy.decide(residual_rose=st.worsened > 0, rung_changed=st.rung_changed,
                                      level_shift=bool(st.level_shift))
            if reason is None and shifts is not None:
                hints.append((st.policy.bounds[0], st.policy.bounds[1], shifts[j]))
            else:
                hints.append(None)
            st.policy._pending_reason = reason
        streams = [SeededStream(step.seeds[s], dev) for s in active]
        init = None if initial_block is None else (initial_block if full else initial_block.index_select(0, sel))
        steps_cap = step.eigen.max_iterations if init is None else FILTER_STEPS_PER_ITERATION
        switch = step.FLOAT_FILTER_SWITCH_RESIDUAL if init is None else None
        h.applications = 0
        # The first full diagonalisation of a mixed solve stops at the float switch: the float phase
        # that follows holds float accuracy anyway, and the float64 refinement sweep and the final
        # float64 diagonalisation set the result's.
        shifted = [j for j, s in enumerate(active) if systems[s].level_shift]
        if not shifted:
            evals, vectors, _, estates = batched_chefsi(h, h32, step.n_states, step.eigen, init, streams, hints,
                                                        steps_cap, switch, float_mask=float_now, stop_at_switch=mixed)
        else:
            # systems on the level-shift rung diagonalise H + shift (1 - P_occ), in float64, in a call of
            # their own (loop.py:353-356: the filter then runs eagerly over the shifted apply)
            plain = [j for j in range(len(active)) if j not in shifted]
            n_occ = int((step.occ > 1e-12).sum())
            evals = torch.empty((len(active), step.n_states), dtype=torch.float64, device=dev)
            vectors = torch.empty((len(active), step.n_states, n), dtype=torch.float64, device=dev)
            estates = [None] * len(active)
            for part, is_shifted in ((plain, False), (shifted, True)):
                if not part:
                    continue
                hp = h.subset(part)
                sub_init = init.index_select(0, torch.tensor(part, dtype=torch.long, device=dev))
                if is_shifted:
                    hp = LevelShiftedBatch(hp, sub_init[:, :n_occ], systems[active[part[0]]].level_shift)
                    hf, fmask = None, None
                else:
                    hf = None if h32 is None else h32.subset(part)
                    fmask = [float_now[j] for j in part]
                ev_p, vec_p, _, es_p = batched_chefsi(hp, hf, step.n_states, step.eigen, sub_init,
                                                      [streams[j] for j in part], [hints[j] for j in part],
                                                      steps_cap, switch if not is_shifted else None, float_mask=fmask,
                                                      stop_at_switch=mixed and not is_shifted)
                idx = torch.tensor(part, dtype=torch.long, device=dev)
                evals.index_copy_(0, idx, ev_p)
                vectors.index_copy_(0, idx, vec_p)
                for j, es in zip(part, es_p):
                    estates[j] = es
        for j, s in enumerate(active):
            st = systems[s]
            es = estates[j]
            info = {"eigen_spectral_bounds": list(es.spectrum), "eigen_top_ritz_fraction": es.top_fraction,
                    "eigen_bounds_source": es.source, "eigen_bounds_shift": es.shift}
            st.policy.observe(st.policy._pending_reason, info)
            st.rung_changed = False
        n_out, rho_out, res_terms = step.output_density_residual(vectors, nin)
        p_out = step.potentials(n_out)
        terms = step.energy_terms(evals, vectors, rho_out, p_in, p_out)
        res_norm = row_sums(res_terms)
        keys = list(terms)
        host = torch.stack([*terms.values(), res_norm]).cpu().numpy()  # (len(keys)+1, S)
        _lib.check_device_status(f"batched SCF iteration {iteration}")
        # mixing (per system: linear in one batched expression when all are linear)
        n_next = torch.empty_like(nin)
        # a preconditioned residual is not the difference of the two densities' linear parts
        linear = all(isinstance(systems[s].mixer, LinearMixer) and systems[s].mixer.preconditioner is None
                     for s in active) and p_in.v_smooth is not None
        lin_next = None
        if linear:
            # x_in + alpha (x_out - x_in) per system (LinearMixer.mix, element for element) in one expression per
            # array, for the density and for the linear parts of the two potentials
            alpha = torch.tensor([systems[s].mixer.alpha for s in active], dtype=torch.float64, device=dev)
            a2 = alpha[:, None]
            n_next = nin + a2 * (n_out - nin)
            # the carried linear parts need no element-for-element match: one lerp pass each
            lin_next = (torch.lerp(p_in.v_smooth, p_out.v_smooth, a2),
                        torch.lerp(p_in.node, p_out.node, alpha[None, :, None]),
                        torch.lerp(p_in.lifted_h, p_out.lifted_h, a2))
        else:
            for j, s in enumerate(active):
                n_next[j] = systems[s].mixer.mix(nin[j:j + 1], n_out[j:j + 1], iteration)[0]
        new_active = []
        for j, s in enumerate(active):
            st = systems[s]
            st.iterations = iteration
            st.applications += estates[j].applications
            total = float(host[keys.index("total"), j])
            rn = float(host[-1, j])
            st.energies.append(total)
            st.residuals.append(rn)
            de = abs(st.energies[-1] - st.energies[-2]) if len(st.energies) > 1 else float("inf")
            last_p_in[s] = (p_in, j)
            last_vectors[s] = vectors[j]
            if iteration >= scf.min_iterations and de < scf.energy_tol and rn < scf.density_tol:
                if st.float_phase:
                    st.float_phase = False
                    st.refinement_from = iteration + 1
                else:
                    st.converged = True
                    continue
            st.worsened = st.worsened + 1 if rn > st.previous_residual else 0
            st.previous_residual = rn
            if scf.fallback_ladder and st.worsened >= 3 and st.rung + 1 < 4:
                st.rung += 1
                if st.rung == 3:
                    st.level_shift = 0.5  # loop.py:320: the last rung shifts the unoccupied states by 0.5 Ha
                st.mixer = make(0.5 * mixing.alpha) if st.rung == 1 else LinearMixer(0.5 * mixing.alpha)
                st.fallback_events.append(f"iteration {iteration}: stepping down to rung {st.rung}")
                st.worsened = 0
                st.rung_changed = True
                n_next[j] = nin[j] + 0.5 * mixing.alpha * (n_out[j] - nin[j])
                if lin_next is not None:
                    a = 0.5 * mixing.alpha
                    lin_next[0][j] = p_in.v_smooth[j] + a * (p_out.v_smooth[j] - p_in.v_smooth[j])
                    lin_next[1][:, j] = p_in.node[:, j] + a * (p_out.node[:, j] - p_in.node[:, j])
                    lin_next[2][j] = p_in.lifted_h[j] + a * (p_out.lifted_h[j] - p_in.lifted_h[j])
            new_active.append(s)
        # write back the per-system state of this iteration
        if full:
            n_in = n_next
            previous_effective = p_in.effective
            initial_block = vectors
            lin_in = lin_next
        else:
            n_in = n_in.index_copy(0, sel, n_next)
            previous_effective = previous_effective.index_copy(0, sel, p_in.effective)
            initial_block = initial_block.index_copy(0, sel, vectors)
            if lin_next is None or lin_in is None:
                lin_in = None
            else:
                lin_in = (lin_in[0].index_copy(0, sel, lin_next[0]), lin_in[1].index_copy(1, sel, lin_next[1]),
                          lin_in[2].index_copy(0, sel, lin_next[2]))
        if previous_effective is None:
            previous_effective = p_in.effective
        active = new_active
    # final full diagonalisation of every system at its last input potential (fresh Lanczos, float64)
    eff = torch.stack([last_p_in[s][0].effective[last_p_in[s][1]] for s in range(b)])
    init = torch.stack([last_vectors[s] for s in range(b)])
    h = step.hamiltonian(eff)
    h.applications = 0
    streams = [SeededStream(step.seeds[s], dev) for s in range(b)]
    evals, vectors, residuals, estates = batched_chefsi(h, None, step.n_states, step.eigen, init, streams, [None] * b,
                                                        step.eigen.max_iterations, None)
    p_in_final = BatchedPotentials(
        effective=eff,
        v_hartree=torch.stack([last_p_in[s][0].v_hartree[last_p_in[s][1]] for s in range(b)]),
        hartree_energy=torch.stack([last_p_in[s][0].hartree_energy[last_p_in[s][1]] for s in range(b)]),
        xc_energy=torch.stack([last_p_in[s][0].xc_energy[last_p_in[s][1]] for s in range(b)]),
        xc_double_counting=torch.stack([last_p_in[s][0].xc_double_counting[last_p_in[s][1]] for s in range(b)]))
    n_out, rho_out = step.output_density(vectors)
    p_out = step.potentials(n_out)
    terms = step.energy_terms(evals, vectors, rho_out, p_in_final, p_out)
    charge = row_sums(mass[None] * rho_out)
    keys = list(terms)
    host = torch.stack([*terms.values(), charge]).cpu().numpy()
    ev = evals.cpu().numpy()
    _lib.check_device_status("batched final diagonalisation")
    energies = [{k: float(host[i, s]) for i, k in enumerate(keys)} for s in range(b)]
    final_converged = [bool(es.converged) for es in estates]
    apps = sum(st.applications for st in systems) + sum(es.applications for es in estates)
    measurements = {
        "batch": b,
        "applications_per_system": [st.applications + es.applications for st, es in zip(systems, estates)],
        "charge_error": [abs(float(host[-1, s]) - step.n_electrons) for s in range(b)],
        "fp64_refinement_from_iteration": [st.refinement_from for st in systems],
        "filter_precision": "float32" if mixed else "float64",
        "energy_history": [st.energies for st in systems],
        "fallbacks": [st.fallback_events for st in systems],
        "fused_kernels": {"tier": "native-sm100a", "library": _lib.LIBRARY_PATH.name},
        "wall_s": time.perf_counter() - started,
    }
    return BatchedOutcome(energies=energies, eigenvalues=[list(ev[s]) for s in range(b)],
                          scf_iterations=[st.iterations for st in systems],
                          converged=[st.converged and final_converged[s] for s, st in enumerate(systems)],
                          applications=float(apps), density=n_out, measurements=measurements)


# ------------------------------------------------------------------------------------------------
# Systems on their own grids in one launch (e.g. a bond-length scan, whose boxes grow with R)


class EmbeddedStream:
    """A system's seeded draws in its own shape, embedded in the common box (zeros elsewhere)."""

    def __init__(self, stream: SeededStream, embed) -> None:
        self.stream = stream
        self.embed = embed
        self.n = None

    def randn(self, shape):
        size = (shape,) if isinstance(shape, int) else tuple(shape)
        own = self.stream.randn((*size[:-1], self.n))
        return self.embed(own)


class MultiGeometryHamiltonian:
    """``A`` on B systems with their own grids (same spacing and order), blocks ``(B, k, N)``.

    Every system is embedded at the low corner of a common box ``max(shape_s)``: its face weights,
    h^3/omega, bare potential and measure are copied in, and are zero outside it. Zero h^3/omega and
    potential keep every point outside a system at zero through the apply and the filter, zero face
    weights couple nothing across its boundary (its own Dirichlet zeros lie there), and a zero measure
    leaves the Rayleigh--Ritz products those of the system alone. The kernels read the per-system
    geometry through ``cdftb_operator.per_system_geometry`` (one launch for all systems).
    """

    def __init__(self, geometries, dtype=torch.float64, potentials=None) -> None:
        if potentials is None:
            spacings = {round(float(g.grid.spacing), 14) for g in geometries}
            if len(spacings) != 1 or any(g.grid.fd_order != 8 for g in geometries):
                raise ValueError("the systems must share the grid spacing and the order-8 stencil")
            self.geometries = list(geometries)
            self.shapes = [tuple(g.grid.shape) for g in geometries]
            common = tuple(max(s[d] for s in self.shapes) for d in range(3))
            first = geometries[0].grid
            self.grid = UniformGrid(common, first.spacing, (0.0, 0.0, 0.0), device=first.device, fd_order=8)
            b = len(geometries)
            n = self.grid.n_points
            nx, ny, nz = common
            f = dict(dtype=torch.float64, device=first.device)
            self._w = [torch.zeros((b, nx + 8, ny, nz), **f), torch.zeros((b, nx, ny + 8, nz), **f),
                       torch.zeros((b, nx, ny, nz + 8), **f)]
            self._inv64 = torch.zeros((b, n), **f)
            self.potentials = torch.zeros((b, n), **f)
            self.q = torch.zeros((b, n), **f)
            for s, g in enumerate(geometries):
                sx, sy, sz = self.shapes[s]
                faces = g.factor.face_weights(8)
                self._w[0][s, :sx + 8, :sy, :sz] = faces[0]
                self._w[1][s, :sx, :sy + 8, :sz] = faces[1]
                self._w[2][s, :sx, :sy, :sz + 8] = faces[2]
                pot, inv, measure = g.quadrature.bare_operator_terms()
                self.embed_into(self._inv64[s], s, inv)
                self.embed_into(self.potentials[s], s, pot)
                self.embed_into(self.q[s], s, measure.quadrature)
            # each system's own grid: the kernel's tiles wholly beyond it store zeros without work
            self._shapes = torch.tensor(self.shapes, dtype=torch.int32, device=first.device).contiguous()
        else:
            raise ValueError("use subset() to select systems")
        self.dtype = dtype
        self._cast()
        self.applications = 0

    def _cast(self) -> None:
        if self.dtype == torch.float64:
            self._faces = tuple(w.contiguous() for w in self._w)
            self._inv = self._inv64.contiguous()
            self._pot = self.potentials.contiguous()
        else:
            self._faces = tuple(cast(w.contiguous(), self.dtype) for w in self._w)
            self._inv = cast(self._inv64.contiguous(), self.dtype)
            self._pot = cast(self.potentials.contiguous(), self.dtype)

    def as_dtype(self, dtype) -> "MultiGeometryHamiltonian":
        other = MultiGeometryHamiltonian.__new__(MultiGeometryHamiltonian)
        other.__dict__.update(self.__dict__)
        other.dtype = dtype
        other._cast()
        other.applications = 0
        return other

    # -- embedding of fields between a system's grid and the common box
    def embed_into(self, dst: torch.Tensor, s: int, field: torch.Tensor) -> None:
        sx, sy, sz = self.shapes[s]
        dst.reshape(self.grid.shape)[:sx, :sy, :sz] = field.reshape(sx, sy, sz)

    def embed(self, s: int, field: torch.Tensor) -> torch.Tensor:
        """``(..., N_s)`` on system s's grid -> ``(..., N)`` in the common box."""
        lead = field.shape[:-1]
        out = torch.zeros((*lead, self.grid.n_points), dtype=field.dtype, device=field.device)
        sx, sy, sz = self.shapes[s]
        out.reshape(*lead, *self.grid.shape)[..., :sx, :sy, :sz] = field.reshape(*lead, sx, sy, sz)
        return out

    def extract(self, s: int, field: torch.Tensor) -> torch.Tensor:
        """``(..., N)`` in the common box -> ``(..., N_s)`` on system s's grid."""
        lead = field.shape[:-1]
        sx, sy, sz = self.shapes[s]
        return field.reshape(*lead, *self.grid.shape)[..., :sx, :sy, :sz].reshape(*lead, sx * sy * sz).contiguous()

    @property
    def batch(self) -> int:
        return self.potentials.shape[0]

    def _op(self, k: int) -> _lib.Operator:
        op = _lib.Operator()
        op.nx, op.ny, op.nz = self.grid.shape
        op.accuracy = 8
        op.spacing = self.grid.spacing
        op.dtype = F64 if self.dtype == torch.float64 else F32
        op.face_weights = (ctypes.c_void_p * 3)(*(w.data_ptr() for w in self._faces))
        op.inverse_weight = self._inv.data_ptr()
        op.potential = self._pot.data_ptr()
        op.potential_stride = self.grid.n_points
        op.orbitals_per_group = int(k)
        op.quadrature = self.q.data_ptr()
        op.per_system_geometry = 1
        op.system_shapes = self._shapes.data_ptr()
        return op

    apply = BatchedHamiltonian.apply
    filter = BatchedHamiltonian.filter

    def subset(self, index: list[int]) -> "MultiGeometryHamiltonian":
        sub = MultiGeometryHamiltonian.__new__(MultiGeometryHamiltonian)
        sub.__dict__.update(self.__dict__)
        idx = torch.tensor(index, dtype=torch.long, device=self.potentials.device)
        sub._w = [w.index_select(0, idx).contiguous() for w in self._w]
        sub._inv64 = self._inv64.index_select(0, idx).contiguous()
        sub.potentials = self.potentials.index_select(0, idx).contiguous()
        sub.q = self.q.index_select(0, idx).contiguous()
        sub.shapes = [self.shapes[i] for i in index]
        sub._shapes = self._shapes.index_select(0, idx).contiguous()
        sub.geometries = [self.geometries[i] for i in index]
        sub._cast()
        sub.applications = 0
        return sub


def solve_noninteracting_batch(geometries, n_electrons: float, *, seeds=None, eigen: EigenConfig | None = None,
                               filter_precision: torch.dtype = torch.float64) -> list[dict]:
    """``solve_noninteracting`` (``src/cdft/scf/noninteracting.py:118-330``) for B systems at once.

    The systems may have different grids (same spacing): one filter launch, one Rayleigh--Ritz
    step and one Lanczos enclosure per CheFSI iteration serve all of them. Each system draws its
    seeded random block in its own shape, as the single-system solve does. Returns one result dict
    per system (``total``, ``eigenvalues``, ``iterations``, ``converged``, ``stop_reason``).
    """
    from .scf import aufbau_occupations, nuclear_repulsion

    from .carriers import eigen_config
    config = eigen_config(eigen)
    b = len(geometries)
    seeds = list(seeds) if seeds is not None else [0] * b
    h = MultiGeometryHamiltonian(geometries)
    h32 = h.as_dtype(torch.float32) if filter_precision == torch.float32 else None
    n_states = max(1, int(-(-float(n_electrons) // 2.0)))
    dev = h.grid.device
    streams = []
    for s in range(b):
        stream = EmbeddedStream(SeededStream(seeds[s], dev), lambda x, s=s: h.embed(s, x))
        stream.n = geometries[s].grid.n_points
        streams.append(stream)
    evals, vectors, residual, states = batched_chefsi(
        h, h32, n_states, config, None, streams, [None] * b, config.max_iterations,
        BatchedKohnShamStep.FLOAT_FILTER_SWITCH_RESIDUAL if h32 is not None else None, ritz_stop=True)
    occ = aufbau_occupations(n_states, float(n_electrons))[0]
    values = evals.cpu().numpy()
    _lib.check_device_status("batched non-interacting solve")
    out = []
    for s, g in enumerate(geometries):
        band = float((occ * values[s]).sum())
        out.append({"total": band + nuclear_repulsion(g.charges, g.positions), "eigenvalues": values[s].tolist(),
                    "iterations": states[s].iterations, "converged": states[s].converged,
                    "stop_reason": states[s].stop_reason, "orbitals": h.extract(s, vectors[s])})
    return out
