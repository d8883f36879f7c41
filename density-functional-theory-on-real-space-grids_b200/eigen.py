"""Chebyshev-filtered subspace iteration and Rayleigh--Ritz on the device.

Host mirror of ``src/cdft/eigen/chefsi.py`` (chebyshev_filter, chebyshev_coefficients,
SpectralBoundsHint, ChebyshevFilteredSubspace) and ``src/cdft/eigen/rayleigh_ritz.py``
(orthonormalise, rayleigh_ritz, residual_norms). The filter is one library call
(``cdftb_chebyshev_filter``: every step of the recurrence fused into the apply); the Rayleigh--Ritz
step is the Gram reduction, a device Cholesky, the column-wise triangular solve, one apply, the
subspace reduction, a device Jacobi eigensolver and a rotation -- no host round trip inside it.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import F32, F64, call, ptr, stream_handle
from .operators import Measure, measure_cross, rowwise_inner, seeded_randn

BOUND_REUSE_RITZ_FRACTION = 0.9


def chebyshev_coefficients(degree: int, lower: float, upper: float, spectrum_min: float):
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


def chebyshev_filter(hamiltonian, block: torch.Tensor, degree: int, lower: float, upper: float,
                     spectrum_min: float, *, precision: torch.dtype | None = None) -> torch.Tensor:
    """The scaled Chebyshev filter of [F2] (``src/cdft/eigen/chefsi.py:81-113``), one library call.

    ``precision=torch.float32`` runs the recurrence in float (the mixed-precision form): the
    float64 block is read once, every intermediate is float, and the result is written back as
    float64 for the float64 Rayleigh--Ritz step.
    """
    if upper <= lower:
        raise ValueError(f"filter interval is empty: lower={lower}, upper={upper}")
    if not hasattr(hamiltonian, "operator"):
        # an operator that is not one diagonal potential (the level-shifted rung of the fallback
        # ladder): the scaled recurrence over its own apply, as chefsi.py:99-113 runs it
        return _eager_filter(hamiltonian, block, degree, lower, upper, spectrum_min)
    rows = chebyshev_coefficients(degree, lower, upper, spectrum_min)
    # pinned + non-blocking: a pageable copy would synchronise the stream (as chefsi.py:316-321 notes)
    table = torch.tensor(rows, dtype=torch.float64).pin_memory().to(block.device, non_blocking=True)
    return filter_with_table(hamiltonian, block, table, degree, orbitals_per_group=block.numel() // block.shape[-1],
                             precision=precision)


def _eager_filter(hamiltonian, block: torch.Tensor, degree: int, lower: float, upper: float,
                  spectrum_min: float) -> torch.Tensor:
    """The scaled three-term recurrence (``src/cdft/eigen/chefsi.py:99-113``) over ``hamiltonian.apply``."""
    e = 0.5 * (upper - lower)
    c = 0.5 * (upper + lower)
    sigma = e / (spectrum_min - c)
    sigma1 = sigma
    x = block.to(torch.float64)
    y = (hamiltonian.apply(x) - c * x) * (sigma1 / e)
    previous = x
    for _ in range(2, degree + 1):
        sigma2 = 1.0 / (2.0 / sigma1 - sigma)
        y_new = (hamiltonian.apply(y) - c * y) * (2.0 * sigma2 / e) - (sigma * sigma2) * previous
        previous, y = y, y_new
        sigma = sigma2
    return y


def filter_workspace(op, batch: int, device: torch.device) -> torch.Tensor:
    """Device scratch of the fused filter (``cdftb_chebyshev_filter_work_bytes``), as bytes."""
    nbytes = _lib.library().cdftb_chebyshev_filter_work_bytes(ctypes.byref(op), batch)
    return torch.empty(nbytes, dtype=torch.uint8, device=device)


def filter_with_table(hamiltonian, block: torch.Tensor, table: torch.Tensor, degree: int, *, orbitals_per_group: int,
                      potential: torch.Tensor | None = None, precision: torch.dtype | None = None) -> torch.Tensor:
    """Run the fused filter with a device coefficient table ``(groups, degree, 3)``."""
    _lib.require_cuda(block, "block")
    x = block.contiguous()
    n = hamiltonian.grid.n_points
    batch = x.numel() // n
    work_dtype = precision or hamiltonian.dtype
    if work_dtype != hamiltonian.dtype:
        raise ValueError("the filter runs in the Hamiltonian's dtype; build it with dtype=float32 for the mixed form")
    out = torch.empty_like(x)
    op = hamiltonian.operator(potential, orbitals_per_group=orbitals_per_group)
    work = filter_workspace(op, batch, x.device)
    hamiltonian.note_applications(degree)
    call("cdftb_chebyshev_filter", ctypes.byref(op), ptr(x), _lib.dtype_code(x), ptr(out), _lib.dtype_code(out),
         ptr(work), work.numel(), batch, ptr(table.contiguous()), degree, stream_handle(x.device))
    return out


GRAPH_MAX_CAPTURES = 8


class GraphedChebyshevFilter:
    """``GraphedChebyshevFilter`` (``src/cdft/eigen/chefsi.py:185-392``): the fused filter replayed
    from a ``torch.cuda.CUDAGraph``.

    One capture per key (operator geometry and dtype, block shape, potential shape, degree) holds
    the ``degree`` launches of one ``cdftb_chebyshev_filter`` call over static buffers: the block,
    the potential (so a new SCF Hamiltonian on the same geometry replays the same graph), the
    coefficient table, the output and the filter's scratch. Before each replay the block and the
    potential are copied in on the device and the table comes from pinned memory by a non-blocking
    copy, so a call reads nothing back to the host. The library call itself neither allocates nor
    synchronises once the tile autotuner has seen the shape, and a direct call before each capture
    makes sure it has.

    As in the reference, nothing falls back silently: an operator without the graph seam (the
    level-shifted rung), a capture or replay error, a first replay that differs from the direct call
    by even one bit, or more than ``GRAPH_MAX_CAPTURES`` captures make the engine call the filter
    directly, each counted by reason in :meth:`record`. A capture's first replay is checked against
    the direct call, whose result that call returns. A capture made before a timed-out launch was
    reported (``_lib.timeouts_reported``) is captured again, since a graph replays its launches with
    their abort token of the capture.
    """

    def __init__(self, device, reason_disabled: str | None = None) -> None:
        self.device = torch.device(device)
        self.disabled_reason = reason_disabled
        self.captures = 0
        self.replays = 0
        self.eager_calls: dict[str, int] = {}
        self.warmup_applications = 0
        self.validation_max_rel_diff: float | None = None
        self._release()

    def record(self) -> dict:
        used = self.disabled_reason is None and self.replays > 0
        out = {"used": used, "captures": self.captures, "replays": self.replays,
               "eager_calls": dict(self.eager_calls), "warmup_applications": self.warmup_applications,
               "validation_max_rel_diff": self.validation_max_rel_diff}
        if not used:
            out["reason"] = self.disabled_reason or (
                "no filter call was graph-capable" if self.eager_calls else "the filter was never called")
        return out

    def _release(self) -> None:
        self._graph = None
        self._key = None
        self._static = None
        self._template = None
        self._validated = False
        self._generation = _lib.timeouts_reported

    def _disable(self, reason: str) -> None:
        self.disabled_reason = reason
        self._release()

    def _filter_directly(self, hamiltonian, block, degree, lower, upper, spectrum_min) -> torch.Tensor:
        """The filter without a graph (the library call, or the recurrence over ``apply``)."""
        return chebyshev_filter(hamiltonian, block, degree, lower, upper, spectrum_min)

    def _direct(self, reason: str, hamiltonian, block, degree, lower, upper, spectrum_min) -> torch.Tensor:
        self.eager_calls[reason] = self.eager_calls.get(reason, 0) + 1
        return self._filter_directly(hamiltonian, block, degree, lower, upper, spectrum_min)

    def _seam(self, hamiltonian, block: torch.Tensor):
        """``(seam, None)``, where the seam builds the capture's operator (``operator``,
        ``filter_potential``, ``graph_geometry_key``, ``note_applications``, ``dtype``), or
        ``(None, why)`` when this call cannot replay."""
        for name in ("operator", "filter_potential", "graph_geometry_key", "note_applications", "dtype"):
            if not hasattr(hamiltonian, name):
                return None, f"operator {type(hamiltonian).__name__} has no graph seam"
        return hamiltonian, None

    def __call__(self, hamiltonian, block: torch.Tensor, degree: int, lower: float, upper: float,
                 spectrum_min: float) -> torch.Tensor:
        if upper <= lower:
            raise ValueError(f"filter interval is empty: lower={lower}, upper={upper}")
        if self.disabled_reason is not None:
            return self._direct("disabled", hamiltonian, block, degree, lower, upper, spectrum_min)
        if block.device.type != "cuda":
            return self._direct(f"block on {block.device.type}; graphs are CUDA-only", hamiltonian, block, degree,
                                lower, upper, spectrum_min)
        seam, why = self._seam(hamiltonian, block)
        if seam is None:
            return self._direct(why, hamiltonian, block, degree, lower, upper, spectrum_min)
        rows = chebyshev_coefficients(degree, lower, upper, spectrum_min)
        potential = seam.filter_potential()
        key = (seam.graph_geometry_key(), seam.dtype, tuple(block.shape), block.dtype, tuple(potential.shape),
               potential.dtype, int(degree))
        if key != self._key or self._generation != _lib.timeouts_reported:
            if self.captures >= GRAPH_MAX_CAPTURES:
                self._disable(f"more than {GRAPH_MAX_CAPTURES} captures (block shape or geometry keeps changing)")
                return self._direct("disabled", hamiltonian, block, degree, lower, upper, spectrum_min)
            try:
                self._capture(seam, block, potential, rows, key)
            except Exception as exc:  # noqa: BLE001 - any capture failure is recorded, then direct calls
                self._disable(f"capture failed: {type(exc).__name__}: {exc}")
                return self._direct("disabled", hamiltonian, block, degree, lower, upper, spectrum_min)
        s = self._static
        try:
            table = torch.tensor(rows, dtype=torch.float64).pin_memory()
            s["table"].copy_(table, non_blocking=True)
            if potential.data_ptr() != s["potential"].data_ptr():
                s["potential"].copy_(potential)
            s["input"].copy_(block)
            self._graph.replay()
        except Exception as exc:  # noqa: BLE001 - a replay failure is recorded, then direct calls
            self._disable(f"replay failed: {type(exc).__name__}: {exc}")
            return self._direct("disabled", hamiltonian, block, degree, lower, upper, spectrum_min)
        if not self._validated:
            direct = self._filter_directly(hamiltonian, block, degree, lower, upper, spectrum_min)
            diff, scale = torch.stack([(direct - s["output"]).abs().max(), direct.abs().max()]).tolist()
            relative = diff / scale if scale > 0.0 else diff
            self.validation_max_rel_diff = max(relative, self.validation_max_rel_diff or 0.0)
            self.eager_calls["validation of a new capture"] = self.eager_calls.get("validation of a new capture", 0) + 1
            if diff != 0.0:
                self._disable(f"replay differs from the direct call by {relative:.3e} (relative)")
            else:
                self._validated = True
            return direct
        self.replays += 1
        seam.note_applications(degree)
        return s["output"].clone()

    def _capture(self, hamiltonian, block: torch.Tensor, potential: torch.Tensor, rows, key) -> None:
        self._release()
        device = block.device
        x = block.contiguous()
        batch = x.numel() // x.shape[-1]
        static = {"input": x.clone(), "potential": potential.detach().clone(),
                  "table": torch.tensor(rows, dtype=torch.float64, device=device), "output": torch.empty_like(x)}
        op = hamiltonian.operator(static["potential"], orbitals_per_group=batch)
        static["work"] = filter_workspace(op, batch, device)
        static["op"] = op
        degree = len(rows)

        def launch():
            call("cdftb_chebyshev_filter", ctypes.byref(op), ptr(static["input"]), _lib.dtype_code(static["input"]),
                 ptr(static["output"]), _lib.dtype_code(static["output"]), ptr(static["work"]),
                 static["work"].numel(), batch, ptr(static["table"]), degree, stream_handle(device))

        # a direct call first: the tile autotuner (which synchronises) sees the shape outside the capture
        launch()
        self.warmup_applications += degree
        torch.cuda.current_stream(device).synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            launch()
        self._graph = graph
        self._template = hamiltonian  # keeps every geometry tensor the graph reads alive
        self._static = static
        self._key = key
        self._validated = False
        self.captures += 1


class RitzWorkspace:
    """Device buffers of one Rayleigh--Ritz step, reused across calls of the same shape."""

    def __init__(self):
        self._key = None

    def get(self, m: int, groups: int, device):
        key = (m, groups, str(device))
        if key != self._key:
            f = dict(dtype=torch.float64, device=device)
            self.lower = torch.empty((groups, m, m), **f)
            self.info = torch.empty(groups, dtype=torch.int32, device=device)
            self.evals = torch.empty((groups, m), **f)
            self.rot = torch.empty((groups, m, m), **f)
            self._key = key
        return self


_WS = RitzWorkspace()


def orthonormalise(block: torch.Tensor, measure: Measure, groups: int = 1) -> torch.Tensor:
    """Cholesky orthonormalisation in the measure (``src/cdft/eigen/rayleigh_ritz.py:51-72``).

    On a Cholesky failure the reference falls back to an eigendecomposition that drops rank; that
    rare branch reads the Gram matrix to the host and builds the reduced basis there.
    """
    n = measure.grid.n_points
    flat = block.to(torch.float64).reshape(groups, -1, n).contiguous()
    m = flat.shape[1]
    gram = measure_cross(flat, flat, measure.quadrature, groups)
    ws = _WS.get(m, groups, block.device)
    stream = stream_handle(block.device)
    call("cdftb_small_cholesky_f64", ptr(gram), ptr(ws.lower), ptr(ws.info), m, groups, stream)
    basis = torch.empty_like(flat)
    call("cdftb_block_trsm_lower_f64", ptr(ws.lower), ptr(flat), flat.stride(0), ptr(basis), F64, basis.stride(0), m, n,
         groups, stream)
    ws.last_info = ws.info
    return basis, gram


def _rank_revealing_basis(flat: torch.Tensor, gram: torch.Tensor) -> torch.Tensor:
    """The eigh fallback of rayleigh_ritz.py:64-70 for one group (host-side small matrix)."""
    g = gram.cpu().numpy()
    evals, evecs = np.linalg.eigh(0.5 * (g + g.T))
    keep = evals > evals[-1] * 1e-14
    if not keep.any():
        raise ValueError("the orbital block collapsed to rank zero")
    scaled = evecs[:, keep] / np.sqrt(evals[keep])
    r = torch.from_numpy(np.ascontiguousarray(scaled.T)).to(flat.device)
    out = torch.empty((1, r.shape[0], flat.shape[-1]), dtype=torch.float64, device=flat.device)
    call("cdftb_block_rotate_f64", ptr(r), ptr(flat.contiguous()), 0, ptr(out), F64, 0, r.shape[0], r.shape[1],
         flat.shape[-1], 1, stream_handle(flat.device))
    return out[0]


def rayleigh_ritz(hamiltonian, block: torch.Tensor, measure: Measure, *, host: bool = True,
                  check_cholesky: bool = True):
    """Diagonalise within span(block) (``src/cdft/eigen/rayleigh_ritz.py:75-102``).

    Returns ``(eigenvalues, eigenvectors, orthonormality_error)``; with ``host=False`` the error is
    a 0-d device tensor. Also leaves ``applied = A @ eigenvectors`` on the result for the residual
    (it equals ``U^T (A Q)`` with ``U`` orthogonal), so :func:`residual_norms` needs no extra apply.
    """
    n = measure.grid.n_points
    flat = block.to(torch.float64).reshape(-1, n)
    basis, gram = orthonormalise(flat, measure)
    ws = _WS.get(flat.shape[0], 1, block.device)
    info = ws.info.clone()
    if check_cholesky:
        # The Cholesky status is read with the caller's per-iteration scalars (no extra sync) when
        # check_cholesky is False; a failure then repeats this step through the eigh fallback.
        if int(info[0].item()) != 0:
            basis = _rank_revealing_basis(flat, gram[0]).reshape(1, -1, n)
    m = basis.shape[1]
    stream = stream_handle(block.device)
    applied = hamiltonian.apply(basis[0]).reshape(1, m, n)
    sub = measure_cross(basis, applied, measure.quadrature)
    ws = _WS.get(m, 1, block.device)
    call("cdftb_small_eigh_f64", ptr(sub), ptr(ws.evals), ptr(ws.rot), m, 1, stream)
    vectors = torch.empty((1, m, n), dtype=torch.float64, device=block.device)
    call("cdftb_block_rotate_f64", ptr(ws.rot), ptr(basis), basis.stride(0), ptr(vectors), F64, vectors.stride(0), m, m,
         n, 1, stream)
    rotated_applied = torch.empty_like(vectors)
    call("cdftb_block_rotate_f64", ptr(ws.rot), ptr(applied), applied.stride(0), ptr(rotated_applied), F64,
         rotated_applied.stride(0), m, m, n, 1, stream)
    g2 = measure_cross(vectors, vectors, measure.quadrature)[0]
    error = (g2 - torch.eye(m, dtype=torch.float64, device=block.device)).abs().max()
    evals = ws.evals[0].clone()
    vec = vectors[0]
    _APPLIED[id(vec)] = (vec, rotated_applied[0])
    if not check_cholesky:
        rayleigh_ritz.last_info = info
    return evals, vec, (float(error) if host else error)


_APPLIED: dict[int, tuple] = {}


def residual_norms(hamiltonian, eigenvalues: torch.Tensor, vectors: torch.Tensor, measure: Measure) -> torch.Tensor:
    """``||H psi_i - eps_i psi_i||`` in the measure (``src/cdft/eigen/rayleigh_ritz.py:105-115``).

    When ``vectors`` came from :func:`rayleigh_ritz`, ``H psi`` is the rotated ``A Q`` it already
    formed (one apply fewer); otherwise the operator is applied.
    """
    n = measure.grid.n_points
    cached = _APPLIED.pop(id(vectors), None)
    if cached is not None and cached[0] is vectors:
        applied = cached[1]
    else:
        applied = hamiltonian.apply(vectors)
    m = vectors.shape[0]
    res = torch.empty((m, n), dtype=torch.float64, device=vectors.device)
    call("cdftb_block_residual_f64", ptr(applied.contiguous()), ptr(vectors.contiguous()),
         ptr(eigenvalues.contiguous()), ptr(res), m, n, 1, m * n, stream_handle(vectors.device))
    return rowwise_inner(res, res, measure.quadrature).clamp_min(0.0).sqrt()


@dataclass(frozen=True)
class SpectralBoundsHint:
    """Bounds carried over from the previous SCF iteration (``src/cdft/eigen/chefsi.py:169-182``)."""

    lower: float
    upper: float
    shift: torch.Tensor | float = 0.0


@dataclass
class EigenConfig:
    """The eigensolver settings of ``contract.EigenConfig`` (contract.py:431-449) the path reads."""

    n_extra_states: int = 4
    extra_states_fraction: float = 0.20
    chebyshev_degree: int = 20
    lanczos_steps: int = 12
    bound_safety: float = 1.02
    max_iterations: int = 300
    residual_tol: float = 1.0e-8
    cross_check: bool = False
    cross_check_tol: float = 1.0e-8


@dataclass
class EigenResult:
    eigenvalues: torch.Tensor
    eigenvectors: torch.Tensor
    residuals: torch.Tensor
    n_iterations: int
    converged: bool


def _interval_fraction(value: float, low: float, high: float) -> float:
    width = high - low
    return (value - low) / width if width > 0.0 else float("inf")


class ChebyshevFilteredSubspace:
    """CheFSI (``src/cdft/eigen/chefsi.py:408-585``) with the native filter and Rayleigh--Ritz.

    ``filter_precision=torch.float32`` filters in float (the Hamiltonian passed in must then be
    built with ``dtype=torch.float32`` for the filter via ``filter_hamiltonian``); every
    Rayleigh--Ritz, residual and Lanczos step stays float64.
    """

    def __init__(self, grid, config: EigenConfig, ritz_stop: bool = True, filter_hamiltonian=None,
                 switch_residual: float | None = None, filter_engine=None) -> None:
        self.grid = grid
        self.config = config
        #: A ``GraphedChebyshevFilter`` to run the filter through (None: direct library calls).
        self.filter_engine = filter_engine
        self.ritz_stop = ritz_stop
        self.filter_hamiltonian = filter_hamiltonian
        #: With a float filter: once the worst wanted residual falls below this, filter in float64
        #: (a float-filtered subspace stalls near residual 1e-5, above a 1e-8 target).
        self.switch_residual = switch_residual
        self.float_filter_iterations = 0
        self.history: list[dict] = []
        self.spectral_bounds = None
        self.bounds_source = "unset"
        self.bounds_shift = 0.0
        self.top_ritz_fraction = float("nan")

    def solve(self, hamiltonian, n_states: int, initial: torch.Tensor | None = None,
              generator: torch.Generator | None = None, bounds: SpectralBoundsHint | None = None) -> EigenResult:
        grid = self.grid
        cfg = self.config
        measure = hamiltonian.measure
        extra = max(cfg.n_extra_states, int(cfg.extra_states_fraction * n_states))
        size = min(n_states + extra, grid.n_points)
        if initial is None:
            block = seeded_randn((size, grid.n_points), generator, device=grid.device)
        else:
            block = initial.to(torch.float64).reshape(-1, grid.n_points)
            if block.shape[0] < size:
                pad = seeded_randn((size - block.shape[0], grid.n_points), generator, device=grid.device)
                block = torch.cat([block, pad], dim=0)

        def lanczos():
            return hamiltonian.spectral_bounds(steps=cfg.lanczos_steps, safety=cfg.bound_safety, generator=generator)

        if bounds is None:
            spectrum_min, spectrum_max = lanczos()
            self.bounds_source = "lanczos"
            self.bounds_shift = 0.0
        evals, vectors, orth = rayleigh_ritz(hamiltonian, block, measure, host=False)
        converged = False
        iteration = 0
        residual = residual_norms(hamiltonian, evals, vectors, measure)
        previous = evals.clone()
        stable = 0
        self.eigenvalue_drift = float("inf")
        self.stop_reason = "iteration limit"
        weak_form = self.ritz_stop and bool(getattr(hamiltonian, "uses_divergence_form", False))
        eigenvalue_tol = 0.1 * cfg.cross_check_tol
        top = min(size, evals.shape[0]) - 1
        if bounds is None:
            next_lower = float(evals[top])
        else:
            shift = bounds.shift if isinstance(bounds.shift, float) else bounds.shift
            vals = torch.stack([evals[top], torch.as_tensor(shift, dtype=torch.float64, device=evals.device)]).tolist()
            next_lower, shift = vals
            spectrum_min, spectrum_max = bounds.lower - shift, bounds.upper + shift
            self.bounds_source = "reused"
            self.bounds_shift = shift
        top_fraction = float("-inf")
        filt = self.filter_hamiltonian or hamiltonian
        for iteration in range(1, cfg.max_iterations + 1):
            lower = next_lower
            fraction = _interval_fraction(lower, spectrum_min, spectrum_max)
            if self.bounds_source == "reused" and not fraction < BOUND_REUSE_RITZ_FRACTION:
                spectrum_min, spectrum_max = lanczos()
                self.bounds_source = (f"lanczos (reuse rejected: top Ritz fraction {fraction:.3f} >= "
                                      f"{BOUND_REUSE_RITZ_FRACTION:g} at iteration {iteration})")
                fraction = _interval_fraction(lower, spectrum_min, spectrum_max)
            top_fraction = max(top_fraction, fraction)
            lower = min(max(lower, spectrum_min + 1e-8), spectrum_max - 1e-8)
            filtered = (self.filter_engine or chebyshev_filter)(filt, vectors, cfg.chebyshev_degree, lower,
                                                                 spectrum_max, spectrum_min)
            if filt is not hamiltonian:
                hamiltonian.note_applications(cfg.chebyshev_degree)
                self.float_filter_iterations += 1
            evals, vectors, orth_error = rayleigh_ritz(hamiltonian, filtered, measure, host=False, check_cholesky=False)
            info = rayleigh_ritz.last_info
            residual = residual_norms(hamiltonian, evals, vectors, measure)
            top = min(size, evals.shape[0]) - 1
            worst, drift, orth, next_lower, chol = torch.stack([
                residual[:n_states].max(), (evals[:n_states] - previous[:n_states]).abs().max(), orth_error,
                evals[top], info[0].to(torch.float64)]).tolist()
            _lib.check_device_status(f"CheFSI iteration {iteration}")
            if chol != 0.0:
                # rank-deficient filtered block: redo this step with the eigh fallback (rayleigh_ritz.py:64-70)
                evals, vectors, orth_error = rayleigh_ritz(hamiltonian, filtered, measure, host=False)
                residual = residual_norms(hamiltonian, evals, vectors, measure)
                top = min(size, evals.shape[0]) - 1
                worst, drift, orth, next_lower = torch.stack([
                    residual[:n_states].max(), (evals[:n_states] - previous[:n_states]).abs().max(), orth_error,
                    evals[top]]).tolist()
            previous = evals.clone()
            self.eigenvalue_drift = drift
            if filt is not hamiltonian and self.switch_residual is not None and worst < self.switch_residual:
                filt = hamiltonian
            self.history.append({"iteration": float(iteration), "residual": worst, "orthonormality": orth,
                                 "eigenvalue_drift": drift})
            if worst < cfg.residual_tol:
                converged = True
                self.stop_reason = "residual below residual_tol"
                break
            stable = stable + 1 if (weak_form and drift < eigenvalue_tol) else 0
            if stable >= 2:
                converged = True
                self.stop_reason = ("Ritz values stable on the weak-form path; the collocation residual is "
                                    f"{worst:.3e}, above residual_tol {cfg.residual_tol:.1e}")
                break
        self.spectral_bounds = (spectrum_min, spectrum_max)
        self.top_ritz_fraction = top_fraction
        _lib.check_device_status("ChebyshevFilteredSubspace.solve")
        return EigenResult(evals[:n_states], vectors[:n_states], residual[:n_states], iteration, converged)


# ---------------------------------------------------------------------------------------------
# LOBPCG: the eigensolver cross-check on the native apply


def _combine(matrix: np.ndarray, block: torch.Tensor) -> torch.Tensor:
    """``matrix @ block`` for a small host matrix ``(a, b)`` and a device block ``(b, N)``, one
    ``cdftb_block_rotate_f64`` launch."""
    mat = np.ascontiguousarray(np.asarray(matrix, dtype=np.float64))
    a, b = mat.shape
    x = block.to(torch.float64).contiguous()
    n = x.shape[-1]
    out = torch.empty((a, n), dtype=torch.float64, device=x.device)
    if a == 0:
        return out
    r = torch.from_numpy(mat).to(x.device, non_blocking=True)
    call("cdftb_block_rotate_f64", ptr(r), ptr(x), 0, ptr(out), F64, 0, a, b, n, 1, stream_handle(x.device))
    return out


def _symmetrise(m: np.ndarray) -> np.ndarray:
    return 0.5 * (m + m.T)


def _stable_basis(block: torch.Tensor, measure: Measure, threshold: float = 1e-12):
    """An orthonormal basis of ``block`` with near-dependent directions dropped, and how many were
    dropped (``src/cdft/eigen/lobpcg.py:253-271``)."""
    if block.shape[0] == 0:
        return block, 0
    g = measure.gram(block).cpu().numpy()
    evals, evecs = np.linalg.eigh(_symmetrise(g))
    keep = evals > evals[-1] * threshold
    if evals[-1] <= 0.0:
        return block[:0], block.shape[0]
    scaled = evecs[:, keep] / np.sqrt(evals[keep])
    return _combine(scaled.T, block), int((~keep).sum())


def _lobpcg_orthonormalise(block: torch.Tensor, measure: Measure) -> torch.Tensor:
    """Cholesky in the measure, the stable basis on failure (``lobpcg.py:221-229``): ``L^-1 block``
    by the native forward substitution."""
    g = measure.gram(block).cpu().numpy()
    try:
        chol = np.linalg.cholesky(g)
    except np.linalg.LinAlgError:
        return _stable_basis(block, measure)[0]
    x = block.to(torch.float64).contiguous()
    m, n = x.shape
    lower = torch.from_numpy(np.ascontiguousarray(chol)).to(x.device)
    out = torch.empty_like(x)
    call("cdftb_block_trsm_lower_f64", ptr(lower), ptr(x), m * n, ptr(out), F64, m * n, m, n, 1,
         stream_handle(x.device))
    return out


def _orthogonalise_against(block: torch.Tensor, basis: torch.Tensor, measure: Measure) -> torch.Tensor:
    """Project ``basis`` out of ``block`` twice, then orthonormalise the rest (``lobpcg.py:232-242``)."""
    for _ in range(2):
        block = block - _combine(measure.cross(block, basis).cpu().numpy(), basis)
    return _stable_basis(block, measure)[0]


class LOBPCG:
    """Locally optimal block preconditioned conjugate gradient (``src/cdft/eigen/lobpcg.py:44-207``),
    the reference's permanent cross-check of the Chebyshev eigensolver (gate G2.5), on the native
    apply and measure products.

    The residual is preconditioned in the similarity frame by default: mapped to the wavefunction
    frame (``r_psi = f r_phi``), filtered with the Teter--Payne--Allan kinetic preconditioner by a
    periodic transform of the box (``cdftb_reciprocal_filter_f64``, kind 1), and mapped back. The
    small projected problems (at most three blocks of states) are solved on the host, one read per
    iteration, as in the reference.
    """

    FRAMES = ("similarity", "transformed", "none")

    def __init__(self, grid, config: EigenConfig, precondition: bool | str = True) -> None:
        if precondition is True:
            precondition = "similarity"
        elif precondition is False:
            precondition = "none"
        if precondition not in self.FRAMES:
            raise ValueError(f"unknown preconditioner frame {precondition!r}; one of {self.FRAMES}")
        self.grid = grid
        self.config = config
        self.frame = precondition
        self.history: list[dict] = []
        self.eigenvalue_tol = 0.1 * config.cross_check_tol
        self.eigenvalue_drift = float("inf")
        self._reference_energy = None

    def _kinetic_reference(self) -> float:
        """The grid's mean kinetic scale: the mean of G^2/2 over the half-spectrum box."""
        if self._reference_energy is None:
            import math

            h = self.grid.spacing
            nx, ny, nz = self.grid.shape
            kx = 2.0 * math.pi * np.fft.fftfreq(nx, d=h)
            ky = 2.0 * math.pi * np.fft.fftfreq(ny, d=h)
            kz = 2.0 * math.pi * np.fft.rfftfreq(nz, d=h)
            g2 = 0.5 * (kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2)
            self._reference_energy = max(float(g2.mean()), 1.0e-6)
        return self._reference_energy

    def _precondition(self, block: torch.Tensor) -> torch.Tensor:
        x = block.to(torch.float64).contiguous()
        rows = x.shape[0]
        nbytes = _lib.library().cdftb_kerker_work_bytes(*self.grid.shape, rows)
        work = torch.empty(nbytes, dtype=torch.uint8, device=x.device)
        out = torch.empty_like(x)
        call("cdftb_reciprocal_filter_f64", ptr(x), rows, *self.grid.shape, self.grid.spacing, 1,
             self._kinetic_reference(), ptr(out), ptr(work), nbytes, stream_handle(x.device))
        return out

    def solve(self, hamiltonian, n_states: int, initial: torch.Tensor | None = None, generator=None) -> EigenResult:
        grid = self.grid
        cfg = self.config
        measure = hamiltonian.measure
        factor = getattr(hamiltonian, "factor", None)
        f = None
        if factor is not None and not getattr(factor, "is_identity", True):
            f = torch.exp(-factor.u).clamp_min(1.0e-150)
        if initial is None:
            x = seeded_randn((n_states, grid.n_points), generator, device=grid.device)
        else:
            x = initial.to(torch.float64).reshape(-1, grid.n_points)[:n_states].clone()
        x = _lobpcg_orthonormalise(x, measure)
        hx = hamiltonian.apply(x)
        evals_h, rotation = np.linalg.eigh(_symmetrise(measure.cross(x, hx).cpu().numpy()))
        x = _combine(rotation.T, x)
        hx = _combine(rotation.T, hx)
        evals = torch.from_numpy(evals_h).to(grid.device)
        p = None
        converged = False
        iteration = 0
        residual = None
        previous = evals_h.copy()
        stable = 0
        self.eigenvalue_drift = float("inf")
        for iteration in range(1, cfg.max_iterations + 1):
            r = hx - evals[:, None] * x
            residual = measure.norm(r)
            res_h = residual.cpu().numpy()
            _lib.check_device_status(f"LOBPCG iteration {iteration}")
            keep = res_h > 0.1 * cfg.residual_tol
            worst = float(res_h.max())
            drift = float(np.abs(evals_h - previous).max()) if iteration > 1 else float("inf")
            previous = evals_h.copy()
            self.eigenvalue_drift = drift
            self.history.append({"iteration": float(iteration), "residual": worst, "eigenvalue_drift": drift})
            if worst < cfg.residual_tol:
                converged = True
                break
            stable = stable + 1 if drift < self.eigenvalue_tol else 0
            if stable >= 2:
                converged = True
                break
            w = r[torch.from_numpy(keep).to(r.device)] if keep.any() else r
            if self.frame == "similarity" and f is not None:
                w = self._precondition(w * f) / f
            elif self.frame != "none":
                w = self._precondition(w)
            w = _orthogonalise_against(w, x, measure)
            if w.shape[0] == 0:
                converged = True
                break
            blocks = [x, w] if p is None else [x, w, p]
            basis, dropped = _stable_basis(torch.cat(blocks, dim=0), measure)
            h_basis = hamiltonian.apply(basis)
            sub_evals, sub_vectors = np.linalg.eigh(_symmetrise(measure.cross(basis, h_basis).cpu().numpy()))
            coeff = sub_vectors[:, :n_states]
            x_new = _combine(coeff.T, basis)
            hx_new = _combine(coeff.T, h_basis)
            p = x_new - _combine(measure.cross(x_new, x).cpu().numpy(), x)
            x, hx = x_new, hx_new
            evals_h = sub_evals[:n_states]
            evals = torch.from_numpy(np.ascontiguousarray(evals_h)).to(grid.device)
            if dropped:
                self.history[-1]["dropped_directions"] = float(dropped)
        return EigenResult(evals[:n_states], x[:n_states], residual[:n_states], iteration, converged)
