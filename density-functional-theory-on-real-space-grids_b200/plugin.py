"""The drop-in: the native kernels bound behind the reference solver's own seams.

    import cdft_b200.plugin as native
    native.install()        # CDFT_NATIVE=auto (default) | on | off
    ...                     # cdft.scf.solve.solve_scenario(..., device=cuda) as before
    native.uninstall()

``install()`` rebinds, in the already importable reference package ``cdft``, exactly the seams its
CUDA path dispatches through, and nothing else:

- ``cdft.operators.fused.device_weighted_divergence`` -- the CUDA branch of ``weighted_divergence``
  (``src/cdft/operators/divergence.py:165-168``): the native staggered stencil, orders 2--8;
- ``CuspFactoredHamiltonian.kinetic_apply`` / ``apply_with_potential``
  (``src/cdft/operators/hamiltonian.py:265-318``): ``0.5 (h^3/omega) div phi (+ V phi)`` in one launch;
- ``cdft.eigen.chefsi.chebyshev_filter`` (``chefsi.py:81``, looked up as a module global by
  ``ChebyshevFilteredSubspace.solve`` and the graph engine): the fused filter, one launch per step;
- ``graphed_filter_for`` in ``cdft.eigen.chefsi`` and, imported there by name, in ``cdft.scf.loop``
  (``loop.py:34``) and ``cdft.scf.noninteracting`` (``noninteracting.py:30``): an engine with the
  graph engine's call and ``record()`` keys that replays the fused filter from a CUDA graph;
- ``CoulombCutoffPoisson.solve`` (``src/cdft/operators/poisson.py:66``, a class method because the
  class is imported by name in ``step.py:53`` and ``loop.py:43``): the native pruned-FFT plan;
- ``SemiLocalFunctional.evaluate`` (``src/cdft/xc/base.py:115``, the base of every functional the
  dispatch table builds): the native functionals, spin-restricted or spin-polarised.

Conventions kept (the reference's, for a replacement on its seams): every replacement returns a
fresh tensor and never writes its inputs; CPU tensors always take the reference's own code, so the
CPU audit path is bit-for-bit unchanged; argument errors are the reference's (``ValueError`` for a
non-1-D Poisson density or a GGA without sigma). A CUDA call the native path does not cover (an
identity cusp factor, a masked domain, a meta-GGA, float32 blocks) runs the reference's code with
the reason counted in :func:`record` under ``auto``, and raises ``RuntimeError`` under ``on``.
Unknown values of ``CDFT_NATIVE`` raise ``ValueError``, as the reference's own switches do
(``src/cdft/precision.py:116-129``).
"""

from __future__ import annotations

import collections
import ctypes
import importlib
import os
from typing import NamedTuple

import torch

from . import _lib
from ._lib import call, ptr, stream_handle
from .eigen import GraphedChebyshevFilter

ENV_NATIVE = "CDFT_NATIVE"
MODES = ("auto", "on", "off")
TIER = "native-sm100a"


def requested_mode(value: str | None = None) -> str:
    """``CDFT_NATIVE`` (or ``value``): ``auto`` (default), ``on`` or ``off``; anything else raises."""
    raw = os.environ.get(ENV_NATIVE, "") if value is None else value
    key = raw.strip().lower() or "auto"
    if key not in MODES:
        raise ValueError(f"{ENV_NATIVE}={raw!r} is not one of {', '.join(MODES)}")
    return key


class _State:
    def __init__(self) -> None:
        self.mode = "off"
        self.saved: dict[tuple[str, str], object] = {}
        self.native_calls: collections.Counter = collections.Counter()
        self.reference_calls: collections.Counter = collections.Counter()
        self.reason: str | None = None


_STATE = _State()


def record() -> dict:
    """What is bound and what ran: for a run's ``measurements`` (the reference's G5.5 convention)."""
    return {
        "tier": TIER if _STATE.saved else "reference",
        "mode": _STATE.mode,
        "seams": sorted(f"{m}.{a}" for m, a in _STATE.saved),
        "native_calls": dict(_STATE.native_calls),
        "reference_calls": dict(_STATE.reference_calls),
        "reason": _STATE.reason,
        "library": str(_lib.LIBRARY_PATH),
    }


def installed() -> bool:
    return bool(_STATE.saved)


def _fallback(seam: str, why: str, original, *args, **kwargs):
    """Run the reference's own code for a CUDA call the native path does not cover."""
    if _STATE.mode == "on":
        raise RuntimeError(f"{ENV_NATIVE}=on: {seam} cannot run natively: {why}")
    _STATE.reference_calls[f"{seam}: {why}"] += 1
    return original(*args, **kwargs)


def _original(module: str, attr: str):
    return _STATE.saved[(module, attr)]


# ---------------------------------------------------------------------------------------------
# (a1) the staggered stencil


def native_weighted_divergence(box, face_weights, spacing, accuracy, shape):
    """The native ``weighted_divergence`` on a CUDA float64 box, or ``None`` with the reason."""
    if box.dtype != torch.float64 or any(w.dtype != torch.float64 for w in face_weights):
        return None, "not float64"
    if int(accuracy) not in (2, 4, 6, 8):
        return None, f"stencil order {accuracy}"
    from .operators import weighted_divergence

    return weighted_divergence(box, face_weights, spacing, int(accuracy), shape), None


def device_weighted_divergence(box, face_weights, spacing, accuracy, shape):
    """``cdft.operators.fused.device_weighted_divergence`` (``src/cdft/operators/fused.py:353``)."""
    out, why = native_weighted_divergence(box, face_weights, spacing, accuracy, shape)
    if out is None:
        return _fallback("device_weighted_divergence", why, _original("cdft.operators.fused",
                                                                       "device_weighted_divergence"),
                         box, face_weights, spacing, accuracy, shape)
    _STATE.native_calls["device_weighted_divergence"] += 1
    return out


# ---------------------------------------------------------------------------------------------
# (a2, b1) the cusp-factorised apply and the fused filter on the reference's operator


def _operator_of(ham, potential: torch.Tensor):
    """A ``cdftb_operator`` for the reference's ``CuspFactoredHamiltonian`` (its grid, cached face
    weights, ``h^3/omega`` and a potential), or ``(None, reason)``."""
    grid, factor = ham.grid, ham.factor
    if getattr(factor, "is_identity", False):
        return None, "identity cusp factor (no nuclei)"
    if not getattr(grid, "_full_box", True):
        return None, "masked domain"
    inv = getattr(ham, "_inverse_weight", None)
    if inv is None or inv.device.type != "cuda" or inv.dtype != torch.float64:
        return None, "no float64 device inverse weight"
    faces = factor.face_weights(grid.fd_order)
    if any(f.device.type != "cuda" or f.dtype != torch.float64 for f in faces):
        return None, "face weights not float64 on the device"
    faces = tuple(f.contiguous() for f in faces)
    inv = inv.contiguous()
    pot = potential.to(torch.float64).contiguous()
    op = _lib.Operator()
    op.nx, op.ny, op.nz = (int(n) for n in grid.shape)
    op.accuracy = int(grid.fd_order)
    op.spacing = float(grid.spacing)
    op.dtype = _lib.F64
    op.face_weights = (ctypes.c_void_p * 3)(*(f.data_ptr() for f in faces))
    op.inverse_weight = inv.data_ptr()
    op.potential = pot.data_ptr()
    op.potential_stride = 0 if pot.dim() == 1 else pot.shape[-1]
    op.orbitals_per_group = 1
    op.quadrature = inv.data_ptr()  # read by no kernel of these calls
    op._keep = (faces, inv, pot)
    return op, None


def native_apply(ham, phi: torch.Tensor, potential: torch.Tensor | None):
    """``A phi`` (or its kinetic part when ``potential`` is None) on the reference's operator."""
    if phi.dtype != torch.float64:
        return None, "not float64"
    n = 1
    for s in ham.grid.shape:
        n *= int(s)
    if phi.shape[-1] != n:
        return None, "orbitals do not match the grid"
    pot = potential if potential is not None else ham._inverse_weight
    if pot.dim() != 1 or pot.shape[0] != n:
        return None, "potential is not one (n_points,) field"
    op, why = _operator_of(ham, pot)
    if op is None:
        return None, why
    from .operators import apply_workspace

    x = phi.contiguous()
    batch = x.numel() // n
    out = torch.empty_like(x)
    work = apply_workspace(op, batch, x.device)
    call("cdftb_cusp_apply", ctypes.byref(op), ptr(x), _lib.F64, ptr(out), _lib.F64, batch,
         1 if potential is None else 0, ptr(work), work.numel(), stream_handle(x.device))
    return out, None


def kinetic_apply(self, phi):
    """``CuspFactoredHamiltonian.kinetic_apply`` (``src/cdft/operators/hamiltonian.py:303-318``)."""
    original = _original("cdft.operators.hamiltonian", "CuspFactoredHamiltonian.kinetic_apply")
    if phi.device.type != "cuda":
        return original(self, phi)
    out, why = native_apply(self, phi, None)
    if out is None:
        return _fallback("kinetic_apply", why, original, self, phi)
    _STATE.native_calls["kinetic_apply"] += 1
    return out


def apply_with_potential(self, phi, potential):
    """``CuspFactoredHamiltonian.apply_with_potential`` (``hamiltonian.py:265-276``), not counted."""
    original = _original("cdft.operators.hamiltonian", "CuspFactoredHamiltonian.apply_with_potential")
    if phi.device.type != "cuda":
        return original(self, phi, potential)
    out, why = native_apply(self, phi, potential)
    if out is None:
        return _fallback("apply_with_potential", why, original, self, phi, potential)
    _STATE.native_calls["apply_with_potential"] += 1
    return out


def native_filter(ham, block: torch.Tensor, degree: int, lower: float, upper: float, spectrum_min: float):
    """The fused Chebyshev filter on the reference's operator at its current potential."""
    from .eigen import chebyshev_coefficients, filter_workspace

    if not all(hasattr(ham, a) for a in ("grid", "factor", "_inverse_weight", "graph_potential")):
        return None, f"operator {type(ham).__name__} is not a cusp-factorised Hamiltonian"
    if block.dtype != torch.float64:
        return None, "not float64"
    potential = ham.graph_potential()
    if potential.dim() != 1:
        return None, "potential is not one (n_points,) field"
    op, why = _operator_of(ham, potential)
    if op is None:
        return None, why
    rows = chebyshev_coefficients(int(degree), float(lower), float(upper), float(spectrum_min))
    table = torch.tensor(rows, dtype=torch.float64).pin_memory().to(block.device, non_blocking=True)
    x = block.contiguous()
    n = x.shape[-1]
    batch = x.numel() // n
    op.orbitals_per_group = batch
    out = torch.empty_like(x)
    work = filter_workspace(op, batch, x.device)
    call("cdftb_chebyshev_filter", ctypes.byref(op), ptr(x), _lib.F64, ptr(out), _lib.F64, ptr(work), work.numel(),
         batch, ptr(table), int(degree), stream_handle(x.device))
    ham.note_applications(int(degree))
    return out, None


def chebyshev_filter(hamiltonian, block, degree, lower, upper, spectrum_min):
    """``cdft.eigen.chefsi.chebyshev_filter`` (``src/cdft/eigen/chefsi.py:81-113``)."""
    original = _original("cdft.eigen.chefsi", "chebyshev_filter")
    if upper <= lower:
        raise ValueError(f"filter interval is empty: lower={lower}, upper={upper}")
    if block.device.type != "cuda":
        return original(hamiltonian, block, degree, lower=lower, upper=upper, spectrum_min=spectrum_min)
    out, why = native_filter(hamiltonian, block, degree, lower, upper, spectrum_min)
    if out is None:
        # a wrapped operator (the level-shifted rung): the reference's recurrence over its apply,
        # whose inner operator is itself native
        _STATE.reference_calls[f"chebyshev_filter: {why}"] += 1
        return original(hamiltonian, block, degree, lower=lower, upper=upper, spectrum_min=spectrum_min)
    _STATE.native_calls["chebyshev_filter"] += 1
    return out


class _ReferenceSeam:
    """The graph seam of the native filter over the reference's ``CuspFactoredHamiltonian``: its
    geometry and potential as a ``cdftb_operator`` (``_operator_of``), keyed by the pointers the
    operator carries."""

    dtype = torch.float64

    def __init__(self, ham, potential: torch.Tensor, op) -> None:
        self.ham = ham
        self._potential = potential
        faces, inv, _ = op._keep
        self._key = ("cusp-reference", tuple(int(n) for n in ham.grid.shape), float(ham.grid.spacing),
                     tuple(f.data_ptr() for f in faces), inv.data_ptr())

    def operator(self, potential: torch.Tensor, orbitals_per_group: int = 1):
        op, why = _operator_of(self.ham, potential)
        if op is None:
            raise RuntimeError(why)
        op.orbitals_per_group = int(orbitals_per_group)
        return op

    def filter_potential(self) -> torch.Tensor:
        return self._potential

    def graph_geometry_key(self) -> tuple:
        return self._key

    def note_applications(self, count: int) -> None:
        self.ham.note_applications(int(count))


class NativeFilterEngine(GraphedChebyshevFilter):
    """In place of ``GraphedChebyshevFilter`` (``chefsi.py:185-392``), with its call and its
    ``record()`` keys: the fused filter on the reference's operator, replayed from a CUDA graph
    per block shape and geometry (this package's engine). An operator the fused filter does not
    cover (the level-shifted rung) runs the reference's eager recurrence, counted by reason as
    the reference's engine counts its eager calls."""

    def _seam(self, ham, block):
        if block.dtype != torch.float64:
            return None, "not float64"
        if not all(hasattr(ham, a) for a in ("grid", "factor", "_inverse_weight", "graph_potential",
                                             "note_applications")):
            return None, f"operator {type(ham).__name__} is not a cusp-factorised Hamiltonian"
        potential = ham.graph_potential()
        if potential.dim() != 1:
            return None, "potential is not one (n_points,) field"
        potential = potential.to(torch.float64).contiguous()
        op, why = _operator_of(ham, potential)
        if op is None:
            return None, why
        return _ReferenceSeam(ham, potential, op), None

    def _filter_directly(self, ham, block, degree, lower, upper, spectrum_min):
        out = None
        if block.device.type == "cuda":
            out, _ = native_filter(ham, block, degree, lower, upper, spectrum_min)
        if out is None:
            original = _original("cdft.eigen.chefsi", "chebyshev_filter")
            return original(ham, block, degree, lower=lower, upper=upper, spectrum_min=spectrum_min)
        return out

    def __call__(self, ham, block, degree, lower, upper, spectrum_min):
        out = super().__call__(ham, block, degree, lower, upper, spectrum_min)
        _STATE.native_calls["filter_engine"] += 1
        return out

    def record(self) -> dict:
        out = super().record()
        out["engine"] = f"{TIER} fused filter (one launch per Chebyshev step) replayed from a CUDA graph"
        return out


def graphed_filter_for(device):
    """``graphed_filter_for`` (``chefsi.py:395-407``): the native engine on CUDA, None elsewhere."""
    device = torch.device(device)
    if device.type != "cuda":
        return None
    return NativeFilterEngine(device)


# ---------------------------------------------------------------------------------------------
# (c1) the Coulomb-cutoff Poisson solve


def native_poisson(solver, density: torch.Tensor):
    """The native plan for the reference's ``CoulombCutoffPoisson`` (built once per instance)."""
    grid = solver.grid
    if not getattr(grid, "_full_box", True):
        return None, "masked domain"
    plan = solver.__dict__.get("_cdftb_plan")
    if plan is None or plan.grid.device != density.device:
        from .grid import UniformGrid
        from .poisson import CoulombCutoffPoisson

        native_grid = UniformGrid(grid.shape, float(grid.spacing), tuple(float(o) for o in grid.origin),
                                  device=density.device)
        plan = CoulombCutoffPoisson(native_grid, pad_factor=float(solver.pad_factor))
        if plan.padded_shape != tuple(solver.padded_shape) or abs(plan.cutoff_radius - solver.cutoff_radius) > 1e-12:
            return None, "padded shape or cutoff differs"
        solver.__dict__["_cdftb_plan"] = plan
    return plan.solve(density.to(torch.float64)), None


def poisson_solve(self, density, grid=None):
    """``CoulombCutoffPoisson.solve`` (``src/cdft/operators/poisson.py:66-84``)."""
    original = _original("cdft.operators.poisson", "CoulombCutoffPoisson.solve")
    if density.device.type != "cuda" or density.dim() != 1 or (grid is not None and grid is not self.grid):
        return original(self, density, grid)  # the reference's own errors and CPU path
    out, why = native_poisson(self, density)
    if out is None:
        return _fallback("CoulombCutoffPoisson.solve", why, original, self, density, grid)
    _STATE.native_calls["poisson"] += 1
    return out


# ---------------------------------------------------------------------------------------------
# (d) exchange-correlation


class _XCOutput(NamedTuple):
    e_xc: torch.Tensor
    v_xc: torch.Tensor
    v_sigma: torch.Tensor | None
    v_tau: torch.Tensor | None = None
    v_lapl: torch.Tensor | None = None
    v_nldf: torch.Tensor | None = None


def _output_type():
    """The reference's ``contract.XCOutput`` when the reference is loaded, else an equivalent."""
    import sys

    contract = sys.modules.get("contract")
    return getattr(contract, "XCOutput", _XCOutput)


def native_evaluate(functional, density, sigma, tau, lapl, nldf):
    from .xc import TABLE, functional_by_name

    name = str(getattr(functional, "name", "")).lower()
    if name not in TABLE:
        return None, f"functional {name!r} has no native kernel"
    if tuple(getattr(functional, "libxc_reference", ())) != TABLE[name][2]:
        return None, f"functional {name!r} is composed differently from the native one"
    if tau is not None or lapl is not None:
        return None, "meta-GGA ingredients"
    rung = getattr(getattr(functional, "rung", None), "value", getattr(functional, "rung", 1))
    if rung >= 2 and sigma is None:
        raise ValueError(f"{name} is a rung-{rung} functional and needs sigma")
    if nldf is not None:
        raise ValueError(f"{name} is semi-local and consumes no non-local features")
    out = functional_by_name(name).evaluate(density, sigma if rung >= 2 else None)
    sig_out = None
    if sigma is not None:
        # the reference returns a zero v_sigma for an LDA given sigma (autograd of an unused input)
        sig_out = out.v_sigma if out.v_sigma is not None else torch.zeros_like(sigma, dtype=torch.float64)
    return _output_type()(e_xc=out.e_xc, v_xc=out.v_xc, v_sigma=sig_out, v_tau=None, v_lapl=None, v_nldf=None), None


def evaluate(self, density, sigma=None, tau=None, lapl=None, nldf=None):
    """``SemiLocalFunctional.evaluate`` (``src/cdft/xc/base.py:115-156``)."""
    original = _original("cdft.xc.base", "SemiLocalFunctional.evaluate")
    if density.device.type != "cuda":
        return original(self, density, sigma, tau, lapl, nldf)
    out, why = native_evaluate(self, density, sigma, tau, lapl, nldf)
    if out is None:
        return _fallback("SemiLocalFunctional.evaluate", why, original, self, density, sigma, tau, lapl, nldf)
    _STATE.native_calls["xc"] += 1
    return out


# ---------------------------------------------------------------------------------------------
# install / uninstall

#: (module, attribute path, replacement)
SEAMS = (
    ("cdft.operators.fused", "device_weighted_divergence", device_weighted_divergence),
    ("cdft.operators.hamiltonian", "CuspFactoredHamiltonian.kinetic_apply", kinetic_apply),
    ("cdft.operators.hamiltonian", "CuspFactoredHamiltonian.apply_with_potential", apply_with_potential),
    ("cdft.eigen.chefsi", "chebyshev_filter", chebyshev_filter),
    ("cdft.eigen.chefsi", "graphed_filter_for", graphed_filter_for),
    ("cdft.scf.loop", "graphed_filter_for", graphed_filter_for),
    ("cdft.scf.noninteracting", "graphed_filter_for", graphed_filter_for),
    ("cdft.operators.poisson", "CoulombCutoffPoisson.solve", poisson_solve),
    ("cdft.xc.base", "SemiLocalFunctional.evaluate", evaluate),
)


def _owner(module: str, path: str):
    obj = importlib.import_module(module)
    parts = path.split(".")
    for p in parts[:-1]:
        obj = getattr(obj, p)
    return obj, parts[-1]


def install(mode: str | None = None) -> dict:
    """Bind the native seams into the importable reference package ``cdft`` (idempotent).

    ``mode`` overrides ``CDFT_NATIVE``. ``off`` binds nothing. ``auto`` binds when the CUDA library
    loads and records the reason when it does not; ``on`` raises instead. Returns :func:`record`.
    """
    m = requested_mode(mode)
    if _STATE.saved:
        _STATE.mode = m if m != "off" else _STATE.mode
        if m == "off":
            uninstall()
        return record()
    _STATE.mode = m
    _STATE.reason = None
    if m == "off":
        _STATE.reason = f"{ENV_NATIVE}=off"
        return record()
    try:
        _lib.library()
    except Exception as exc:  # noqa: BLE001 - recorded (auto) or raised (on)
        if m == "on":
            raise RuntimeError(f"{ENV_NATIVE}=on: the native library does not load: {exc}") from exc
        _STATE.reason = f"the native library does not load: {exc}"
        return record()
    for module, path, replacement in SEAMS:
        owner, name = _owner(module, path)
        _STATE.saved[(module, path)] = owner.__dict__[name] if isinstance(owner, type) else getattr(owner, name)
    for module, path, replacement in SEAMS:
        owner, name = _owner(module, path)
        setattr(owner, name, replacement)
    return record()


def uninstall() -> None:
    """Restore every seam :func:`install` bound."""
    for (module, path), original in list(_STATE.saved.items()):
        owner, name = _owner(module, path)
        setattr(owner, name, original)
    _STATE.saved.clear()
    _STATE.mode = "off"
