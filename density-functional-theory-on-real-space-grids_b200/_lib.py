"""ctypes binding of ``lib/libcdftb.so`` (declared in ``include/cdftb.h``).

The library is the only compute path: if it cannot be loaded, importing the operators raises
``RuntimeError`` instead of falling back to anything else. Every call checks the returned status
and raises ``CdftbError`` with the library's status text.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import torch

HERE = Path(__file__).resolve().parent
LIBRARY_PATH = Path(os.environ.get("CDFTB_LIBRARY", HERE / "lib" / "libcdftb.so"))

F64, F32 = 0, 1
_DTYPES = {torch.float64: F64, torch.float32: F32}

c_int, c_int64, c_double, c_void_p = ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_void_p
c_char_p = ctypes.c_char_p


class Operator(ctypes.Structure):
    """``cdftb_operator`` (include/cdftb.h)."""

    _fields_ = [
        ("nx", c_int), ("ny", c_int), ("nz", c_int), ("accuracy", c_int), ("spacing", c_double),
        ("dtype", c_int), ("face_weights", c_void_p * 3), ("inverse_weight", c_void_p),
        ("potential", c_void_p), ("potential_stride", c_int64), ("orbitals_per_group", c_int),
        ("quadrature", c_void_p), ("per_system_geometry", c_int), ("system_shapes", c_void_p),
    ]


# name -> (restype, argtypes)
SIGNATURES: dict[str, tuple] = {
    "cdftb_version": (c_int, []),
    "cdftb_status_string": (c_char_p, [c_int]),
    "cdftb_last_cuda_error": (c_int, []),
    "cdftb_launch_count": (ctypes.c_ulonglong, []),
    "cdftb_weighted_divergence_f64": (c_int, [c_void_p, c_void_p, c_int64, c_int, c_int, c_int, c_void_p, c_void_p,
                                              c_void_p, c_double, c_int, c_void_p]),
    "cdftb_cusp_apply_work_bytes": (c_int64, [ctypes.POINTER(Operator), c_int64]),
    "cdftb_cusp_apply": (c_int, [ctypes.POINTER(Operator), c_void_p, c_int, c_void_p, c_int, c_int64, c_int, c_void_p,
                                 c_int64, c_void_p]),
    "cdftb_chebyshev_filter_work_bytes": (c_int64, [ctypes.POINTER(Operator), c_int64]),
    "cdftb_chebyshev_filter": (c_int, [ctypes.POINTER(Operator), c_void_p, c_int, c_void_p, c_int, c_void_p, c_int64,
                                       c_int64, c_void_p, c_int, c_void_p]),
    "cdftb_device_status": (c_int, [ctypes.POINTER(c_int)]),
    "cdftb_measure_cross_scratch_bytes": (c_int64, [c_int, c_int, c_int64, c_int]),
    "cdftb_measure_cross_f64": (c_int, [c_void_p, c_int, c_int64, c_void_p, c_int, c_int64, c_void_p, c_int64, c_int,
                                        c_void_p, c_void_p, c_int64, c_void_p]),
    "cdftb_measure_cross_grouped_f64": (c_int, [c_void_p, c_int, c_int64, c_void_p, c_int, c_int64, c_void_p, c_int64,
                                                c_int64, c_int, c_void_p, c_void_p, c_int64, c_void_p]),
    "cdftb_measure_cross_static_capacity_bytes": (c_int64, []),
    "cdftb_measure_cross_static_f64": (c_int, [c_void_p, c_int, c_int64, c_void_p, c_int, c_int64, c_void_p, c_int64,
                                               c_int, c_void_p, c_void_p]),
    "cdftb_small_cholesky_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]),
    "cdftb_block_trsm_lower_f64": (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int, c_int64, c_int, c_int64, c_int,
                                           c_void_p]),
    "cdftb_small_eigh_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]),
    "cdftb_block_rotate_f64": (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_int, c_int64, c_int, c_int, c_int64,
                                       c_int, c_void_p]),
    "cdftb_block_ritz_scratch_bytes": (c_int64, [c_int, c_int64, c_int]),
    "cdftb_block_ritz_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int64, c_int,
                                     c_void_p, c_void_p, c_void_p, c_int64, c_void_p]),
    "cdftb_block_residual_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int64, c_int, c_int64,
                                         c_void_p]),
    "cdftb_lanczos_update_f64": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int,
                                         c_void_p]),
    "cdftb_cast": (c_int, [c_void_p, c_int, c_void_p, c_int, c_int64, c_void_p]),
    "cdftb_stencil_set_tile": (c_int, [c_int, c_int, c_int]),
    "cdftb_filter_autotune": (c_int, [c_int]),
    "cdftb_filter_wide": (c_int, [c_int]),
    "cdftb_filter_test_withhold": (c_int, [c_int]),
    "cdftb_density_residual_f64": (c_int, [c_void_p, c_void_p, c_int, c_int64, c_int, c_void_p, c_void_p, c_void_p,
                                           c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_external_grid_terms_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                              c_int, c_void_p, c_void_p]),
    "cdftb_filter_tuned_tile": (c_int, [c_int, c_int, c_int, c_int, c_int64, c_void_p, c_void_p]),
    "cdftb_filter_tuned_tile_rows": (c_int, [c_int, c_int, c_int, c_int, c_int64, c_void_p]),
    "cdftb_poisson_plan_create": (c_int, [c_int, c_int, c_int, c_double, c_double, c_int, ctypes.POINTER(c_void_p),
                                          ctypes.POINTER(c_int), ctypes.POINTER(c_double)]),
    "cdftb_poisson_plan_destroy": (c_int, [c_void_p]),
    "cdftb_poisson_kernel_table": (c_int, [c_void_p, ctypes.POINTER(c_void_p)]),
    "cdftb_poisson_solve": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "cdftb_xc_lda_vwn_f64": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p]),
    "cdftb_xc_pbe_f64": (c_int, [c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_xc_is_gga": (c_int, [c_int]),
    "cdftb_kerker_work_bytes": (c_int64, [c_int, c_int, c_int, c_int]),
    "cdftb_kerker_precondition_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_double, c_double, c_void_p,
                                              c_void_p, c_int64, c_void_p]),
    "cdftb_reciprocal_filter_f64": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_double, c_int, c_double, c_void_p,
                                            c_void_p, c_int64, c_void_p]),
    "cdftb_xc_eval_f64": (c_int, [c_int, c_int, c_void_p, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_quadrature_stencils": (c_int, [c_void_p, c_int64, c_int, c_int, c_int, c_double, c_double, c_double, c_double,
                                          c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_lift_plan_scratch_bytes": (c_int64, [c_int64, c_int64]),
    "cdftb_lift_plan_build": (c_int, [c_void_p, c_int64, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_int64,
                                      c_void_p]),
    "cdftb_quadrature_interpolate_f64": (c_int, [c_void_p, c_void_p, c_int64, c_int, c_int, c_int, c_void_p, c_int,
                                                 c_int64, c_void_p, c_int64, c_void_p]),
    "cdftb_lift_plan_values_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_void_p,
                                           c_void_p]),
    "cdftb_quadrature_lift_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int,
                                          c_void_p, c_int, c_int64, c_void_p, c_int64, c_void_p]),
    "cdftb_quadrature_many_scratch_bytes": (c_int64, [c_int64, c_int64]),
    "cdftb_quadrature_interpolate_many_f64": (c_int, [c_void_p, c_void_p, c_int64, c_int, c_int, c_int, c_void_p, c_int,
                                                      c_int64, c_void_p, c_int64, c_void_p, c_int64, c_void_p]),
    "cdftb_quadrature_interpolate_grouped_f64": (c_int, [c_void_p, c_void_p, c_int64, c_int, c_int, c_int, c_void_p,
                                                         c_void_p, c_int64, c_void_p, c_int, c_int64, c_void_p,
                                                         c_int64, c_void_p, c_int64, c_void_p]),
    "cdftb_lift_segments_capacity": (c_int64, [c_int64, c_int64]),
    "cdftb_lift_segments_scratch_bytes": (c_int64, [c_int64]),
    "cdftb_lift_plan_segments": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int64, c_void_p, c_int64,
                                         c_void_p]),
    "cdftb_quadrature_lift_many_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int, c_int,
                                               c_int, c_int64, c_void_p, c_int, c_int64, c_void_p, c_int64, c_void_p,
                                               c_int64, c_void_p]),
    "cdftb_cusp_coefficients_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "cdftb_hartree_split_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int64, c_int, c_void_p,
                                        c_void_p, c_void_p]),
    "cdftb_potentials_node_lda_f64": (c_int, [c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int,
                                              c_void_p, c_void_p, c_void_p]),
    "cdftb_potentials_grid_lda_f64": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                              c_void_p, c_int, c_void_p, c_int64, c_int, c_void_p, c_void_p, c_void_p,
                                              c_void_p, c_void_p]),
    "cdftb_row_sums_scratch_bytes": (c_int64, [c_int, c_int64]),
    "cdftb_row_sums_f64": (c_int, [c_void_p, c_int, c_int64, c_void_p, c_void_p, c_int64, c_void_p]),
    "cdftb_gradient_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_double, c_int64,
                                   c_void_p]),
    "cdftb_fd_derivative_f64": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_double,
                                        c_int64, c_int, c_double, c_void_p]),
    "cdftb_geometry_cusp_fields": (c_int, [c_int, c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_double, c_double,
                                           c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                           c_void_p]),
    "cdftb_geometry_face_weights": (c_int, [c_int, c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_double, c_double,
                                            c_double, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_geometry_node_fields": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p,
                                           c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_geometry_grid_far": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_double,
                                        c_double, c_double, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_geometry_lumped_far": (c_int, [c_int, c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_double,
                                          c_double, c_double, c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                          c_void_p, c_double, c_double, c_void_p, c_void_p, c_void_p]),
    "cdftb_geometry_bare_terms": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_double, c_void_p,
                                          c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_geometry_step_fields": (c_int, [c_int, c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_double, c_double,
                                           c_double, c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "cdftb_geometry_initial_density": (c_int, [c_int, c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_double,
                                               c_double, c_double, c_double, c_void_p, c_void_p, c_void_p, c_void_p,
                                               c_void_p]),
    "cdftb_scale_f64": (c_int, [c_void_p, c_int64, c_double, c_void_p]),
}


class CdftbError(RuntimeError):
    """A cdftb entry point returned a non-zero status."""


_LIB = None


def library() -> ctypes.CDLL:
    """Load (once) and return the CUDA library; raise if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIBRARY_PATH.exists():
        raise RuntimeError(
            f"the cdftb CUDA library is not built ({LIBRARY_PATH} missing); run "
            "`python density-functional-theory-on-real-space-grids_b200/build.py` -- there is no CPU fallback")
    lib = ctypes.CDLL(str(LIBRARY_PATH))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    # The slab kernels' tiling is tuned on first use per grid shape and lane count (the first filter
    # call for a shape times the candidates and synchronises; results do not depend on the tiling).
    lib.cdftb_filter_autotune(0 if os.environ.get("CDFTB_AUTOTUNE", "1") == "0" else 1)
    _LIB = lib
    return lib


def register(name: str, restype, argtypes) -> None:
    """Declare the signature of an entry point defined by another module of this package."""
    SIGNATURES[name] = (restype, argtypes)
    if _LIB is not None:
        fn = getattr(_LIB, name)
        fn.restype = restype
        fn.argtypes = argtypes


def call(name: str, *args) -> None:
    """Call ``name`` and raise ``CdftbError`` on a non-zero status."""
    lib = library()
    status = getattr(lib, name)(*args)
    if status != 0:
        text = lib.cdftb_status_string(status).decode()
        cuda = lib.cdftb_last_cuda_error()
        raise CdftbError(f"{name}: {text} (status {status}, last CUDA error {cuda})")


class DeviceTimeout(CdftbError):
    """A kernel's bounded wait gave up (``CDFTB_ERR_TIMEOUT``): its outputs are not valid."""


#: How many timed-out launches :func:`check_device_status` has reported in this process. A captured
#: graph replays its launches with the abort token they had at capture, so a graph captured before a
#: timeout is not replayed after one (``eigen.GraphedChebyshevFilter`` captures again).
timeouts_reported = 0


def check_device_status(where: str = "") -> None:
    """Read and clear the library's device error flags; raise :class:`DeviceTimeout` if any was set.

    Synchronises the device. The drivers call it once per SCF or eigensolver iteration, where they
    already wait for the device to read their scalars, so that a timed-out launch stops the solve
    instead of feeding unwritten outputs into the next step.
    """
    lib = library()
    flags = c_int(0)
    status = lib.cdftb_device_status(ctypes.byref(flags))
    if status == 0:
        return
    text = lib.cdftb_status_string(status).decode()
    if flags.value:
        global timeouts_reported
        timeouts_reported += 1
        raise DeviceTimeout(f"{where or 'cdftb'}: a kernel gave up waiting ({text}, flags {flags.value}); "
                            "its results were discarded")
    raise CdftbError(f"cdftb_device_status: {text} (status {status})")


def ptr(t: torch.Tensor | None):
    """Device pointer of a contiguous tensor (``None`` -> NULL)."""
    if t is None:
        return None
    if not t.is_contiguous():
        raise ValueError("cdftb needs contiguous tensors")
    return t.data_ptr()


def dtype_code(t: torch.Tensor) -> int:
    try:
        return _DTYPES[t.dtype]
    except KeyError:
        raise ValueError(f"unsupported dtype {t.dtype}; cdftb takes float64 or float32") from None


def stream_handle(device: torch.device | None = None):
    """The current torch CUDA stream as a raw ``cudaStream_t``."""
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(t: torch.Tensor, name: str = "tensor") -> None:
    if t.device.type != "cuda":
        raise ValueError(f"{name} must be on a CUDA device (got {t.device}); cdftb has no CPU path")
