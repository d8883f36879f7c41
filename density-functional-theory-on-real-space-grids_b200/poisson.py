"""The Coulomb-cutoff Poisson solver on the device (host mirror of ``src/cdft/operators/poisson.py``).

The plan (padded shape, truncated kernel K(G), transform buffers) is built once per grid by
``cdftb_poisson_plan_create``; ``solve`` is one library call: five pruned axis-wise transforms with
the kernel multiply fused into the x pass.
"""

from __future__ import annotations

import ctypes
import math

import torch

from . import _lib
from ._lib import call, ptr, stream_handle
from .grid import UniformGrid


def fft_friendly(n: int) -> int:
    """Next 2,3,5-smooth integer (``src/cdft/operators/poisson.py:110-120``)."""
    c = n
    while True:
        r = c
        for p in (2, 3, 5):
            while r % p == 0:
                r //= p
        if r == 1:
            return c
        c += 1


class CoulombCutoffPoisson:
    """Free-space Hartree solver (``src/cdft/operators/poisson.py:21``)."""

    def __init__(self, grid: UniformGrid, pad_factor: float = 2.0, max_batch: int = 1) -> None:
        if pad_factor < 2.0:
            raise ValueError("pad_factor must be at least 2.0 for the convolution to be linear")
        self.grid = grid
        self.pad_factor = pad_factor
        self.max_batch = int(max_batch)
        plan = ctypes.c_void_p()
        shape = (ctypes.c_int * 3)()
        radius = ctypes.c_double()
        torch.cuda.set_device(grid.device)
        call("cdftb_poisson_plan_create", *grid.shape, grid.spacing, float(pad_factor), self.max_batch,
             ctypes.byref(plan), shape, ctypes.byref(radius))
        self._plan = plan
        self.padded_shape = tuple(int(s) for s in shape)
        self.cutoff_radius = float(radius.value)
        expected = tuple(fft_friendly(int(math.ceil(pad_factor * n))) for n in grid.shape)
        if self.padded_shape != expected:
            raise RuntimeError(f"padded shape {self.padded_shape} != {expected}")

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _lib.library().cdftb_poisson_plan_destroy(plan)
            except Exception:  # noqa: BLE001 - interpreter shutdown
                pass
            self._plan = None

    def kernel(self) -> torch.Tensor:
        """The device kernel table K on the half spectrum, shape (N0, N1, N2/2+1) (a copy)."""
        table = ctypes.c_void_p()
        call("cdftb_poisson_kernel_table", self._plan, ctypes.byref(table))
        n0, n1, n2 = self.padded_shape
        count = n0 * n1 * (n2 // 2 + 1)
        out = torch.empty(count, dtype=torch.float64, device=self.grid.device)
        # device-to-device copy through the library's cast (f64 -> f64 is a plain copy)
        call("cdftb_cast", table.value, 0, ptr(out), 0, count, stream_handle(self.grid.device))
        return out.reshape(n0, n1, n2 // 2 + 1)

    def solve(self, density: torch.Tensor, grid: UniformGrid | None = None) -> torch.Tensor:
        """``v_H`` on the domain for a total density ``(n_points,)`` (poisson.py:66-84)."""
        if density.dim() != 1:
            raise ValueError(f"expected a total density of shape (n_points,), got {tuple(density.shape)}; "
                             "sum over the spin axis before calling the Hartree solver")
        return self.solve_batch(density.reshape(1, -1))[0]

    def solve_batch(self, densities: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
        """Solve for ``(batch, n_points)`` densities on the same grid in one call."""
        _lib.require_cuda(densities, "density")
        x = densities.to(torch.float64).contiguous()
        batch = x.shape[0]
        if x.shape[-1] != self.grid.n_points:
            raise ValueError(f"density has {x.shape[-1]} points, grid has {self.grid.n_points}")
        if batch > self.max_batch:
            raise ValueError(f"batch {batch} exceeds the plan's max_batch {self.max_batch}")
        if out is None:
            out = torch.empty_like(x)
        call("cdftb_poisson_solve", self._plan, ptr(x), ptr(out), batch, stream_handle(x.device))
        return out

    def energy(self, density: torch.Tensor, v_hartree: torch.Tensor) -> float:
        return float(0.5 * (density * v_hartree).sum() * self.grid.volume_element)
