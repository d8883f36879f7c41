"""The uniform box grid (the full-box, zero-halo case of ``src/cdft/grid.py:480-760``).

Fields are flat ``(..., n_points)`` in C order over ``(nx, ny, nz)``: the flattened box, so the
reference's ``scatter_to_box`` / ``gather_from_box`` are views here.
"""

from __future__ import annotations

import torch


class UniformGrid:
    """Shape, spacing and origin of a full box (``src/cdft/grid.py:482``)."""

    def __init__(self, shape, spacing: float, origin, device: torch.device | str = "cuda", fd_order: int = 8,
                 gradient_order: int = 8) -> None:
        self.shape = tuple(int(n) for n in shape)
        self.spacing = float(spacing)
        self.origin = tuple(float(o) for o in origin)
        self.device = torch.device(device)
        self.fd_order = int(fd_order)
        self.gradient_order = int(gradient_order)
        self.n_points = self.shape[0] * self.shape[1] * self.shape[2]

    @classmethod
    def box(cls, lengths, spacing: float, anchor=None, device="cuda", fd_order: int = 8) -> "UniformGrid":
        """``UniformGrid.from_config`` for ``DomainMode.BOX`` with a zero halo (grid.py:580-605).

        ``counts = round(L/h) + 1``, ``h`` re-derived from the first edge, and the origin snapped
        so the coordinate origin (or ``anchor``) is a lattice point. Python's ``round`` (half to
        even) is the reference's.
        """
        h = float(spacing)
        counts = tuple(max(int(round(length / h)) + 1, 1) for length in lengths)
        h = lengths[0] / (counts[0] - 1) if counts[0] > 1 else h
        if anchor is None:
            origin = tuple(-h * round(0.5 * length / h) for length in lengths)
        else:
            origin = tuple(float(a) - h * round((float(a) + 0.5 * length) / h) for a, length in zip(anchor, lengths))
        return cls(counts, h, origin, device=device, fd_order=fd_order)

    @property
    def volume_element(self) -> float:
        return self.spacing ** 3

    def points(self) -> torch.Tensor:
        """Cartesian coordinates of every grid point, ``(N, 3)`` float64 in C order (grid.py points)."""
        axes = [torch.arange(n, dtype=torch.float64, device=self.device) * self.spacing + o
                for n, o in zip(self.shape, self.origin)]
        x, y, z = torch.meshgrid(*axes, indexing="ij")
        return torch.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], dim=1)

    def scatter_to_box(self, field: torch.Tensor) -> torch.Tensor:
        return field.reshape(*field.shape[:-1], *self.shape)

    def gather_from_box(self, box: torch.Tensor) -> torch.Tensor:
        return box.reshape(*box.shape[: box.dim() - 3], -1)

    def describe(self) -> dict:
        return {"shape": self.shape, "spacing_bohr": self.spacing, "origin_bohr": self.origin, "n_points": self.n_points}

    def __repr__(self) -> str:
        return f"UniformGrid(shape={self.shape}, h={self.spacing:.4f})"
