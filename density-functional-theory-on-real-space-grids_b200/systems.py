"""The systems the measured workloads solve: nuclei, electrons, box and spacing.

Each definition restates the reference's own configuration of that system:

- ``he_lda``: He, two electrons, a cubic box of 16 bohr at h = 0.25 (65^3), the scenario
  ``he_atom_lda`` (``physics_config.py:389``) at ``numerics_for("he_atom_lda", "standard",
  half_box=8.0)``; at h = 0.16 the same box holds 101^3 points.
- ``h2_plus``: H2+, two protons at z = -R/2 and +R/2 and one electron (``physics_config.py:179``),
  in a box of transverse^2 x (R + 12) bohr at h = 0.25 with the lattice unanchored
  (``derive_grid=False``): the bond scan's members.

A system carries what the device geometry and the solve take (``UniformGrid.box`` and
``build_cusp_geometry``); the functional and the mixing are the caller's.
"""

from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class System:
    """Point nuclei (charges, positions in bohr), the electron count and the grid's box."""

    charges: tuple
    positions: tuple
    n_electrons: float
    box_lengths: tuple
    spacing: float
    anchor: tuple | None = None  # None: the lattice is not anchored on a nucleus


def he_lda(spacing: float = 0.25, edge: float = 16.0) -> System:
    """He in a cubic box of ``edge`` bohr (65^3 points at h = 0.25, 101^3 at h = 0.16)."""
    return System(charges=(2.0,), positions=((0.0, 0.0, 0.0),), n_electrons=2.0, box_lengths=(edge,) * 3,
                  spacing=spacing)


def h2_plus(bond: float = 2.0, spacing: float = 0.25, transverse: float = 12.0) -> System:
    """H2+ along z with bond length ``bond`` bohr, box ``transverse^2 x (bond + 12)``."""
    half = bond / 2.0
    return System(charges=(1.0, 1.0), positions=((0.0, 0.0, -half), (0.0, 0.0, half)), n_electrons=1.0,
                  box_lengths=(transverse, transverse, bond + 12.0), spacing=spacing)
