"""cdft_b200: the cdft hot path (cusp-factorised apply, CheFSI + Rayleigh--Ritz, Coulomb-cutoff
Poisson, LDA/PBE XC with the cusp-aware quadrature, and the SCF driver around them) as sm_100a CUDA
kernels behind a C ABI (``include/cdftb.h``), with a host layer that mirrors the reference's Python
interfaces (``src/cdft/operators``, ``src/cdft/eigen``, ``src/cdft/xc``, ``src/cdft/scf``).

The package directory's name is not a Python identifier; ``__graft_entry__.package()`` imports it
and registers it as ``cdft_b200``.
"""

from __future__ import annotations

from . import _lib, adjoint, batch, carriers, eigen, geometry, operators, poisson, replicas, rng, scf, systems, xc
from .eigen import (
    ChebyshevFilteredSubspace,
    EigenConfig,
    EigenResult,
    SpectralBoundsHint,
    chebyshev_coefficients,
    chebyshev_filter,
    rayleigh_ritz,
    residual_norms,
)
from .grid import UniformGrid
from .geometry import CuspFactor, CuspGeometry, CuspQuadrature, StepGeometry, build_cusp_geometry
from .operators import CuspFactoredHamiltonian, Measure, lanczos_bounds, measure_cross, seeded_randn, weighted_divergence
from .poisson import CoulombCutoffPoisson
from .scf import (KohnShamStep, MixingConfig, SCFConfig, initial_density, solve_noninteracting,
                  solve_self_consistent)
from .xc import LDA, PBE, functional_by_name

__all__ = [
    "CoulombCutoffPoisson",
    "CuspFactor",
    "CuspGeometry",
    "CuspQuadrature",
    "KohnShamStep",
    "LDA",
    "MixingConfig",
    "PBE",
    "SCFConfig",
    "StepGeometry",
    "build_cusp_geometry",
    "functional_by_name",
    "initial_density",
    "solve_noninteracting",
    "solve_self_consistent",
    "ChebyshevFilteredSubspace",
    "CuspFactoredHamiltonian",
    "EigenConfig",
    "EigenResult",
    "Measure",
    "SpectralBoundsHint",
    "UniformGrid",
    "chebyshev_coefficients",
    "chebyshev_filter",
    "lanczos_bounds",
    "measure_cross",
    "rayleigh_ritz",
    "residual_norms",
    "seeded_randn",
    "weighted_divergence",
]


def library_path() -> str:
    return str(_lib.LIBRARY_PATH)
