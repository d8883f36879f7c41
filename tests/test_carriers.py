"""The reference's contract carriers (``contract.py:431-528``) accepted by the solve entry points.

The CPU tests convert the reference's own dataclasses where its checkout is readable
(``CDFT_REFERENCE``), and a stand-in with the same fields everywhere. The GPU test solves config 1
with a stand-in of the reference's ``EigenConfig`` and checks it bit for bit against the same
settings in this package's own dataclass.
"""

from __future__ import annotations

import dataclasses
import enum
import importlib
import os
import sys
from pathlib import Path

import pytest

REFERENCE = Path(os.environ.get("CDFT_REFERENCE", "/root/reference"))


class _Kind(str, enum.Enum):
    CHEFSI = "chefsi"
    LOBPCG = "lobpcg"


class _Scheme(str, enum.Enum):
    LINEAR = "linear"
    PERIODIC_PULAY = "periodic_pulay"


@dataclasses.dataclass(frozen=True)
class _EigenLike:
    """The fields of the reference's ``contract.EigenConfig``, with its enum for ``kind``."""

    kind: _Kind = _Kind.CHEFSI
    n_extra_states: int = 8
    extra_states_fraction: float = 0.20
    chebyshev_degree: int = 12
    lanczos_steps: int = 12
    bound_safety: float = 1.02
    max_iterations: int = 60
    residual_tol: float = 1.0e-6
    cross_check: bool = False
    cross_check_tol: float = 1.0e-8


@dataclasses.dataclass(frozen=True)
class _MixingLike:
    scheme: _Scheme = _Scheme.LINEAR
    alpha: float = 0.3
    history: int = 8
    pulay_period: int = 3
    kerker: bool = False
    kerker_q0: float = 1.5


@pytest.fixture(scope="module")
def contract():
    if not (REFERENCE / "contract.py").is_file():
        pytest.skip("the reference checkout is not available here")
    sys.dont_write_bytecode = True
    if str(REFERENCE) not in sys.path:
        sys.path.insert(0, str(REFERENCE))
    return importlib.import_module("contract")


@pytest.fixture(scope="module")
def carriers(pkg):
    return importlib.import_module("cdft_b200.carriers")


def test_reference_numerics_convert(contract, carriers, pkg):
    numerics = contract.NumericsConfig(
        eigen=contract.EigenConfig(chebyshev_degree=17, residual_tol=1e-9, cross_check=True),
        mixing=contract.MixingConfig(scheme=contract.MixingScheme.LINEAR, alpha=0.25),
        scf=contract.SCFConfig(energy_tol=1e-9, max_iterations=77),
    )
    eigen, mixing, scf = carriers.from_numerics(numerics)
    assert isinstance(eigen, pkg.EigenConfig) and isinstance(mixing, pkg.MixingConfig)
    assert isinstance(scf, pkg.SCFConfig)
    assert (eigen.chebyshev_degree, eigen.residual_tol, eigen.cross_check) == (17, 1e-9, True)
    assert eigen.n_extra_states == contract.EigenConfig().n_extra_states
    assert eigen.max_iterations == contract.EigenConfig().max_iterations
    assert mixing.scheme == "linear" and mixing.alpha == 0.25
    assert (scf.energy_tol, scf.max_iterations, scf.density_tol) == (1e-9, 77, contract.SCFConfig().density_tol)
    # every field this package reads has the reference's value
    for ours, theirs in ((eigen, numerics.eigen), (mixing, numerics.mixing), (scf, numerics.scf)):
        for f in dataclasses.fields(ours):
            assert getattr(ours, f.name) == getattr(getattr(theirs, f.name), "value", getattr(theirs, f.name))


def test_reference_defaults_build_a_mixer(contract, carriers, pkg):
    mixing = carriers.mixing_config(contract.MixingConfig())
    assert mixing.scheme == "periodic_pulay"
    mixer = pkg.scf.make_mixer(mixing, mixing.alpha, inner_weights=None)
    assert type(mixer).__name__ == "PulayMixer"


def test_reference_settings_the_path_does_not_run_are_refused(contract, carriers):
    with pytest.raises(ValueError, match="lobpcg"):
        carriers.eigen_config(contract.EigenConfig(kind=contract.EigensolverKind.LOBPCG))
    with pytest.raises(ValueError, match="fermi"):
        carriers.scf_config(contract.SCFConfig(occupation=contract.OccupationScheme.FERMI))


def test_stand_in_and_own_types(carriers, pkg):
    assert carriers.eigen_config(None) == pkg.EigenConfig()
    own = pkg.EigenConfig(chebyshev_degree=9)
    assert carriers.eigen_config(own) is own
    converted = carriers.eigen_config(_EigenLike())
    assert converted.chebyshev_degree == 12 and converted.max_iterations == 60
    assert carriers.mixing_config(_MixingLike()).scheme == "linear"
    with pytest.raises(TypeError, match="pulay_period"):
        carriers.mixing_config(type("Partial", (), {"scheme": "linear", "alpha": 0.3})())
    with pytest.raises(TypeError, match="NumericsConfig"):
        carriers.from_numerics(object())


@pytest.mark.gpu
def test_solve_with_the_reference_eigen_carrier(pkg, cuda):
    from oracle import scf as oscf

    system = oscf.h_atom(points_per_edge=17, half_box=4.0)
    geo = pkg.geometry.build_cusp_geometry(pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, cuda),
                                           system.charges, system.positions)
    like = _EigenLike(chebyshev_degree=14, residual_tol=1e-9, max_iterations=200, n_extra_states=4)
    own = pkg.EigenConfig(chebyshev_degree=14, residual_tol=1e-9, max_iterations=200, n_extra_states=4,
                          extra_states_fraction=0.20, lanczos_steps=12, bound_safety=1.02)
    a = pkg.scf.solve_noninteracting(geo, n_electrons=1.0, seed=3, eigen=like)
    b = pkg.scf.solve_noninteracting(geo, n_electrons=1.0, seed=3, eigen=own)
    assert a["total"] == b["total"] and a["iterations"] == b["iterations"]
    assert abs(a["total"] - (-0.5)) < 5e-3
