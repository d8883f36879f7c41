"""The reference's contract carriers accepted where this package takes its own settings.

A caller of the reference holds ``contract.EigenConfig``, ``contract.MixingConfig``,
``contract.SCFConfig`` (``contract.py:431-490``) and the ``contract.NumericsConfig`` that bundles
them (``contract.py:512-528``). Every solve entry point of this package passes its settings
through :func:`eigen_config`, :func:`mixing_config` or :func:`scf_config`, so it accepts either
this package's dataclass or the reference's, by field name (the reference's module is not
imported: any object carrying the fields converts). Enum members are read by ``.value``.

Fields the reference carries but does not act on are checked rather than dropped silently:
``SCFConfig.occupation`` must be ``fixed`` (the reference's ``KohnShamStep.occupy``,
``src/cdft/scf/step.py:357-364``, is Aufbau only) and ``EigenConfig.kind`` must be ``chefsi``
(the production solver; LOBPCG runs as the cross-check, ``src/cdft/scf/noninteracting.py:182``).
"""

from __future__ import annotations

import dataclasses

from .eigen import EigenConfig
from .scf import MixingConfig, SCFConfig


def _plain(value):
    """An enum member's value, anything else unchanged."""
    return getattr(value, "value", value)


def _convert(value, cls, what: str):
    if value is None:
        return cls()
    if isinstance(value, cls):
        return value
    names = [f.name for f in dataclasses.fields(cls)]
    missing = [name for name in names if not hasattr(value, name)]
    if missing:
        raise TypeError(f"{type(value).__name__} cannot stand for {what}: it has no {', '.join(missing)}")
    return cls(**{name: _plain(getattr(value, name)) for name in names})


def eigen_config(value) -> EigenConfig:
    """This package's ``EigenConfig`` from itself, ``None`` (defaults) or ``contract.EigenConfig``."""
    kind = _plain(getattr(value, "kind", "chefsi"))
    if str(kind).lower() != "chefsi":
        raise ValueError(f"eigensolver kind {kind!r} is not the production solver here; only 'chefsi' runs "
                         "(LOBPCG is the cross-check, EigenConfig.cross_check)")
    return _convert(value, EigenConfig, "the eigensolver settings")


def mixing_config(value) -> MixingConfig:
    """This package's ``MixingConfig`` from itself, ``None`` or ``contract.MixingConfig``."""
    return _convert(value, MixingConfig, "the mixing settings")


def scf_config(value) -> SCFConfig:
    """This package's ``SCFConfig`` from itself, ``None`` or ``contract.SCFConfig``."""
    occupation = _plain(getattr(value, "occupation", "fixed"))
    if str(occupation).lower() != "fixed":
        raise ValueError(f"occupation scheme {occupation!r} is not wired: occupations are Aufbau ('fixed'), "
                         "as in the reference's KohnShamStep.occupy")
    return _convert(value, SCFConfig, "the SCF settings")


def from_numerics(numerics) -> tuple[EigenConfig, MixingConfig, SCFConfig]:
    """The three settings a solve reads, from a ``contract.NumericsConfig`` (its ``eigen``, ``mixing``
    and ``scf`` fields)."""
    for name in ("eigen", "mixing", "scf"):
        if not hasattr(numerics, name):
            raise TypeError(f"{type(numerics).__name__} is not a NumericsConfig: it has no {name}")
    return eigen_config(numerics.eigen), mixing_config(numerics.mixing), scf_config(numerics.scf)
