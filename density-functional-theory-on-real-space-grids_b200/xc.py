"""The native semi-local functionals on the device (host mirror of ``src/cdft/xc``).

``evaluate`` keeps the contract of ``SemiLocalFunctional.evaluate`` (``src/cdft/xc/base.py:115``):
``(n_spin, P)`` density with n_spin 1 or 2, ``(1 or 3, P)`` sigma; a GGA without sigma and any
non-local feature raise ``ValueError``, a wrong spin extent raises ``ValueError`` as ``split_spin``
does. Every name of the reference's table (``src/cdft/xc/dispatch.py:26-44``) is native:

- spin-restricted ``lda_vwn`` and ``pbe`` (the self-consistent path's functionals) run in the
  hand-differentiated kernels ``cdftb_xc_lda_vwn_f64`` / ``cdftb_xc_pbe_f64``;
- everything else -- the other LDAs and GGAs, the component functionals, and every spin-polarised
  input -- runs in ``cdftb_xc_eval_f64``, which differentiates the energy density with forward-mode
  dual numbers.
"""

from __future__ import annotations

from typing import NamedTuple

import torch

from . import _lib
from ._lib import call, ptr, stream_handle


class XCOutput(NamedTuple):
    """``contract.XCOutput`` (contract.py:759): energy density per volume and its derivatives."""

    e_xc: torch.Tensor
    v_xc: torch.Tensor
    v_sigma: torch.Tensor | None
    v_tau: torch.Tensor | None = None
    v_lapl: torch.Tensor | None = None
    v_nldf: torch.Tensor | None = None


#: name -> (cdftb_xc_id, rung, libxc identifiers) (``src/cdft/xc/dispatch.py:26-44``, ``lda.py``, ``gga.py``)
TABLE = {
    "lda_vwn": (0, 1, ("lda_x", "lda_c_vwn")),
    "lda_pw92": (1, 1, ("lda_x", "lda_c_pw")),
    "lda_pw92_mod": (2, 1, ("lda_x", "lda_c_pw_mod")),
    "lda_pz81": (3, 1, ("lda_x", "lda_c_pz")),
    "pbe": (4, 2, ("gga_x_pbe", "gga_c_pbe")),
    "blyp": (5, 2, ("gga_x_b88", "gga_c_lyp")),
    "lda_x": (6, 1, ("lda_x",)),
    "lda_c_vwn": (7, 1, ("lda_c_vwn",)),
    "lda_c_pw": (8, 1, ("lda_c_pw",)),
    "lda_c_pw_mod": (9, 1, ("lda_c_pw_mod",)),
    "lda_c_pz": (10, 1, ("lda_c_pz",)),
    "gga_x_pbe": (11, 2, ("gga_x_pbe",)),
    "gga_c_pbe": (12, 2, ("gga_c_pbe",)),
    "gga_x_b88": (13, 2, ("gga_x_b88",)),
    "gga_c_lyp": (14, 2, ("gga_c_lyp",)),
}

#: Every native functional name (``src/cdft/xc/dispatch.py:47``).
NATIVE: tuple[str, ...] = tuple(TABLE)


class SemiLocalFunctional:
    """One native functional (``src/cdft/xc/base.py:83-189``): ``rung``, ``name``, ``libxc_reference``."""

    def __init__(self, name: str) -> None:
        key = name.lower()
        if key not in TABLE:
            raise KeyError(f"unknown functional {name!r}. Native: {', '.join(NATIVE)}")
        self.name = key
        self.id, self.rung, self.libxc_reference = TABLE[key]

    def evaluate(self, density, sigma=None, tau=None, lapl=None, nldf=None) -> XCOutput:
        if self.rung >= 2 and sigma is None:
            raise ValueError(f"{self.name} is a rung-{self.rung} functional and needs sigma")
        if nldf is not None:
            raise ValueError(f"{self.name} is semi-local and consumes no non-local features")
        n_spin = density.shape[0]
        if n_spin not in (1, 2):
            raise ValueError(f"density must have a leading spin axis of extent 1 or 2, got {n_spin}")
        _lib.require_cuda(density, "density")
        dens = density.to(torch.float64).contiguous()
        p = dens.shape[-1]
        dev = dens.device
        stream = stream_handle(dev)
        e = torch.empty(p, dtype=torch.float64, device=dev)
        v = torch.empty((n_spin, p), dtype=torch.float64, device=dev)
        sig = None
        if self.rung >= 2:
            n_sigma = 1 if n_spin == 1 else 3
            if sigma.shape[0] != n_sigma:
                raise ValueError(f"a spin-polarised sigma has three components (uu, ud, dd), got {sigma.shape[0]}"
                                 if n_spin == 2 else f"a spin-restricted sigma has one component, got {sigma.shape[0]}")
            sig = sigma.to(torch.float64).contiguous()
        vs = None if sig is None else torch.empty_like(sig)
        if n_spin == 1 and self.name == "lda_vwn":
            call("cdftb_xc_lda_vwn_f64", ptr(dens[0]), p, ptr(e), ptr(v[0]), stream)
        elif n_spin == 1 and self.name == "pbe":
            call("cdftb_xc_pbe_f64", ptr(dens[0]), ptr(sig[0]), p, ptr(e), ptr(v[0]), ptr(vs[0]), stream)
        else:
            call("cdftb_xc_eval_f64", self.id, n_spin, ptr(dens), ptr(sig), p, ptr(e), ptr(v), ptr(vs), stream)
        return XCOutput(e, v, vs)

    def __repr__(self) -> str:
        return f"SemiLocalFunctional(name={self.name!r}, rung={self.rung})"


class LDA(SemiLocalFunctional):
    """Slater exchange + VWN5 correlation (``src/cdft/xc/lda.py:198``, dispatch name ``lda_vwn``)."""

    def __init__(self, name: str = "lda_vwn") -> None:
        super().__init__(name)


class PBE(SemiLocalFunctional):
    """PBE exchange + correlation (``src/cdft/xc/gga.py:162``, dispatch name ``pbe``)."""

    def __init__(self, name: str = "pbe") -> None:
        super().__init__(name)


def functional_by_name(name: str) -> SemiLocalFunctional:
    """A fresh native functional by its dispatch name (``src/cdft/xc/dispatch.py:50-58``)."""
    return SemiLocalFunctional(name)
