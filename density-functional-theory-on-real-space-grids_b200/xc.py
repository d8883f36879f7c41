"""LDA (VWN) and PBE exchange--correlation on the device (host mirror of ``src/cdft/xc``).

``evaluate`` keeps the contract of ``SemiLocalFunctional.evaluate`` (``src/cdft/xc/base.py:115``):
``(n_spin, P)`` density, ``(n_sigma, P)`` sigma, a GGA without sigma and any non-local feature raise
``ValueError``. The spin-restricted case (n_spin = 1) is what the self-consistent path uses; it runs
in the library's hand-differentiated kernels.
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


class _Functional:
    rung: int = 1
    name: str = ""
    libxc_reference: tuple[str, ...] = ()

    def evaluate(self, density, sigma=None, tau=None, lapl=None, nldf=None) -> XCOutput:
        if self.rung >= 2 and sigma is None:
            raise ValueError(f"{self.name} is a rung-{self.rung} functional and needs sigma")
        if nldf is not None:
            raise ValueError(f"{self.name} is semi-local and consumes no non-local features")
        if density.shape[0] != 1:
            raise NotImplementedError("the native XC kernels are spin-restricted (n_spin = 1)")
        _lib.require_cuda(density, "density")
        n = density[0].to(torch.float64).contiguous()
        p = n.numel()
        e = torch.empty_like(n)
        v = torch.empty_like(n)
        stream = stream_handle(n.device)
        if self.rung == 1:
            call("cdftb_xc_lda_vwn_f64", ptr(n), p, ptr(e), ptr(v), stream)
            return XCOutput(e, v[None, :], None)
        s = sigma[0].to(torch.float64).contiguous()
        vs = torch.empty_like(n)
        call("cdftb_xc_pbe_f64", ptr(n), ptr(s), p, ptr(e), ptr(v), ptr(vs), stream)
        return XCOutput(e, v[None, :], vs[None, :])


class LDA(_Functional):
    """Slater exchange + VWN5 correlation (``src/cdft/xc/lda.py:201``, dispatch name ``lda_vwn``)."""

    rung = 1
    name = "lda_vwn"
    libxc_reference = ("lda_x", "lda_c_vwn")


class PBE(_Functional):
    """PBE exchange + correlation (``src/cdft/xc/gga.py:162``, dispatch name ``pbe``)."""

    rung = 2
    name = "pbe"
    libxc_reference = ("gga_x_pbe", "gga_c_pbe")


def functional_by_name(name: str) -> _Functional:
    """The native functionals (``src/cdft/xc/dispatch.py:26-62``); others raise ``KeyError``."""
    table = {"lda_vwn": LDA, "pbe": PBE}
    key = name.lower()
    if key not in table:
        raise KeyError(f"unknown or non-native functional {name!r}; native: {', '.join(table)}")
    return table[key]()
