"""Shared tolerance for exchange--correlation comparisons.

Energy densities and their derivatives cancel between terms (PBE's H against e_c at large reduced
gradients, LYP's terms at one nearly empty channel), so a relative tolerance on the result alone is
meaningless where the result is tiny. Each quantity is compared against the magnitude of its
terms at that density, n = n_up + n_dn: e against n^(4/3) (the exchange energy's scale), v against
n^(1/3), v_sigma against n^(-4/3). Empty points (n < 1e-14) must be exactly zero.

Device results are compared with ``DEVICE_STOL``: CUDA's ``pow``/``log``/``exp`` and the host's
libm differ by an ulp or two, and near full spin polarisation (one channel a few 1e-13 against
the other's 1) the derivative terms of (1 -/+ zeta)^(1/3) are four orders larger than the result
they cancel to, so the host-to-device difference reaches a few 1e-12 of the n^(1/3) scale there.
"""

from __future__ import annotations

import numpy as np

DEVICE_STOL = 1e-11

THRESHOLD = 1.0e-14
SCALE_POWER = {"e": 4.0 / 3.0, "v": 1.0 / 3.0, "vs": -4.0 / 3.0}


def assert_xc_close(kind: str, got, want, density, rtol: float = 1e-12, stol: float = 1e-12, what: str = ""):
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    total = np.atleast_2d(np.asarray(density, dtype=np.float64)).sum(axis=0)
    empty = total < THRESHOLD
    assert got.shape == want.shape, f"{what}: shape {got.shape} vs {want.shape}"
    assert np.all(np.isfinite(got)), f"{what}: non-finite values"
    assert np.all(got[..., empty] == 0.0), f"{what}: empty points are not exactly zero"
    scale = np.maximum(total, THRESHOLD) ** SCALE_POWER[kind]
    err = np.abs(got - want)[..., ~empty]
    bound = (rtol * np.abs(want) + stol * scale)[..., ~empty]
    worst = float(np.max(err / bound)) if err.size else 0.0
    assert worst <= 1.0, f"{what}: error {worst:.2f} x the tolerance"
