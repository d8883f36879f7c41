"""LDA (Slater + VWN5) and PBE exchange--correlation, values and first derivatives (oracle).

Restates ``src/cdft/xc/base.py`` (spin split, thresholds, empty points), ``src/cdft/xc/lda.py``
(Slater exchange, VWN5, PW92) and ``src/cdft/xc/gga.py`` (PBE exchange and correlation). The
reference differentiates its energy densities with torch autograd (``base.py:115-156``); here the
same energy expressions are evaluated on forward-mode dual numbers, so ``v_xc = de/dn`` and
``v_sigma = de/dsigma`` are exact derivatives of the restated energy density, independent of the
hand-derived formulas the CUDA kernels use.
"""

from __future__ import annotations

import math

import numpy as np

DENSITY_THRESHOLD = 1.0e-14
SIGMA_THRESHOLD = 1.0e-40


class Dual:
    """``val + eps * der`` with ``eps^2 = 0``, elementwise over numpy arrays."""

    __array_priority__ = 1000

    def __init__(self, val, der=None):
        self.val = np.asarray(val, dtype=np.float64)
        self.der = np.zeros_like(self.val) if der is None else np.asarray(der, dtype=np.float64)

    @staticmethod
    def lift(x):
        return x if isinstance(x, Dual) else Dual(x)

    def __add__(self, o):
        o = Dual.lift(o)
        return Dual(self.val + o.val, self.der + o.der)

    __radd__ = __add__

    def __sub__(self, o):
        o = Dual.lift(o)
        return Dual(self.val - o.val, self.der - o.der)

    def __rsub__(self, o):
        return Dual.lift(o) - self

    def __neg__(self):
        return Dual(-self.val, -self.der)

    def __mul__(self, o):
        o = Dual.lift(o)
        return Dual(self.val * o.val, self.der * o.val + self.val * o.der)

    __rmul__ = __mul__

    def __truediv__(self, o):
        o = Dual.lift(o)
        return Dual(self.val / o.val, (self.der * o.val - self.val * o.der) / (o.val * o.val))

    def __rtruediv__(self, o):
        return Dual.lift(o) / self

    def __pow__(self, p: float):
        return Dual(self.val ** p, p * self.val ** (p - 1.0) * self.der)


def _f(name):
    table = {
        "sqrt": (np.sqrt, lambda v: 0.5 / np.sqrt(v)),
        "log": (np.log, lambda v: 1.0 / v),
        "log1p": (np.log1p, lambda v: 1.0 / (1.0 + v)),
        "atan": (np.arctan, lambda v: 1.0 / (1.0 + v * v)),
        "exp": (np.exp, np.exp),
    }
    fn, d = table[name]

    def apply(x):
        if isinstance(x, Dual):
            return Dual(fn(x.val), d(x.val) * x.der)
        return fn(x)
    return apply


sqrt, log, log1p, atan, exp = (_f(n) for n in ("sqrt", "log", "log1p", "atan", "exp"))


def clamp_min(x, floor):
    if isinstance(x, Dual):
        keep = x.val >= floor
        return Dual(np.maximum(x.val, floor), np.where(keep, x.der, 0.0))
    return np.maximum(x, floor)


def clamp(x, lo, hi):
    if isinstance(x, Dual):
        keep = (x.val >= lo) & (x.val <= hi)
        return Dual(np.clip(x.val, lo, hi), np.where(keep, x.der, 0.0))
    return np.clip(x, lo, hi)


_SLATER = 0.75 * (3.0 / math.pi) ** (1.0 / 3.0)
_FPP0 = 4.0 / (9.0 * (2.0 ** (1.0 / 3.0) - 1.0))
_VWN5 = {
    "para": (0.0310907, -0.10498, 3.72744, 12.9352),
    "ferro": (0.01554535, -0.32500, 7.06042, 18.0578),
    "stiffness": (-1.0 / (6.0 * math.pi ** 2), -0.0047584, 1.13107, 13.0045),
}
_PW92_MOD = {
    "para": (0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294),
    "ferro": (0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517),
    "stiffness": (0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671),
}
_KF = (3.0 * math.pi ** 2) ** (1.0 / 3.0)
_PBE_KAPPA = 0.804
_PBE_MU = 0.2195149727645171
_PBE_BETA = 0.06672455060314922
_PBE_GAMMA = (1.0 - math.log(2.0)) / math.pi ** 2


def _rs(n):
    return (3.0 / (4.0 * math.pi * n)) ** (1.0 / 3.0)


def _zeta(n_up, n_dn):
    return clamp((n_up - n_dn) / (n_up + n_dn), -1.0 + 1.0e-15, 1.0 - 1.0e-15)


def _f_zeta(z):
    return ((1.0 + z) ** (4.0 / 3.0) + (1.0 - z) ** (4.0 / 3.0) - 2.0) / (2.0 ** (4.0 / 3.0) - 2.0)


def slater(n_up, n_dn):
    """``src/cdft/xc/base.py:202-210``"""
    return -(2.0 ** (1.0 / 3.0) * _SLATER) * (n_up ** (4.0 / 3.0) + n_dn ** (4.0 / 3.0))


def _vwn_aux(x, params):
    """``src/cdft/xc/lda.py:122-134``"""
    a, x0, b, c = params
    big_x = x * x + b * x + c
    big_x0 = x0 * x0 + b * x0 + c
    q = math.sqrt(4.0 * c - b * b)
    atan_term = atan(q / (2.0 * x + b))
    return a * (log(x * x / big_x) + (2.0 * b / q) * atan_term
                - (b * x0 / big_x0) * (log((x - x0) ** 2.0 / big_x) + (2.0 * (b + 2.0 * x0) / q) * atan_term))


def vwn5(n_up, n_dn):
    """``src/cdft/xc/lda.py:150-159``"""
    n = n_up + n_dn
    x = sqrt(_rs(n))
    zeta = _zeta(n_up, n_dn)
    para = _vwn_aux(x, _VWN5["para"])
    ferro = _vwn_aux(x, _VWN5["ferro"])
    alpha_c = _vwn_aux(x, _VWN5["stiffness"])
    fz = _f_zeta(zeta)
    z4 = zeta ** 4.0
    return n * (para + alpha_c * fz * (1.0 - z4) / _FPP0 + (ferro - para) * fz * z4)


def _pw92_g(rs, params):
    """``src/cdft/xc/lda.py:55-61``"""
    a, a1, b1, b2, b3, b4 = params
    s = sqrt(rs)
    den = 2.0 * a * (b1 * s + b2 * rs + b3 * rs * s + b4 * rs * rs)
    return -2.0 * a * (1.0 + a1 * rs) * log1p(1.0 / den)


def pw92_mod(rs, zeta):
    """``src/cdft/xc/lda.py:79-91`` with the modified parameter set"""
    para = _pw92_g(rs, _PW92_MOD["para"])
    ferro = _pw92_g(rs, _PW92_MOD["ferro"])
    alpha_c = -1.0 * _pw92_g(rs, _PW92_MOD["stiffness"])
    fz = _f_zeta(zeta)
    z4 = zeta ** 4.0
    return para + alpha_c * fz * (1.0 - z4) / _FPP0 + (ferro - para) * fz * z4


def pbe_x(n_up, n_dn, s_uu, s_dd):
    """``src/cdft/xc/gga.py:28-59``"""
    total = 0.0
    for n_s, sig in ((n_up, s_uu), (n_dn, s_dd)):
        n2 = 2.0 * n_s
        s2 = (4.0 * sig) / (4.0 * _KF ** 2 * n2 ** (8.0 / 3.0))
        fx = 1.0 + _PBE_KAPPA - _PBE_KAPPA / (1.0 + _PBE_MU * s2 / _PBE_KAPPA)
        total = total + 0.5 * (-_SLATER * n2 ** (4.0 / 3.0)) * fx
    return total


def pbe_c(n_up, n_dn, s_uu, s_ud, s_dd):
    """``src/cdft/xc/gga.py:73-90``"""
    n = n_up + n_dn
    rs = _rs(n)
    zeta = _zeta(n_up, n_dn)
    eps = pw92_mod(rs, zeta)
    phi = 0.5 * ((1.0 + zeta) ** (2.0 / 3.0) + (1.0 - zeta) ** (2.0 / 3.0))
    sigma = s_uu + 2.0 * s_ud + s_dd
    k_f = _KF * n ** (1.0 / 3.0)
    k_s_sq = 4.0 * k_f / math.pi
    t2 = sigma / (4.0 * phi * phi * k_s_sq * n * n)
    phi3 = phi ** 3.0
    a = (_PBE_BETA / _PBE_GAMMA) / (exp(-1.0 * eps / (_PBE_GAMMA * phi3)) - 1.0)
    at2 = a * t2
    h = _PBE_GAMMA * phi3 * log1p((_PBE_BETA / _PBE_GAMMA) * t2 * (1.0 + at2) / (1.0 + at2 + at2 * at2))
    return n * (eps + h)


def _energy(name, density, sigma):
    """Spin split, thresholds and empty points (``src/cdft/xc/base.py:45-80, 171-189``), n_spin = 1."""
    n_up = 0.5 * density
    n_dn = 0.5 * density
    total_val = (n_up + n_dn).val if isinstance(n_up, Dual) else n_up + n_dn
    empty = total_val < DENSITY_THRESHOLD
    floor = 0.5 * DENSITY_THRESHOLD
    n_up_c = clamp_min(n_up, floor)
    n_dn_c = clamp_min(n_dn, floor)
    if name == "lda_vwn":
        e = slater(n_up_c, n_dn_c) + vwn5(n_up_c, n_dn_c)
    elif name == "pbe":
        s = 0.25 * sigma
        s_c = clamp_min(s, SIGMA_THRESHOLD)
        e = pbe_x(n_up_c, n_dn_c, s_c, s_c) + pbe_c(n_up_c, n_dn_c, s_c, s, s_c)
    else:
        raise KeyError(name)
    if isinstance(e, Dual):
        return Dual(np.where(empty, 0.0, e.val), np.where(empty, 0.0, e.der))
    return np.where(empty, 0.0, e)


def evaluate(name: str, density: np.ndarray, sigma: np.ndarray | None = None):
    """``(e_xc, v_xc, v_sigma)`` for a spin-restricted density ``(P,)`` (``src/cdft/xc/base.py:115-156``)."""
    density = np.asarray(density, dtype=np.float64)
    if name == "pbe" and sigma is None:
        raise ValueError("pbe is a rung-2 functional and needs sigma")
    sig = None if sigma is None else np.asarray(sigma, dtype=np.float64)
    dn = _energy(name, Dual(density, np.ones_like(density)), sig)
    v_sigma = None
    if sig is not None:
        ds = _energy(name, density, Dual(sig, np.ones_like(sig)))
        v_sigma = ds.der
    return dn.val, dn.der, v_sigma
