"""The native semi-local functionals, values and first derivatives (oracle).

Restates ``src/cdft/xc/base.py`` (spin split, thresholds, empty points), ``src/cdft/xc/lda.py``
(Slater exchange, VWN5, PW92 in both parameter sets, PZ81), ``src/cdft/xc/gga.py`` (PBE exchange
and correlation, B88 exchange, LYP correlation) and the name table of ``src/cdft/xc/dispatch.py``,
for spin-restricted (n_spin = 1) and spin-polarised (n_spin = 2) inputs. The
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
        "asinh": (np.arcsinh, lambda v: 1.0 / np.sqrt(1.0 + v * v)),
    }
    fn, d = table[name]

    def apply(x):
        if isinstance(x, Dual):
            return Dual(fn(x.val), d(x.val) * x.der)
        return fn(x)
    return apply


sqrt, log, log1p, atan, exp, asinh = (_f(n) for n in ("sqrt", "log", "log1p", "atan", "exp", "asinh"))


def select(cond, a, b):
    """``torch.where(cond, a, b)``: the value and the derivative of the branch taken."""
    if isinstance(a, Dual) or isinstance(b, Dual):
        a, b = Dual.lift(a), Dual.lift(b)
        return Dual(np.where(cond, a.val, b.val), np.where(cond, a.der, b.der))
    return np.where(cond, a, b)


def _value(x):
    return x.val if isinstance(x, Dual) else np.asarray(x)


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


_PW92_ORIGINAL = {
    "para": (0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294),
    "ferro": (0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517),
    "stiffness": (0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671),
}
_PW92_ORIGINAL_FPP0 = 1.709921


def pw92(rs, zeta, modified: bool):
    """``src/cdft/xc/lda.py:64-91``: PW92 in the original (``LDA_C_PW``) or modified set."""
    if modified:
        return pw92_mod(rs, zeta)
    table = _PW92_ORIGINAL
    para = _pw92_g(rs, table["para"])
    ferro = _pw92_g(rs, table["ferro"])
    alpha_c = -1.0 * _pw92_g(rs, table["stiffness"])
    fz = _f_zeta(zeta)
    z4 = zeta ** 4.0
    return para + alpha_c * fz * (1.0 - z4) / _PW92_ORIGINAL_FPP0 + (ferro - para) * fz * z4


def pw92_c(n_up, n_dn, modified: bool):
    """``src/cdft/xc/lda.py:108-110``: ``n e_c(r_s, zeta)``."""
    n = n_up + n_dn
    return n * pw92(_rs(n), _zeta(n_up, n_dn), modified)


_PZ81 = {
    "para": (-0.1423, 1.0529, 0.3334, 0.0311, -0.048, 0.0020, -0.0116),
    "ferro": (-0.0843, 1.3981, 0.2611, 0.01555, -0.0269, 0.0007, -0.0048),
}


def _pz81_epsilon(rs, params):
    """``src/cdft/xc/lda.py:170-177``: the ``r_s >= 1`` Pade branch and the ``r_s < 1`` log branch."""
    gamma, beta1, beta2, a, b, c, d = params
    high = gamma / (1.0 + beta1 * sqrt(rs) + beta2 * rs)
    log_rs = log(rs)
    low = a * log_rs + b + c * rs * log_rs + d * rs
    return select(_value(rs) >= 1.0, high, low)


def pz81_c(n_up, n_dn):
    """``src/cdft/xc/lda.py:188-195``: ``n [e_U + f(zeta)(e_P - e_U)]``."""
    n = n_up + n_dn
    rs = _rs(n)
    zeta = _zeta(n_up, n_dn)
    para = _pz81_epsilon(rs, _PZ81["para"])
    ferro = _pz81_epsilon(rs, _PZ81["ferro"])
    return n * (para + _f_zeta(zeta) * (ferro - para))


_B88_BETA = 0.0042


def b88_x(n_up, n_dn, s_uu, s_dd):
    """``src/cdft/xc/gga.py:114-122``: per spin ``-C n^4/3 - beta n^4/3 x^2 / (1 + 6 beta x asinh x)``."""
    c_lda = 1.5 * (3.0 / (4.0 * math.pi)) ** (1.0 / 3.0)
    total = 0.0
    for n_s, sig in ((n_up, s_uu), (n_dn, s_dd)):
        n43 = n_s ** (4.0 / 3.0)
        x2 = sig / (n43 * n43)
        x = sqrt(x2)
        total = total - c_lda * n43 - _B88_BETA * n43 * x2 / (1.0 + 6.0 * _B88_BETA * x * asinh(x))
    return total


_LYP = (0.04918, 0.132, 0.2533, 0.349)


def lyp_c(n_up, n_dn, s_uu, s_ud, s_dd):
    """``src/cdft/xc/gga.py:139-159``: LYP in the Laplacian-free form of Miehlich et al. eq. (2)."""
    a, b, c, d = _LYP
    c_f = 0.3 * (3.0 * math.pi ** 2) ** (2.0 / 3.0)
    n = n_up + n_dn
    n_m13 = n ** (-1.0 / 3.0)
    denom = 1.0 + d * n_m13
    omega = exp(-c * n_m13) / denom * n ** (-11.0 / 3.0)
    delta = c * n_m13 + d * n_m13 / denom
    sigma = s_uu + 2.0 * s_ud + s_dd
    nab = n_up * n_dn
    first = -a * 4.0 / denom * nab / n
    bracket = (nab * (2.0 ** (11.0 / 3.0) * c_f * (n_up ** (8.0 / 3.0) + n_dn ** (8.0 / 3.0))
                      + (47.0 / 18.0 - 7.0 * delta / 18.0) * sigma
                      - (2.5 - delta / 18.0) * (s_uu + s_dd)
                      - (delta - 11.0) / 9.0 * (n_up / n * s_uu + n_dn / n * s_dd))
               - (2.0 / 3.0) * n * n * sigma
               + ((2.0 / 3.0) * n * n - n_up * n_up) * s_dd
               + ((2.0 / 3.0) * n * n - n_dn * n_dn) * s_uu)
    return first - a * b * omega * bracket


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


#: rung per name (``src/cdft/xc/dispatch.py:26-44``): 1 LDA, 2 GGA
RUNG = {
    "lda_vwn": 1, "lda_pw92": 1, "lda_pw92_mod": 1, "lda_pz81": 1, "pbe": 2, "blyp": 2,
    "lda_x": 1, "lda_c_vwn": 1, "lda_c_pw": 1, "lda_c_pw_mod": 1, "lda_c_pz": 1,
    "gga_x_pbe": 2, "gga_c_pbe": 2, "gga_x_b88": 2, "gga_c_lyp": 2,
}


def energy_density(name, n_up, n_dn, s_uu=None, s_ud=None, s_dd=None):
    """The named functional's energy per volume on clamped per-spin ingredients
    (``src/cdft/xc/dispatch.py:26-44`` name table)."""
    if name not in RUNG:
        raise KeyError(f"unknown functional {name!r}")
    forms = {
        "lda_x": lambda: slater(n_up, n_dn),
        "lda_c_vwn": lambda: vwn5(n_up, n_dn),
        "lda_c_pw": lambda: pw92_c(n_up, n_dn, False),
        "lda_c_pw_mod": lambda: pw92_c(n_up, n_dn, True),
        "lda_c_pz": lambda: pz81_c(n_up, n_dn),
        "lda_vwn": lambda: slater(n_up, n_dn) + vwn5(n_up, n_dn),
        "lda_pw92": lambda: slater(n_up, n_dn) + pw92_c(n_up, n_dn, False),
        "lda_pw92_mod": lambda: slater(n_up, n_dn) + pw92_c(n_up, n_dn, True),
        "lda_pz81": lambda: slater(n_up, n_dn) + pz81_c(n_up, n_dn),
        "gga_x_pbe": lambda: pbe_x(n_up, n_dn, s_uu, s_dd),
        "gga_c_pbe": lambda: pbe_c(n_up, n_dn, s_uu, s_ud, s_dd),
        "gga_x_b88": lambda: b88_x(n_up, n_dn, s_uu, s_dd),
        "gga_c_lyp": lambda: lyp_c(n_up, n_dn, s_uu, s_ud, s_dd),
        "pbe": lambda: pbe_x(n_up, n_dn, s_uu, s_dd) + pbe_c(n_up, n_dn, s_uu, s_ud, s_dd),
        "blyp": lambda: b88_x(n_up, n_dn, s_uu, s_dd) + lyp_c(n_up, n_dn, s_uu, s_ud, s_dd),
    }
    return forms[name]()


def _split(density, sigma):
    """``split_spin`` (``src/cdft/xc/base.py:45-80``): rows -> the five per-spin ingredients."""
    if len(density) == 1:
        n_up = n_dn = 0.5 * density[0]
        s = None if sigma is None else 0.25 * sigma[0]
        return n_up, n_dn, s, s, s
    if len(density) != 2:
        raise ValueError(f"density must have a leading spin axis of extent 1 or 2, got {len(density)}")
    if sigma is None:
        return density[0], density[1], None, None, None
    if len(sigma) != 3:
        raise ValueError(f"a spin-polarised sigma has three components (uu, ud, dd), got {len(sigma)}")
    return density[0], density[1], sigma[0], sigma[1], sigma[2]


def _energy_rows(name, density, sigma):
    """Spin split, thresholds and empty points (``src/cdft/xc/base.py:171-189``) on rows that may
    hold one dual component."""
    n_up, n_dn, s_uu, s_ud, s_dd = _split(density, sigma)
    empty = _value(n_up + n_dn) < DENSITY_THRESHOLD
    floor = 0.5 * DENSITY_THRESHOLD
    n_up_c = clamp_min(n_up, floor)
    n_dn_c = clamp_min(n_dn, floor)
    clamp_s = lambda x: None if x is None else clamp_min(x, SIGMA_THRESHOLD)  # noqa: E731
    e = energy_density(name, n_up_c, n_dn_c, clamp_s(s_uu), s_ud, clamp_s(s_dd))
    if isinstance(e, Dual):
        return Dual(np.where(empty, 0.0, e.val), np.where(empty, 0.0, e.der))
    return np.where(empty, 0.0, e)


def evaluate_spin(name: str, density, sigma=None):
    """``(e_xc (P,), v_xc (n_spin, P), v_sigma (n_sigma, P) | None)`` for contract-shaped inputs:
    ``density (n_spin, P)``, ``sigma (1 or 3, P)`` (``src/cdft/xc/base.py:115-156``). Each derivative
    is one forward-mode pass seeded on one input row."""
    if name not in RUNG:
        raise KeyError(f"unknown functional {name!r}")
    rows = [np.asarray(r, dtype=np.float64) for r in np.atleast_2d(np.asarray(density, dtype=np.float64))]
    sig = None if sigma is None else [np.asarray(r, dtype=np.float64)
                                      for r in np.atleast_2d(np.asarray(sigma, dtype=np.float64))]
    if RUNG[name] >= 2 and sig is None:
        raise ValueError(f"{name} is a rung-{RUNG[name]} functional and needs sigma")
    if RUNG[name] == 1:
        sig = None

    def seeded(which, k):
        """The derivative along one input row (zero where the energy does not depend on it)."""
        d = [Dual(r, np.ones_like(r)) if which == "n" and i == k else r for i, r in enumerate(rows)]
        s = sig if which != "s" else [Dual(r, np.ones_like(r)) if i == k else r for i, r in enumerate(sig)]
        out = _energy_rows(name, d, s)
        return out.der if isinstance(out, Dual) else np.zeros_like(rows[0])

    e = _energy_rows(name, rows, sig)
    v = np.stack([seeded("n", k) for k in range(len(rows))])
    vs = None if sig is None else np.stack([seeded("s", k) for k in range(len(sig))])
    return np.asarray(e, dtype=np.float64), v, vs


def evaluate(name: str, density: np.ndarray, sigma: np.ndarray | None = None):
    """``(e_xc, v_xc, v_sigma)`` for a spin-restricted density ``(P,)`` (``src/cdft/xc/base.py:115-156``)."""
    density = np.asarray(density, dtype=np.float64)
    if RUNG.get(name, 0) >= 2 and sigma is None:
        raise ValueError(f"{name} is a rung-2 functional and needs sigma")
    e, v, vs = evaluate_spin(name, density[None, :], None if sigma is None else np.asarray(sigma)[None, :])
    return e, v[0], None if vs is None else vs[0]
