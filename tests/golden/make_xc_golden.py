"""Generate the exchange--correlation fixtures by running the reference's own functionals.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_xc_golden.py

Reads the reference checkout at ``CDFT_REFERENCE`` (default ``/root/reference``) and writes
``tests/golden/xc_fixtures.npz``: for every functional name of the reference's dispatch table
(``src/cdft/xc/dispatch.py:26-44``), ``SemiLocalFunctional.evaluate`` (energy density and autograd
derivatives, ``src/cdft/xc/base.py:115-156``) on seeded points, spin-restricted (``r_*``) and
spin-polarised (``p_*``). The points cover empty points (below the 1e-14 threshold), a channel at
zero (full polarisation), equal channels, zero gradients and reduced gradients from 1e-4 to 30.
It also records self-consistent He solves (h = 0.5, box 12, linear mixing 0.3) with the functionals
other than lda_vwn and pbe (``scf_<name>_total``, ``scf_<name>_iterations``). Nothing else reads the
reference; the tests use only the committed file.
"""

from __future__ import annotations

import math
import os
import sys
from pathlib import Path

REFERENCE = Path(os.environ.get("CDFT_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent / "xc_fixtures.npz"

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
sys.path[:0] = [str(REFERENCE), str(REFERENCE / "src")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

from cdft.xc.dispatch import NATIVE, functional_by_name  # noqa: E402

#: functionals solved self-consistently for the SCF fixtures: name -> (rung, libxc identifiers)
SCF_FUNCTIONALS = {"lda_pw92": ("LDA", ("lda_x", "lda_c_pw")), "lda_pz81": ("LDA", ("lda_x", "lda_c_pz")),
                   "blyp": ("GGA", ("gga_x_b88", "gga_c_lyp"))}


def scf_solves(out: dict) -> None:
    """He, box 12, h = 0.5, linear mixing 0.3, with each functional of ``SCF_FUNCTIONALS``."""
    import dataclasses

    from contract import MixingConfig, MixingScheme, XCRung, XCSpec
    from cdft.config import ALL_ELECTRON_NUMERICS
    from cdft.physics_config import helium
    from cdft.scf.loop import solve_self_consistent

    base = ALL_ELECTRON_NUMERICS
    num = dataclasses.replace(
        base, grid=dataclasses.replace(base.grid, spacing=0.5, box_lengths=(12.0, 12.0, 12.0)),
        eigen=dataclasses.replace(base.eigen, cross_check=False, chebyshev_degree=20, residual_tol=1e-8),
        mixing=MixingConfig(scheme=MixingScheme.LINEAR, alpha=0.3))
    for name, (rung, libxc) in SCF_FUNCTIONALS.items():
        spec = XCSpec(name=name, rung=getattr(XCRung, rung), libxc_reference=libxc)
        art = solve_self_consistent(dataclasses.replace(helium(), xc=spec), num, derive_grid=False)
        assert art.result is not None, art.error_message
        out[f"scf_{name}_total"] = np.array(art.result.energies.total)
        out[f"scf_{name}_iterations"] = np.array(art.result.n_iterations)
        print(name, art.result.energies.total, art.result.n_iterations, flush=True)

KF2 = (3.0 * math.pi ** 2) ** (2.0 / 3.0)


def _density(rng, p):
    n = 10.0 ** rng.uniform(-16.0, 2.0, p)
    n[:10] = 0.0
    n[10:20] = 1.0e-14 * rng.uniform(0.5, 2.0, 10)
    return n


def _sigma_for(rng, n):
    """|grad n|^2 from a reduced gradient s in 10^U(-4, 1.5): sigma = 4 k_F^2 n^(8/3) s^2."""
    s = 10.0 ** rng.uniform(-4.0, 1.5, n.shape[0])
    sigma = 4.0 * KF2 * n ** (8.0 / 3.0) * s * s
    sigma[20:40] = 0.0
    return sigma


def points(seed: int = 7, p: int = 600):
    rng = np.random.default_rng(seed)
    n = _density(rng, p)
    restricted = (n[None, :], _sigma_for(rng, n)[None, :])
    up = _density(rng, p)
    dn = _density(rng, p)
    dn[40:80] = 0.0               # fully polarised
    dn[80:120] = up[80:120]       # unpolarised, given as two channels
    s_uu = _sigma_for(rng, 2.0 * up) / 4.0
    s_dd = _sigma_for(rng, 2.0 * dn) / 4.0
    s_ud = rng.uniform(-1.0, 1.0, p) * np.sqrt(s_uu * s_dd)
    polarised = (np.stack([up, dn]), np.stack([s_uu, s_ud, s_dd]))
    return restricted, polarised


def main() -> None:
    restricted, polarised = points()
    out = {"r_density": restricted[0], "r_sigma": restricted[1], "p_density": polarised[0],
           "p_sigma": polarised[1]}
    for name in NATIVE:
        fn = functional_by_name(name)
        gga = fn.rung.value >= 2
        for tag, (dens, sig) in (("r", restricted), ("p", polarised)):
            res = fn.evaluate(torch.from_numpy(dens), torch.from_numpy(sig) if gga else None)
            out[f"{tag}_{name}_e"] = res.e_xc.numpy()
            out[f"{tag}_{name}_v"] = res.v_xc.numpy()
            if gga:
                out[f"{tag}_{name}_vs"] = res.v_sigma.numpy()
    out["names"] = np.array(list(NATIVE))
    scf_solves(out)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({len(NATIVE)} functionals)")


if __name__ == "__main__":
    main()
