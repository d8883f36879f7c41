"""The oracle's functionals against the reference's own: every name of the dispatch table,
spin-restricted and spin-polarised, energy densities and autograd derivatives
(``tests/golden/xc_fixtures.npz``, written by ``make_xc_golden.py``)."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from oracle import xc as oxc

from _xc_check import assert_xc_close

FIXTURES = Path(__file__).resolve().parent / "golden" / "xc_fixtures.npz"


@pytest.fixture(scope="module")
def xc_golden():
    with np.load(FIXTURES) as data:
        return {k: data[k] for k in data.files}


def test_every_dispatch_name_is_covered(xc_golden):
    assert sorted(str(n) for n in xc_golden["names"]) == sorted(oxc.RUNG)


@pytest.mark.parametrize("tag", ["r", "p"], ids=["restricted", "polarised"])
@pytest.mark.parametrize("name", sorted(oxc.RUNG))
def test_oracle_matches_the_reference(xc_golden, name, tag):
    dens = xc_golden[f"{tag}_density"]
    sig = xc_golden[f"{tag}_sigma"] if oxc.RUNG[name] >= 2 else None
    e, v, vs = oxc.evaluate_spin(name, dens, sig)
    assert_xc_close("e", e, xc_golden[f"{tag}_{name}_e"], dens, what=f"{name} e")
    assert_xc_close("v", v, xc_golden[f"{tag}_{name}_v"], dens, what=f"{name} v")
    if sig is not None:
        assert_xc_close("vs", vs, xc_golden[f"{tag}_{name}_vs"], dens, what=f"{name} v_sigma")


def test_polarised_equal_channels_are_the_restricted_functional():
    """n_up = n_dn = n/2 and sigma_uu = sigma_ud = sigma_dd = sigma/4 given as two channels give the
    restricted energy, and the per-channel potentials equal the restricted one."""
    rng = np.random.default_rng(3)
    n = 10.0 ** rng.uniform(-6, 1, 200)
    sigma = 10.0 ** rng.uniform(-8, 2, 200)
    for name, rung in oxc.RUNG.items():
        sig_r = sigma[None] if rung >= 2 else None
        sig_p = np.stack([sigma / 4] * 3) if rung >= 2 else None
        e_r, v_r, vs_r = oxc.evaluate_spin(name, n[None], sig_r)
        e_p, v_p, vs_p = oxc.evaluate_spin(name, np.stack([n / 2, n / 2]), sig_p)
        np.testing.assert_allclose(e_p, e_r, rtol=1e-13, atol=1e-300)
        np.testing.assert_allclose(v_p[0], v_r[0], rtol=1e-11)
        np.testing.assert_allclose(v_p[1], v_r[0], rtol=1e-11)
        if rung >= 2:
            # d/dsigma of the restricted energy = (g_uu + g_ud + g_dd) / 4
            np.testing.assert_allclose(vs_p.sum(axis=0) / 4, vs_r[0], rtol=1e-10)


def test_errors_follow_the_reference():
    with pytest.raises(ValueError, match="needs sigma"):
        oxc.evaluate_spin("blyp", np.ones((1, 3)))
    with pytest.raises(ValueError, match="leading spin axis"):
        oxc.evaluate_spin("lda_vwn", np.ones((3, 3)))
    with pytest.raises(ValueError, match="three components"):
        oxc.evaluate_spin("pbe", np.ones((2, 3)), np.ones((2, 3)))
    with pytest.raises(KeyError):
        oxc.evaluate_spin("r2scan", np.ones((1, 3)))


def test_oracle_scf_with_pz81_matches_the_reference():
    """The oracle's SCF with a functional other than lda_vwn / pbe (He, box 12, h = 0.5)."""
    from oracle import scf as oscf

    with np.load(FIXTURES) as data:
        total = float(data["scf_lda_pz81_total"])
        iterations = int(data["scf_lda_pz81_iterations"])
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    system.functional = "lda_pz81"
    out = oscf.solve_self_consistent(system)
    assert out["scf_iterations"] == iterations
    assert abs(out["energies"]["total"] - total) < 1e-10
