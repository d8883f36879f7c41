"""Every native functional on the device (``cdftb_xc_eval_f64`` and the two fused restricted kernels)
against the reference's own autograd values and the oracle, spin-restricted and spin-polarised; and
self-consistent He solves with the functionals other than lda_vwn and pbe against the reference's."""

from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import scf as oscf
from oracle import xc as oxc

from _xc_check import DEVICE_STOL, assert_xc_close

pytestmark = pytest.mark.gpu

FIXTURES = Path(__file__).resolve().parent / "golden" / "xc_fixtures.npz"


@pytest.fixture(scope="module")
def xc_golden():
    with np.load(FIXTURES) as data:
        return {k: data[k] for k in data.files}


def _np(t):
    return None if t is None else t.detach().cpu().numpy()


@pytest.mark.parametrize("tag", ["r", "p"], ids=["restricted", "polarised"])
@pytest.mark.parametrize("name", sorted(oxc.RUNG))
def test_device_functional_matches_the_reference(pkg, cuda, xc_golden, name, tag):
    dens = xc_golden[f"{tag}_density"]
    gga = oxc.RUNG[name] >= 2
    sig = xc_golden[f"{tag}_sigma"] if gga else None
    fn = pkg.functional_by_name(name)
    out = fn.evaluate(torch.from_numpy(dens).to(cuda), None if sig is None else torch.from_numpy(sig).to(cuda))
    torch.cuda.synchronize()
    e, v, vs = _np(out.e_xc), _np(out.v_xc), _np(out.v_sigma)
    assert_xc_close("e", e, xc_golden[f"{tag}_{name}_e"], dens, what=f"{name} e")
    assert_xc_close("v", v, xc_golden[f"{tag}_{name}_v"], dens, stol=DEVICE_STOL, what=f"{name} v")
    oe, ov, ovs = oxc.evaluate_spin(name, dens, sig)
    assert_xc_close("e", e, oe, dens, what=f"{name} e vs oracle")
    assert_xc_close("v", v, ov, dens, stol=DEVICE_STOL, what=f"{name} v vs oracle")
    if gga:
        assert_xc_close("vs", vs, xc_golden[f"{tag}_{name}_vs"], dens, stol=DEVICE_STOL, what=f"{name} v_sigma")
        assert_xc_close("vs", vs, ovs, dens, stol=DEVICE_STOL, what=f"{name} v_sigma vs oracle")
    else:
        assert vs is None


@pytest.mark.parametrize("name,fid", [("lda_vwn", 0), ("pbe", 4)])
def test_general_kernel_agrees_with_the_fused_kernels(pkg, cuda, xc_golden, name, fid):
    """The dual-number kernel and the hand-differentiated restricted kernels give the same values."""
    dens = torch.from_numpy(xc_golden["r_density"]).to(cuda)
    sig = torch.from_numpy(xc_golden["r_sigma"]).to(cuda) if fid == 4 else None
    fused = pkg.functional_by_name(name).evaluate(dens, sig)
    lib = pkg._lib
    p = dens.shape[-1]
    e = torch.empty(p, dtype=torch.float64, device=cuda)
    v = torch.empty((1, p), dtype=torch.float64, device=cuda)
    vs = torch.empty((1, p), dtype=torch.float64, device=cuda) if sig is not None else None
    lib.call("cdftb_xc_eval_f64", fid, 1, lib.ptr(dens), lib.ptr(sig), p, lib.ptr(e), lib.ptr(v), lib.ptr(vs),
             lib.stream_handle(cuda))
    d = xc_golden["r_density"]
    assert_xc_close("e", _np(e), _np(fused.e_xc), d, what="e")
    assert_xc_close("v", _np(v), _np(fused.v_xc), d, what="v")
    if sig is not None:
        assert_xc_close("vs", _np(vs), _np(fused.v_sigma), d, what="v_sigma")


def test_argument_errors(pkg, cuda):
    fn = pkg.functional_by_name("blyp")
    x = torch.ones((1, 4), dtype=torch.float64, device=cuda)
    with pytest.raises(ValueError, match="needs sigma"):
        fn.evaluate(x)
    with pytest.raises(ValueError, match="three components"):
        fn.evaluate(torch.ones((2, 4), dtype=torch.float64, device=cuda), x)
    with pytest.raises(ValueError, match="leading spin axis"):
        pkg.functional_by_name("lda_pz81").evaluate(torch.ones((3, 4), dtype=torch.float64, device=cuda))
    with pytest.raises(ValueError, match="non-local"):
        pkg.functional_by_name("lda_x").evaluate(x, nldf=x)
    with pytest.raises(KeyError):
        pkg.functional_by_name("r2scan")
    lib = pkg._lib.library()
    assert lib.cdftb_xc_is_gga(5) == 1 and lib.cdftb_xc_is_gga(3) == 0 and lib.cdftb_xc_is_gga(15) == -1
    assert lib.cdftb_xc_eval_f64(4, 1, None, None, 4, None, None, None, None) != 0


@pytest.fixture(scope="module")
def he25(pkg, cuda):
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=cuda)
    return pkg.build_cusp_geometry(grid, system.charges, system.positions)


@pytest.mark.parametrize("name", ["lda_pw92", "lda_pz81", "blyp"])
def test_he25_scf_other_functionals(pkg, he25, xc_golden, name):
    """He, box 12, h = 0.5, linear mixing 0.3: the reference's energy and iteration count."""
    step = pkg.KohnShamStep(he25, name, 2.0)
    out = pkg.solve_self_consistent(step, pkg.MixingConfig(scheme="linear", alpha=0.3))
    assert out.converged
    assert out.scf_iterations == int(xc_golden[f"scf_{name}_iterations"])
    assert abs(out.energies["total"] - float(xc_golden[f"scf_{name}_total"])) < 1e-10
