"""The drop-in's native seam functions on the device, on objects shaped like the reference's.

The reference does not travel to the GPU box, so these tests hand the plugin's seam functions
stand-ins with the attributes its classes carry (``grid.shape/spacing/fd_order/_full_box``,
``factor.face_weights()``, ``_inverse_weight``, ``graph_potential()``, ``note_applications()``;
``CoulombCutoffPoisson``'s ``grid/pad_factor/padded_shape/cutoff_radius``; a functional's
``name/rung/libxc_reference``) and compare with the oracle and the reference's own fixtures.
"""

from __future__ import annotations

import importlib
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import eigen as oeigen
from oracle import scf as oscf
from oracle.operators import CoulombCutoffPoisson as OraclePoisson
from oracle.operators import CuspHamiltonian

from _xc_check import DEVICE_STOL, assert_xc_close

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plugin(pkg):
    return importlib.import_module("cdft_b200.plugin")


class RefLikeHamiltonian:
    """The attributes of ``cdft.operators.hamiltonian.CuspFactoredHamiltonian`` the plugin reads."""

    def __init__(self, grid, faces, inverse_weight, potential):
        self.grid = grid
        self.factor = SimpleNamespace(is_identity=False, face_weights=lambda order: faces)
        self._inverse_weight = inverse_weight
        self._potential = potential
        self._apply_count = 0

    def graph_potential(self):
        return self._potential

    def note_applications(self, count):
        self._apply_count += int(count)


@pytest.fixture(scope="module")
def he17(cuda):
    system = oscf.he_lda(spacing=0.5, edge=8.0)
    grid_o, factor_o, quad_o = oscf.build_geometry(system)
    pot, inv, q = quad_o.bare_operator_terms()
    faces = factor_o.face_weights(8)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    grid = SimpleNamespace(shape=grid_o.shape, spacing=grid_o.spacing, fd_order=8, _full_box=True,
                           origin=tuple(grid_o.origin))
    ref_like = RefLikeHamiltonian(grid, tuple(t(f) for f in faces), t(inv), t(pot))
    return ref_like, CuspHamiltonian(grid_o, factor_o, quad_o), grid_o


def test_apply_and_kinetic_apply(plugin, he17):
    ham, ham_o, grid_o = he17
    phi = np.random.default_rng(2).standard_normal((3, grid_o.n_points))
    x = torch.from_numpy(phi).to(ham._potential.device)
    out, why = plugin.native_apply(ham, x, ham._potential)
    assert why is None
    want = ham_o.apply_with_potential(phi, ham_o.potential)
    assert np.abs(out.cpu().numpy() - want).max() < 1e-12 * np.abs(want).max()
    kin, _ = plugin.native_apply(ham, x, None)
    want_k = ham_o.kinetic_apply(phi)
    assert np.abs(kin.cpu().numpy() - want_k).max() < 1e-12 * np.abs(want_k).max()
    assert torch.equal(x, torch.from_numpy(phi).to(x.device))  # inputs untouched


def test_filter_and_engine(plugin, he17):
    ham, ham_o, grid_o = he17
    block = np.random.default_rng(4).standard_normal((5, grid_o.n_points))
    x = torch.from_numpy(block).to(ham._potential.device)
    args = (12, 0.5, 40.0, -2.5)
    want = oeigen.chebyshev_filter(ham_o, block, *args)
    out, why = plugin.native_filter(ham, x, *args)
    assert why is None and ham._apply_count == 12
    assert np.abs(out.cpu().numpy() - want).max() < 1e-11 * np.abs(want).max()
    engine = plugin.graphed_filter_for(x.device)
    first = engine(ham, x, *args)  # captures, replays once and returns the direct call it checked against
    again = engine(ham, x, *args)  # a replay
    assert torch.equal(first, out) and torch.equal(again, out)
    rec = engine.record()
    assert rec["used"] and rec["replays"] == 1 and rec["captures"] == 1
    assert rec["validation_max_rel_diff"] == 0.0
    assert {"used", "captures", "replays", "eager_calls", "warmup_applications",
            "validation_max_rel_diff"} <= set(rec)
    assert plugin.graphed_filter_for(torch.device("cpu")) is None
    # an operator without the seam is refused, with the reason, so the caller runs the reference's
    assert plugin.native_filter(SimpleNamespace(), x, *args)[0] is None
    ident = RefLikeHamiltonian(ham.grid, None, ham._inverse_weight, ham._potential)
    ident.factor = SimpleNamespace(is_identity=True)
    assert plugin.native_filter(ident, x, *args)[1] == "identity cusp factor (no nuclei)"


def test_weighted_divergence_against_the_reference_fixture(plugin, cuda, golden_arrays):
    box = torch.from_numpy(golden_arrays["div_box"]).to(cuda)
    faces = tuple(torch.from_numpy(golden_arrays[f"div_w{a}"]).to(cuda) for a in range(3))
    out, why = plugin.native_weighted_divergence(box, faces, 0.37, 8, tuple(box.shape[-3:]))
    want = golden_arrays["div_out"]
    assert why is None
    assert np.abs(out.cpu().numpy() - want).max() < 1e-13 * np.abs(want).max()


def test_poisson(plugin, cuda):
    system = oscf.he_lda(spacing=0.5, edge=12.0)
    grid_o, _, _ = oscf.build_geometry(system)
    oracle = OraclePoisson(grid_o, 2.5)
    solver = SimpleNamespace(grid=SimpleNamespace(shape=grid_o.shape, spacing=grid_o.spacing, _full_box=True,
                                                  origin=tuple(grid_o.origin)),
                             pad_factor=2.5, padded_shape=oracle.padded_shape, cutoff_radius=oracle.cutoff_radius)
    rho = np.exp(-np.linalg.norm(grid_o.points(), axis=-1) ** 2)
    got, why = plugin.native_poisson(solver, torch.from_numpy(rho).to(cuda))
    want = oracle.solve(rho)
    assert why is None
    assert np.abs(got.cpu().numpy() - want).max() < 1e-12 * np.abs(want).max()
    solver.padded_shape = (1, 1, 1)
    solver.__dict__.pop("_cdftb_plan")
    assert plugin.native_poisson(solver, torch.from_numpy(rho).to(cuda))[0] is None


@pytest.mark.parametrize("name,rung,libxc", [("lda_pz81", 1, ("lda_x", "lda_c_pz")),
                                             ("blyp", 2, ("gga_x_b88", "gga_c_lyp")),
                                             ("gga_c_pbe", 2, ("gga_c_pbe",))])
def test_xc_evaluate(plugin, cuda, name, rung, libxc):
    with np.load(Path(__file__).resolve().parent / "golden" / "xc_fixtures.npz") as f:
        dens, sig = f["p_density"], f["p_sigma"]
        want_e, want_v = f[f"p_{name}_e"], f[f"p_{name}_v"]
        want_vs = f[f"p_{name}_vs"] if rung >= 2 else None
    functional = SimpleNamespace(name=name, rung=SimpleNamespace(value=rung), libxc_reference=libxc)
    out, why = plugin.native_evaluate(functional, torch.from_numpy(dens).to(cuda),
                                      torch.from_numpy(sig).to(cuda) if rung >= 2 else None, None, None, None)
    assert why is None
    assert_xc_close("e", out.e_xc.cpu().numpy(), want_e, dens)
    assert_xc_close("v", out.v_xc.cpu().numpy(), want_v, dens, stol=DEVICE_STOL)
    if rung >= 2:
        assert_xc_close("vs", out.v_sigma.cpu().numpy(), want_vs, dens, stol=DEVICE_STOL)
    mislabelled = SimpleNamespace(name=name, rung=SimpleNamespace(value=rung), libxc_reference=("lda_x",))
    assert plugin.native_evaluate(mislabelled, torch.from_numpy(dens).to(cuda), None, None, None, None)[0] is None
