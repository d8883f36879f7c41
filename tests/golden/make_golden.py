"""Generate the golden fixtures by running the reference solver ``cdft`` itself.

Run where the reference checkout is readable (``CDFT_REFERENCE``, default ``/root/reference``):

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py [--with-65]

Writes ``tests/golden/reference_fixtures.npz`` (small arrays) and
``tests/golden/reference_values.json`` (scalars). Nothing else reads the reference; the GPU tests and
the benchmark use only these committed files. ``--with-65`` adds the He-LDA 65^3 end-to-end solve
(about two minutes on eight cores).
"""

from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys
import time
from pathlib import Path

REFERENCE = Path(os.environ.get("CDFT_REFERENCE", "/root/reference"))  # the reference checkout (read only)
OUT = Path(__file__).resolve().parent

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
sys.path[:0] = [str(REFERENCE), str(REFERENCE / "src")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

from contract import BoundaryMode, DomainMode, GridConfig, MixingConfig, MixingScheme  # noqa: E402
from cdft.config import ALL_ELECTRON_NUMERICS  # noqa: E402
from cdft.eigen.chefsi import chebyshev_coefficients, chebyshev_filter  # noqa: E402
from cdft.eigen.rayleigh_ritz import rayleigh_ritz, residual_norms  # noqa: E402
from cdft.grid import UniformGrid  # noqa: E402
from cdft.operators.cusp import CuspFactor  # noqa: E402
from cdft.operators.divergence import _weighted_divergence_eager, staggered_coefficients  # noqa: E402
from cdft.operators.hamiltonian import CuspFactoredHamiltonian  # noqa: E402
from cdft.operators.laplacian import fd_coefficients  # noqa: E402
from cdft.operators.poisson import CoulombCutoffPoisson  # noqa: E402
from cdft.operators.quadrature import CuspQuadrature  # noqa: E402
from cdft.physics_config import REGISTRY, h2_plus, helium, hydrogen_molecule, lda_functional, pbe_functional  # noqa: E402
from cdft.scf.loop import build_interacting_step, initial_density, solve_self_consistent  # noqa: E402
from cdft.scf.noninteracting import solve_noninteracting  # noqa: E402
from cdft.xc.dispatch import functional_by_name  # noqa: E402

torch.set_num_threads(os.cpu_count() or 1)


def numerics(spacing, box, degree=20, mixing=None, residual_tol=1e-8):
    base = ALL_ELECTRON_NUMERICS
    out = dataclasses.replace(
        base,
        grid=dataclasses.replace(base.grid, spacing=spacing, box_lengths=tuple(box)),
        eigen=dataclasses.replace(base.eigen, cross_check=False, chebyshev_degree=degree, residual_tol=residual_tol),
    )
    if mixing is not None:
        out = dataclasses.replace(out, mixing=mixing)
    return out


LINEAR = MixingConfig(scheme=MixingScheme.LINEAR, alpha=0.3)
# config 4's scan is R = 0.8 + k * 5.2 / 47, k = 0..47; these are five of its members
SCAN_SAMPLES = tuple(0.8 + k * 5.2 / 47 for k in (0, 11, 23, 35, 47))
PROBE_SEED = 1234


def probe(n):
    g = torch.Generator().manual_seed(PROBE_SEED)
    return torch.randn(n, dtype=torch.float64, generator=g)


def checks(t: torch.Tensor) -> list[float]:
    """Size-independent summaries of a field: sum, sum of squares, dot with the seeded probe."""
    flat = t.reshape(-1).to(torch.float64)
    return [float(flat.sum()), float((flat * flat).sum()), float((flat * probe(flat.numel())).sum())]


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--with-65", action="store_true")
    parser.add_argument("--with-config3", action="store_true", help="H2 PBE at 81 x 81 x 91 (tens of minutes)")
    parser.add_argument("--with-scan", action="store_true", help="five members of the H2+ bond scan")
    parser.add_argument("--with-adjoint", action="store_true", help="Hellmann-Feynman and nuclear-gradient references")
    args = parser.parse_args()
    arrays: dict[str, np.ndarray] = {}
    values: dict[str, object] = {}

    # -- coefficients (divergence.py:31, laplacian.py:36)
    for acc in (2, 4, 6, 8):
        arrays[f"staggered_{acc}"] = np.array(staggered_coefficients(acc))
    arrays["fd1_8"] = np.array(fd_coefficients(1, 8))

    # -- (a1) the eager divergence on (9, 11, 13), h = 0.37, order 8, batch 2
    g = torch.Generator().manual_seed(3)
    shape = (9, 11, 13)
    box = torch.randn((2, *shape), dtype=torch.float64, generator=g)
    faces = []
    for axis in range(3):
        sizes = list(shape)
        sizes[axis] += 8
        faces.append(0.1 + torch.rand(sizes, dtype=torch.float64, generator=g))
    out = _weighted_divergence_eager(box, tuple(faces), 0.37, 8, shape)
    arrays["div_box"] = box.numpy()
    for axis in range(3):
        arrays[f"div_w{axis}"] = faces[axis].numpy()
    arrays["div_out"] = out.numpy()

    # -- He h = 0.5, box 12 (25^3) geometry, operator, filter, RR, Poisson, potentials
    scenario = dataclasses.replace(helium(), xc=lda_functional("vwn"))
    num = numerics(0.5, (12.0, 12.0, 12.0), mixing=LINEAR)
    grid, step = build_interacting_step(scenario, num, derive_grid=False)
    factor, quad = step.factor, step.quadrature
    he = {}
    he["shape"] = list(grid.shape)
    he["origin"] = list(grid.origin)
    he["n_nodes"] = quad.n_nodes
    he["f2_grid"] = checks(factor.weight)
    he["grad_u"] = checks(factor.grad_u)
    he["transformed_potential"] = checks(factor.transformed_potential)
    for axis, w in enumerate(factor.face_weights(8)):
        he[f"face_{axis}"] = checks(w)
    he["node_points"] = checks(quad.points)
    he["node_weights"] = checks(quad.weights)
    he["node_partition"] = checks(quad.partition)
    he["node_f2"] = checks(quad.f2)
    he["far"] = checks(quad.far)
    he["mass_weights"] = checks(quad.mass_weights)
    potential, inverse_weight, measure = quad.bare_operator_terms()
    he["bare_potential"] = checks(potential)
    he["inverse_weight"] = checks(inverse_weight)
    arrays["he25_mass_weights"] = quad.mass_weights.numpy()
    arrays["he25_bare_potential"] = potential.numpy()
    arrays["he25_W"] = factor.transformed_potential.numpy()

    ham = CuspFactoredHamiltonian(grid, factor, quadrature=quad)
    gen = torch.Generator().manual_seed(11)
    block = torch.randn((5, grid.n_points), dtype=torch.float64, generator=gen)
    applied = ham.apply(block)
    he["apply_rows"] = [checks(applied[i]) for i in range(5)]
    arrays["he25_apply_sub"] = applied[:, ::97].numpy()
    gen = torch.Generator().manual_seed(0)
    lo, hi = ham.spectral_bounds(generator=gen)
    he["lanczos_bounds"] = [lo, hi]
    evals, vectors, orth = rayleigh_ritz(ham, block, ham.measure)
    he["rr_evals"] = evals.tolist()
    he["rr_orth"] = float(orth)
    res = residual_norms(ham, evals, vectors, ham.measure)
    he["rr_residuals"] = res.tolist()
    lower = float(evals[-1])
    filtered = chebyshev_filter(ham, block, 20, lower, hi, lo)
    he["filter_rows"] = [checks(filtered[i]) for i in range(5)]
    he["filter_args"] = [20, lower, hi, lo]
    he["cheb_rows"] = [list(r) for r in chebyshev_coefficients(20, lower, hi, lo)]

    poisson = CoulombCutoffPoisson(grid, pad_factor=2.5)
    pts = grid.points()
    rsq = (pts * pts).sum(dim=-1)
    gauss = torch.exp(-rsq / (2 * 1.2 ** 2)) / ((2 * np.pi) ** 1.5 * 1.2 ** 3)
    vpois = poisson.solve(gauss)
    he["poisson_padded_shape"] = list(poisson.padded_shape)
    he["poisson"] = checks(vpois)
    arrays["he25_poisson_sub"] = vpois[::13].numpy()

    n0 = initial_density(step)
    arrays["he25_initial_density_sub"] = n0[0, ::13].numpy()
    he["initial_density"] = checks(n0)
    pots = step.potentials(n0)
    he["hartree_energy"] = float(pots.hartree_energy)
    he["xc_energy"] = float(pots.xc_energy)
    he["xc_double_counting"] = float(pots.xc_double_counting)
    he["effective"] = checks(pots.effective)
    he["v_hartree"] = checks(pots.v_hartree)
    arrays["he25_effective_sub"] = pots.effective[::13].numpy()
    values["he25"] = he

    # -- (d) XC pointwise, LDA and PBE
    gen = torch.Generator().manual_seed(5)
    n = 10.0 ** (torch.rand(3000, dtype=torch.float64, generator=gen) * 18.0 - 16.0)
    n[:5] = torch.tensor([0.0, 1e-15, 0.99e-14, 1.0e-14, 2e-14], dtype=torch.float64)
    sigma = (10.0 ** (torch.rand(3000, dtype=torch.float64, generator=gen) * 8.0 - 6.0)) * n ** (8.0 / 3.0)
    sigma[5:10] = 0.0
    arrays["xc_n"] = n.numpy()
    arrays["xc_sigma"] = sigma.numpy()
    lda = functional_by_name("lda_vwn").evaluate(n[None, :])
    arrays["xc_lda_e"] = lda.e_xc.numpy()
    arrays["xc_lda_v"] = lda.v_xc[0].numpy()
    pbe = functional_by_name("pbe").evaluate(n[None, :], sigma[None, :])
    arrays["xc_pbe_e"] = pbe.e_xc.numpy()
    arrays["xc_pbe_v"] = pbe.v_xc[0].numpy()
    arrays["xc_pbe_vs"] = pbe.v_sigma[0].numpy()

    # -- operator identities pinned by the reference's own golden values (tests/golden/values.json)
    pins = json.loads((REFERENCE / "tests/golden/values.json").read_text())
    values["reference_pins"] = {k: pins[k]["value"] for k in (
        "eigenvalue.ground.h_atom", "kinetic.h_atom", "eigenvalue.ground.he_plus", "kinetic.he_plus",
        "checkerboard.rayleigh.Z1", "checkerboard.rayleigh.Z2")}

    # -- end to end
    def timed(label, fn):
        t = time.perf_counter()
        art = fn()
        dt = time.perf_counter() - t
        assert art.result is not None, art.error_message
        rec = {
            "total": art.result.energies.total,
            "kinetic": art.result.energies.kinetic,
            "hartree": art.result.energies.hartree,
            "xc": art.result.energies.xc,
            "eigenvalues": art.result.eigenvalues[0].tolist(),
            "iterations": art.result.n_iterations,
            "applications": art.measurements.get("hamiltonian_applications"),
            "converged": bool(art.result.converged),
            "wall_s": dt,
            "threads": torch.get_num_threads(),
        }
        print(label, rec, flush=True)
        values[label] = rec

    timed("he25_lda_linear", lambda: solve_self_consistent(scenario, num, derive_grid=False))
    # config 1: bare H, 33^3, box 8 (h = 0.25), nucleus on the lattice
    hs = REGISTRY["h_atom"]
    timed("h33_box8", lambda: solve_noninteracting(hs, numerics(0.25, (8.0, 8.0, 8.0)), derive_grid=False))
    # the reference's golden-pin grid for H: box 32, h = 1.0
    timed("h33_box32", lambda: solve_noninteracting(hs, numerics(1.0, (32.0, 32.0, 32.0)), derive_grid=False))
    # H2+ R = 2 on a small box (two-centre quadrature, lumped far weights), h = 0.4
    timed("h2plus_R2_h04", lambda: solve_noninteracting(h2_plus(2.0), numerics(0.4, (10.0, 10.0, 12.0)), derive_grid=False))
    # H2 PBE on a small box, h = 0.4
    h2 = dataclasses.replace(hydrogen_molecule(1.4), xc=pbe_functional())
    timed("h2_pbe_h04", lambda: solve_self_consistent(h2, numerics(0.4, (10.0, 10.0, 11.2), degree=16), derive_grid=False))
    if args.with_65:
        timed("he65_lda_linear", lambda: solve_self_consistent(scenario, numerics(0.25, (16.0, 16.0, 16.0), mixing=LINEAR), derive_grid=False))
    if args.with_adjoint:
        # Hellmann--Feynman gradient of the He 25^3 energy with respect to eight seeded Gaussians
        # g_k = exp(-|r - c_k|^2 / (2 w_k^2)) (the seeding of adjoint.seeded_gaussians), from the
        # reference's converged density through its own quadrature (effective_potential,
        # quadrature.py:747-753): dE/d alpha_k = sum_grid dv_k * mass_weights * n / f^2.
        rng = np.random.default_rng(2024)
        centres = rng.uniform(-3.0, 3.0, size=(8, 3))
        widths = rng.uniform(0.5, 1.5, size=8)
        art = solve_self_consistent(scenario, num, derive_grid=False)
        density = art.result.density.reshape(-1).to(torch.float64)
        c = torch.tensor(centres, dtype=torch.float64)
        w = torch.tensor(widths, dtype=torch.float64)

        def gauss(points):
            d2 = ((points[None, :, :] - c[:, None, :]) ** 2).sum(dim=-1)
            return torch.exp(-d2 / (2.0 * w[:, None] ** 2))

        g_node, g_grid = gauss(quad.points), gauss(grid.points())
        rho = density / factor.weight
        hf = [float((quad.effective_potential(g_node[k], g_grid[k]) * quad.mass_weights * rho).sum()) for k in range(8)]
        values["he25_external_gradient"] = {"centres": centres.tolist(), "widths": widths.tolist(),
                                            "hellmann_feynman": hf, "total": art.result.energies.total}
        print("he25_external_gradient", hf, flush=True)
        # H2+ (R = 2, h = 0.4): the bond-length derivative by central differences (1e-4 bohr)
        energies = {}
        for sign in (+1, -1):
            art = solve_noninteracting(h2_plus(2.0 + sign * 1e-4), numerics(0.4, (10.0, 10.0, 12.0)),
                                       derive_grid=False)
            energies[sign] = art.result.energies.total
        values["h2plus_R2_h04_bond_derivative"] = {"plus": energies[1], "minus": energies[-1],
                                                   "derivative": (energies[1] - energies[-1]) / 2e-4}
        print("h2plus bond derivative", values["h2plus_R2_h04_bond_derivative"], flush=True)
    if args.with_config3:
        # config 3: H2 (R = 1.4) PBE, box 16 x 16 x 18, h = 0.20 -> 81 x 81 x 91, degree 16, unanchored lattice
        timed("h2_pbe_h020", lambda: solve_self_consistent(h2, numerics(0.20, (16.0, 16.0, 18.0), degree=16),
                                                          derive_grid=False))
    if args.with_scan:
        # config 4 samples: bare H2+ at R in [0.8, 6.0], box (12, 12, R + 12), h = 0.25
        for bond in SCAN_SAMPLES:
            timed(f"h2plus_scan_R{bond:.4f}", lambda b=bond: solve_noninteracting(
                h2_plus(b), numerics(0.25, (12.0, 12.0, b + 12.0)), derive_grid=False))

    np.savez_compressed(OUT / "reference_fixtures.npz", **arrays)
    old = {}
    path = OUT / "reference_values.json"
    if path.exists():
        old = json.loads(path.read_text())
    old.update(values)
    path.write_text(json.dumps(old, indent=1, sort_keys=True))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
