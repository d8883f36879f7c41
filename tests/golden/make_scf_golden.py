"""Generate the SCF-driver fixtures by running the reference solver itself.

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_scf_golden.py

Reads the reference checkout at ``CDFT_REFERENCE`` (default ``/root/reference``) and writes
``tests/golden/scf_fixtures.npz``:

- ``kerker_*``: the reference's ``KerkerPreconditioner`` (``src/cdft/scf/mixing.py:35-56``) applied
  to two seeded residual rows on an uneven box (18 x 19 x 21 points, h = 0.4, q0 = 1.5);
- ``lobpcg_*``: the reference's LOBPCG (``src/cdft/eigen/lobpcg.py``) on the bare H atom (box 8,
  h = 0.5, the nucleus on the lattice), one state and two states, seeded 1: eigenvalues and
  iteration counts; and its two-solver check inside ``solve_noninteracting(cross_check=True)``;
- ``scf_kerker_*`` / ``scf_linear_kerker_*``: He (box 12, h = 0.5) solved with the Kerker scheme
  (periodic Pulay + Kerker, q0 = 0.5) and with linear mixing alpha 0.3 plus ``kerker=True``
  (q0 = 1.5): total energy and SCF iteration count.

Nothing else reads the reference; the tests use only the committed file.
"""

from __future__ import annotations

import dataclasses
import os
import sys
from pathlib import Path

REFERENCE = Path(os.environ.get("CDFT_REFERENCE", "/root/reference"))
OUT = Path(__file__).resolve().parent / "scf_fixtures.npz"

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
sys.path[:0] = [str(REFERENCE), str(REFERENCE / "src")]

import numpy as np  # noqa: E402
import torch  # noqa: E402

from contract import MixingConfig, MixingScheme  # noqa: E402
from cdft.config import ALL_ELECTRON_NUMERICS  # noqa: E402
from cdft.physics_config import helium, lda_functional  # noqa: E402
from cdft.scf.loop import build_interacting_step, solve_self_consistent  # noqa: E402
from cdft.scf.mixing import KerkerPreconditioner  # noqa: E402
from cdft.eigen.lobpcg import LOBPCG  # noqa: E402
from cdft.physics_config import REGISTRY  # noqa: E402
from cdft.scf.noninteracting import build_hamiltonian, solve_noninteracting  # noqa: E402

torch.set_num_threads(os.cpu_count() or 1)


def numerics(spacing, box, mixing=None):
    base = ALL_ELECTRON_NUMERICS
    out = dataclasses.replace(
        base, grid=dataclasses.replace(base.grid, spacing=spacing, box_lengths=tuple(box)),
        eigen=dataclasses.replace(base.eigen, cross_check=False, chebyshev_degree=20, residual_tol=1e-8))
    return out if mixing is None else dataclasses.replace(out, mixing=mixing)


def main() -> None:
    out = {}
    scenario = dataclasses.replace(helium(), xc=lda_functional("vwn"))
    grid, _ = build_interacting_step(scenario, numerics(0.4, (6.8, 7.2, 8.0)), derive_grid=False)
    gen = torch.Generator().manual_seed(21)
    residual = torch.randn((2, grid.n_points), dtype=torch.float64, generator=gen)
    pre = KerkerPreconditioner(grid, 1.5)
    out["kerker_shape"] = np.array(grid.shape)
    out["kerker_spacing"] = np.array(grid.spacing)
    out["kerker_residual"] = residual.numpy()
    out["kerker_out"] = pre(residual).numpy()
    print("kerker grid", grid.shape, grid.spacing, flush=True)
    h_atom = REGISTRY["h_atom"]
    num_h = numerics(0.5, (8.0, 8.0, 8.0))
    _, ham, _ = build_hamiltonian(h_atom, num_h, torch.device("cpu"), derive_grid=False)
    for k in (1, 2):
        second = LOBPCG(ham.grid, num_h.eigen).solve(ham, k, generator=torch.Generator(device="cpu").manual_seed(1))
        out[f"lobpcg_{k}_eigenvalues"] = second.eigenvalues.numpy()
        out[f"lobpcg_{k}_iterations"] = np.array(second.n_iterations)
        out[f"lobpcg_{k}_converged"] = np.array(bool(second.converged))
        print("lobpcg", k, second.eigenvalues.tolist(), second.n_iterations, flush=True)
    art = solve_noninteracting(h_atom, num_h, cross_check=True, derive_grid=False)
    for key in ("two_solver_max_delta", "lobpcg_iterations"):
        out[f"cross_{key}"] = np.array(art.measurements[key])
    out["cross_eigenvalue"] = art.result.eigenvalues.reshape(-1).numpy()
    print("cross", {k: art.measurements[k] for k in ("two_solver_max_delta", "lobpcg_iterations")}, flush=True)
    for tag, mixing in (("scf_kerker", MixingConfig(scheme=MixingScheme.KERKER, kerker_q0=0.5)),
                        ("scf_linear_kerker", MixingConfig(scheme=MixingScheme.LINEAR, alpha=0.3, kerker=True))):
        art = solve_self_consistent(scenario, numerics(0.5, (12.0, 12.0, 12.0), mixing), derive_grid=False)
        assert art.result is not None, art.error_message
        out[f"{tag}_total"] = np.array(art.result.energies.total)
        out[f"{tag}_iterations"] = np.array(art.result.n_iterations)
        print(tag, art.result.energies.total, art.result.n_iterations, flush=True)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}")


if __name__ == "__main__":
    main()
