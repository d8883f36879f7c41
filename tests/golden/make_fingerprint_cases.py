"""Write the reference's scenario fingerprint as test cases (``fingerprint_cases.json``).

Run where the reference checkout is readable (``CDFT_REFERENCE``, default ``/root/reference``):

    python tests/golden/make_fingerprint_cases.py [--check he_atom he_atom_lda ...]

The reference ships a full-precision fingerprint of its registered scenarios, solved at their
production settings on the CPU (``reports/fingerprint_cpu_reference.json``, written by its
``scripts/fingerprint.py``). For every scenario whose external potential is the nuclear Coulomb
field (the path built here), this script records what a native solve needs -- nuclear charges and
positions, electron count, functional, the grid the fingerprint was solved on, and the eigensolver,
mixing and SCF settings ``cdft.config.numerics_for_spec`` gives it -- beside the fingerprint's
energies, eigenvalues and iteration count. ``--check`` re-solves the named scenarios with the
reference here (``cdft.scf.solve.solve_scenario``) and records the total energy it gives now, so the
fixture also shows that the shipped fingerprint is the current reference's.
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
OUT = Path(__file__).resolve().parent / "fingerprint_cases.json"

os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
sys.dont_write_bytecode = True
sys.path[:0] = [str(REFERENCE), str(REFERENCE / "src")]


def _plain(value):
    value = getattr(value, "value", value)
    if isinstance(value, tuple):
        return [_plain(v) for v in value]
    return value


def _fields(config, names=None) -> dict:
    return {f.name: _plain(getattr(config, f.name)) for f in dataclasses.fields(config)
            if names is None or f.name in names}


def main() -> None:
    parser = argparse.ArgumentParser()
    parser.add_argument("--check", nargs="*", default=[], help="scenarios to re-solve with the reference here")
    args = parser.parse_args()

    from cdft.config import numerics_for_spec
    from cdft.physics_config import REGISTRY
    from contract import ExternalPotentialKind

    fingerprint = json.loads((REFERENCE / "reports" / "fingerprint_cpu_reference.json").read_text())
    cases = []
    for scenario in REGISTRY:
        entry = fingerprint.get(scenario.scenario_id)
        if scenario.external.kind is not ExternalPotentialKind.NUCLEAR_COULOMB or not entry:
            continue
        if entry.get("status") not in ("ok", "converged", "success") and "energies" not in entry:
            continue
        numerics, _ = numerics_for_spec(scenario)
        grid = entry["grid"]
        case = {
            "scenario": scenario.scenario_id,
            "charges": [float(z) for z in scenario.structure.numbers],
            "positions": [[float(c) for c in row] for row in scenario.structure.positions],
            "n_electrons": float(scenario.electrons.n_electrons),
            "functional": scenario.xc.name,
            "grid": {"shape": grid["shape"], "spacing": grid["spacing_bohr"], "origin": grid["origin_bohr"],
                     "fd_order": grid["fd_order"], "boundary": grid["boundary"]},
            "eigen": _fields(numerics.eigen),
            "mixing": _fields(numerics.mixing),
            "scf": _fields(numerics.scf),
            "seed": int(numerics.seed),
            "fingerprint": {
                "status": entry.get("status"),
                "energies": {k: float(v) for k, v in entry["energies"].items()},
                "eigenvalues": [float(v) for v in entry["eigenvalues"]],
                "occupations": [float(v) for v in entry["occupations"]],
                "n_iterations": entry.get("n_iterations"),
                "wall_time_s": entry.get("wall_time_s"),
            },
        }
        if scenario.scenario_id in args.check:
            from cdft.scf.solve import solve_scenario

            started = time.perf_counter()
            artifact = solve_scenario(scenario, dataclasses.replace(
                numerics, eigen=dataclasses.replace(numerics.eigen, cross_check=False)))
            case["reference_now"] = {"total": float(artifact.result.energies.total),
                                     "n_iterations": int(artifact.result.n_iterations),
                                     "seconds": time.perf_counter() - started}
            print(f"{scenario.scenario_id}: now {case['reference_now']['total']!r}, "
                  f"fingerprint {case['fingerprint']['energies']['total']!r}", flush=True)
        cases.append(case)
    meta = {"source": "reports/fingerprint_cpu_reference.json of the reference",
            "fingerprint_meta": fingerprint.get("_meta", {})}
    OUT.write_text(json.dumps({"_meta": meta, "cases": cases}, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(cases)} cases to {OUT}")


if __name__ == "__main__":
    main()
