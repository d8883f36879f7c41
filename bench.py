"""Benchmark: He-LDA 65^3 SCF solves per second on one B200 (or N replicas, one per GPU).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form mixed|fp64] [--impl native|reference]

A step is one complete self-consistent solve of He at VWN-LDA on the 16-bohr, h = 0.25 (65^3) grid
with linear density mixing alpha = 0.3 -- from the hydrogenic initial density to the converged
energy (|dE| < 1e-8 Ha, ||dn||_1 < 1e-6), then the final full diagonalisation -- with the geometry
(cusp factor, quadrature, Poisson plan) built before the timed region, as the reference caches it.
``--form mixed`` (default) filters in float32 and refines in float64 over a batch of systems;
``fp64`` is the plain float64 drop-in. Every timed step copies the initial density from pinned host
memory, solves, and reads the converged density back: ``value`` is timed with CUDA events around the
solve alone (its input already in HBM), ``e2e`` around the whole step. The L2 cache is flushed (a
256 MiB write) before every step, outside the timed events. The line also carries the plain FP64
drop-in's rate on the same box (``plain_fp64``) and the ratio the metric names.

``--impl reference`` times whole solves of the CPU restatement of the reference (``oracle/``) on this
host's threads and prints the same metric; ``cpu_baseline`` in the native line is one such solve.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "He-LDA 65^3 SCF solves/s at <=1e-8 Ha vs FP64"
UNIT = "solves/s"
REFERENCE_ENERGY_KEY = "he65_lda_linear"


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("native", "reference"), default="native")
    p.add_argument("--form", choices=("mixed", "fp64"), default="mixed")
    p.add_argument("--batch", type=int, default=None,
                   help="systems solved together per GPU (default 128 for the mixed form, 1 for fp64)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--kernel-only", action="store_true",
                   help="time only the fused Chebyshev step on a He grid of --edge points (for profiling)")
    p.add_argument("--breakdown", action="store_true",
                   help="device time per kernel of one solve (torch.profiler, no replay) instead of the bench line; "
                        "with --workload h2plus-scan, of one batched scan solve (one GPU)")
    p.add_argument("--workload", choices=("he-lda", "h2plus-scan", "adjoint"), default="he-lda",
                   help="he-lda: the headline He-LDA 65^3 solve; h2plus-scan: the 48-system bond scan; "
                        "adjoint: energy gradients of He-LDA at h 0.16 (101^3) against central differences")
    p.add_argument("--edge", type=int, default=65)
    p.add_argument("--orbitals", type=int, default=5)
    return p.parse_args()


def _golden():
    return json.loads((ROOT / "tests" / "golden" / "reference_values.json").read_text())[REFERENCE_ENERGY_KEY]


class ClockSampler:
    """nvidia-smi clock / throttle samples every 200 ms while running."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self._proc = None
        self._thread = None

    def start(self):
        try:
            self._proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                           "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                          stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self._proc = None
            return
        self._thread = threading.Thread(target=self._read, daemon=True)
        self._thread.start()

    def _read(self):
        for line in self._proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self) -> dict:
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._proc.kill()
        if self._thread is not None:
            self._thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def _peaks():
    path = ROOT / "MEASURED_PEAKS.json"
    if path.exists():
        data = json.loads(path.read_text())
        return float(data["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _profile_figure(name: str, kernel_tag: str):
    """A figure (``name[kernel_tag] = value``) of the dominant kernel from the committed ncu summaries."""
    for file in ("slab_filter_wide_he65.txt", "slab_filter_he65.txt"):
        path = ROOT / "profiles" / file
        if not path.exists():
            continue
        for line in path.read_text().splitlines():
            if line.startswith(f"{name}[{kernel_tag}]"):
                try:
                    return float(line.rsplit("=", 1)[1].strip())
                except ValueError:
                    return None
    return None


def _profile_traffic(kernel_tag: str):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summaries, if present."""
    return _profile_figure("traffic_bytes_per_launch", kernel_tag)


def _profile_pipe(tag: str, batch: int):
    """The arithmetic pipe's active fraction of the dominant kernel (ncu sm__pipe_fma_cycles_active for
    float32, sm__pipe_fp64_cycles_active for float64, over elapsed cycles), from the committed capture
    at this batch or, failing that, the largest batch captured (a rate, nearly independent of the
    batch once the grid fills the GPU)."""
    name = "fma_pipe_frac" if tag == "f32x4" else "fp64_pipe_frac"
    exact = _profile_figure(name, f"{tag},batch={batch}")
    if exact is not None:
        return exact, batch
    for b in (64, 32, 16, 8, 1):
        value = _profile_figure(name, f"{tag},batch={b}")
        if value is not None:
            return value, b
    return None, None


def filter_step_roofline(pkg, dev, grid, hamiltonian, m: int, precision, reps: int = 5, degree: int = 20):
    """Average device time of one fused Chebyshev step (stencil apply + recurrence) on m orbitals."""
    import torch

    block = torch.randn((m, grid.n_points), dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    for _ in range(2):
        pkg.chebyshev_filter(hamiltonian, block, degree, 1.0, 100.0, -3.0)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(reps):
        flush.fill_(1.0)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        pkg.chebyshev_filter(hamiltonian, block, degree, 1.0, 100.0, -3.0)
        end.record(stream)
        end.synchronize()
        total += start.elapsed_time(end) / 1e3
    per_launch_s = total / (reps * degree)
    s_bytes = 4 if precision == torch.float32 else 8
    algorithmic = grid.n_points * s_bytes * (3 * m + 5)
    return per_launch_s, algorithmic


def batched_filter_roofline(pkg, dev, grid, bham, m: int, precision, reps: int = 5, degree: int = 20):
    """Average device time of one fused Chebyshev step over a batch of systems (m orbitals each)."""
    import torch

    b = bham.batch
    block = torch.randn((b, m, grid.n_points), dtype=torch.float64, device=dev)
    rows = [pkg.chebyshev_coefficients(degree, 1.0, 100.0, -3.0)] * b
    table = torch.tensor(rows, dtype=torch.float64, device=dev)
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    for _ in range(2):
        bham.filter(block, table, degree)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(reps):
        flush.fill_(1.0)
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        bham.filter(block, table, degree)
        end.record(stream)
        end.synchronize()
        total += start.elapsed_time(end) / 1e3
    per_launch_s = total / (reps * degree)
    s_bytes = 4 if precision == torch.float32 else 8
    algorithmic = grid.n_points * s_bytes * (3 * b * m + b + 4)
    return per_launch_s, algorithmic


def run_kernel_only(args) -> None:
    """The fused Chebyshev step alone on a He grid (profiling entry: small, bounded).

    With ``--batch B`` (B > 1) the step runs over B systems of 5 orbitals with their own potentials
    (the bare potential, repeated), as in the batched solve.
    """
    import torch

    import __graft_entry__

    pkg = __graft_entry__.package()
    dev = torch.device("cuda:0")
    spacing = 16.0 / (args.edge - 1)
    grid = pkg.UniformGrid.box((16.0, 16.0, 16.0), spacing, (0.0, 0.0, 0.0), device=dev)
    geometry = pkg.build_cusp_geometry(grid, (2.0,), ((0.0, 0.0, 0.0),))
    precision = torch.float32 if args.form == "mixed" else torch.float64
    batch = args.batch or 1
    if batch > 1:
        bare = geometry.quadrature.bare_operator_terms()[0]
        bham = pkg.batch.BatchedHamiltonian(grid, geometry.factor, geometry.quadrature,
                                            bare[None, :].repeat(batch, 1).contiguous(), dtype=precision)
        per_launch_s, algorithmic = batched_filter_roofline(pkg, dev, grid, bham, args.orbitals, precision,
                                                            reps=args.steps)
    else:
        ham = pkg.CuspFactoredHamiltonian(grid, geometry.factor, quadrature=geometry.quadrature, dtype=precision)
        per_launch_s, algorithmic = filter_step_roofline(pkg, dev, grid, ham, args.orbitals, precision,
                                                         reps=args.steps)
    peak, kind = _peaks()
    achieved = algorithmic / per_launch_s / 1e9
    print(json.dumps({"kernel": "slab filter (one Chebyshev step)", "grid": grid.shape, "systems": batch,
                      "orbitals": args.orbitals, "form": args.form, "us_per_launch": per_launch_s * 1e6,
                      "algorithmic_bytes": algorithmic, "achieved_gbs": achieved, "peak_gbs": peak,
                      "peak_kind": kind, "frac": achieved / peak}), flush=True)


def run_adjoint(args) -> None:
    """Energy gradients of He-LDA at h = 0.16 (box 16 bohr, 101^3), float64, against central differences.

    The gradient with respect to the seeded Gaussian external perturbation (8 centres, widths
    U[0.5, 1.5] bohr) is the Hellmann--Feynman expectation value at the converged density (one SCF
    solve and 8 quadratures); it is checked against central differences of tightly converged total
    energies (step 1e-4 Ha, 16 more solves). The nuclear gradient is taken by central differences
    (step 1e-4 bohr, 6 solves) on the fixed grid. One JSON line: timings and the agreement.
    """
    import torch

    import __graft_entry__
    pkg = __graft_entry__.package()
    dev = torch.device("cuda:0")
    system = pkg.systems.he_lda(spacing=0.16, edge=16.0)
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=dev)
    geo = pkg.build_cusp_geometry(grid, system.charges, system.positions)
    scf = pkg.SCFConfig(energy_tol=1e-11, density_tol=1e-8, max_iterations=400)
    mixing = pkg.MixingConfig(scheme="linear", alpha=0.3)

    def solve(step):
        out = pkg.solve_self_consistent(step, mixing, scf)
        if not out.converged:
            raise RuntimeError("an SCF solve of the adjoint workload did not converge")
        return out

    def timed(fn):
        torch.cuda.synchronize()
        t = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return out, time.perf_counter() - t

    centres, widths, _ = pkg.adjoint.seeded_gaussians()
    base, t_scf = timed(lambda: solve(pkg.KohnShamStep(geo, "lda_vwn", system.n_electrons)))

    def gradient():
        g_node, g_grid = pkg.adjoint.perturbation_fields(geo, centres, widths)
        return pkg.adjoint.external_potential_gradient(geo, base.density, g_node, g_grid).cpu().numpy()

    grad, t_grad = timed(gradient)
    g_node, g_grid = pkg.adjoint.perturbation_fields(geo, centres, widths)
    dv = pkg.adjoint.effective_perturbation(geo, g_node, g_grid)
    step = 1.0e-4
    fd = []
    t0 = time.perf_counter()
    for k in range(dv.shape[0]):
        e = [float(solve(pkg.KohnShamStep(geo, "lda_vwn", system.n_electrons,
                                          external_potential=sign * step * dv[k])).energies["total"])
             for sign in (+1, -1)]
        fd.append((e[0] - e[1]) / (2 * step))
    t_fd = time.perf_counter() - t0
    rel = [abs(f - g) / abs(g) for f, g in zip(fd, grad)]

    def energy_at(positions):
        moved = pkg.build_cusp_geometry(grid, system.charges, [tuple(p) for p in positions])
        return float(solve(pkg.KohnShamStep(moved, "lda_vwn", system.n_electrons)).energies["total"])

    t0 = time.perf_counter()
    nuclear = pkg.adjoint.nuclear_gradient(energy_at, system.positions, delta=1.0e-4)
    t_nuc = time.perf_counter() - t0
    print(json.dumps({
        "workload": "adjoint: He-LDA h 0.16, box 16 bohr (101^3), float64; 8 seeded Gaussian perturbations",
        "energy_ha": float(base.energies["total"]), "scf_iterations": base.scf_iterations,
        "scf_seconds": t_scf, "gradient_seconds_after_scf": t_grad,
        "hellmann_feynman": [float(g) for g in grad], "central_differences": fd,
        "relative_difference": rel, "max_relative_difference": max(rel), "finite_difference_seconds": t_fd,
        "nuclear_gradient_central_differences": nuclear.tolist(), "nuclear_seconds": t_nuc,
        "grid": list(grid.shape)}), flush=True)


SCAN_BONDS = [0.8 + k * 5.2 / 47 for k in range(48)]


def scan_system(bond: float):
    import __graft_entry__

    return __graft_entry__.package().systems.h2_plus(bond, spacing=0.25, transverse=12.0)


def scan_figures(pkg, dev, precision, warmup: int, one_by_one: bool = True, indices=None) -> dict:
    """The bare H2+ bond scan: 48 systems, R = 0.8 + k 5.2 / 47, box (12, 12, R + 12), h = 0.25.

    Every system has its own grid (49 x 49 x 52 .. 73) and device geometry; one batched solve runs
    them together (one filter launch per CheFSI iteration for all of them). Returns systems per second
    of the batched solve (the geometry builds timed separately) and, if asked, of one-by-one solves.
    ``indices`` selects a share of the 48 (a rank's, under a cost partition); ``totals`` maps each
    solved index to its total energy.
    """
    import torch

    indices = list(range(len(SCAN_BONDS))) if indices is None else list(indices)
    stream = torch.cuda.current_stream()

    def timed(fn):
        torch.cuda.synchronize()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record(stream)
        out = fn()
        end.record(stream)
        end.synchronize()
        return out, start.elapsed_time(end) / 1e3

    def build_all():
        geos = []
        for k in indices:
            system = scan_system(SCAN_BONDS[k])
            grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=dev)
            geos.append(pkg.build_cusp_geometry(grid, system.charges, system.positions))
        return geos

    if not indices:
        return {"value": 0.0, "unit": "solves/s", "batched_solve_s": 0.0, "one_by_one_solve_s": None,
                "geometry_build_s": 0.0, "grids": [], "totals": {}}
    geos, build_s = timed(build_all)
    for _ in range(max(1, warmup)):
        pkg.batch.solve_noninteracting_batch(geos, 1.0, filter_precision=precision)
    batched, batched_s = timed(lambda: pkg.batch.solve_noninteracting_batch(geos, 1.0, filter_precision=precision))
    single_s = None
    if one_by_one:
        _, single_s = timed(lambda: [pkg.solve_noninteracting(g, n_electrons=1.0) for g in geos])
    return {"metric": "H2+ bond scan (48 systems, own grids) solves/s", "value": len(indices) / batched_s,
            "unit": "solves/s", "batched_solve_s": batched_s, "one_by_one_solve_s": single_s,
            "geometry_build_s": build_s, "grids": sorted({g.grid.shape for g in geos}),
            "totals": {k: float(batched[j]["total"]) for j, k in enumerate(indices)}}


def scan_errors(totals: list[float]) -> list[float]:
    """|E - E_reference| for the scan members the reference fixtures hold."""
    golden = json.loads((ROOT / "tests" / "golden" / "reference_values.json").read_text())
    return [abs(totals[k] - golden[f"h2plus_scan_R{SCAN_BONDS[k]:.4f}"]["total"])
            for k in range(len(SCAN_BONDS)) if f"h2plus_scan_R{SCAN_BONDS[k]:.4f}" in golden]


def run_scan(args) -> None:
    """The H2+ bond scan (``--workload h2plus-scan``) on N GPUs: the 48 systems are partitioned by
    cost (grid points; every member takes a similar number of applies) with one batched solve per
    rank and no collective during the solve; the time is the max over ranks and rank 0 gathers the
    energies on the host."""
    import torch

    import __graft_entry__

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    pkg = __graft_entry__.package()
    precision = torch.float32 if args.form == "mixed" else torch.float64
    shapes = []
    for bond in SCAN_BONDS:
        system = scan_system(bond)
        shapes.append(pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=dev).shape)
    if args.breakdown and world == 1:
        geos = []
        for bond in SCAN_BONDS:
            system = scan_system(bond)
            grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=dev)
            geos.append(pkg.build_cusp_geometry(grid, system.charges, system.positions))

        def solve(_):
            solve.last = None
            return pkg.batch.solve_noninteracting_batch(geos, 1.0, filter_precision=precision)

        for _ in range(args.warmup):  # the first solve also runs the tile autotuner's timings
            solve(None)
        _breakdown(solve, None)
        return
    costs = [pkg.replicas.system_cost(s) for s in shapes]
    shares = pkg.replicas.partition_by_cost(costs, world)
    figures = scan_figures(pkg, dev, precision, args.warmup, one_by_one=world == 1, indices=shares[rank])
    slowest = max_over_ranks(figures["batched_solve_s"], dist, dev)
    totals = pkg.replicas.gather_by_index(figures.pop("totals"), len(SCAN_BONDS), dist)
    if rank == 0:
        errors = scan_errors(totals)
        figures.update({"value": len(SCAN_BONDS) / slowest, "batched_solve_s": slowest, "n_gpus": world,
                        "form": args.form, "partition": "by cost (grid points), longest processing time first",
                        "share_loads": pkg.replicas.share_loads(costs, shares),
                        "max_energy_error_vs_reference_ha": max(errors) if errors else None,
                        "reference_members_checked": len(errors),
                        "data": "synthetic (the H2+ systems themselves)"})
        print(json.dumps(figures), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def _axis_term(ham, box, axis: int):
    """One axis's part ``D_d^T [w_d D_d phi]`` of the oracle's ``weighted_divergence`` for one orbital
    ``box`` (nx, ny, nz): the same element-wise operations in the same order as its loop body."""
    from oracle.grid import _pad_axis, _slice_along, staggered_coefficients

    acc = ham.grid.fd_order
    half = acc // 2
    coeffs = staggered_coefficients(acc)
    scale = 1.0 / ham.grid.spacing
    shape = box.shape
    padded = _pad_axis(box, axis, acc)
    faces = None
    for index, c in enumerate(coeffs):
        term = _slice_along(padded, axis, acc - half + 1 + (index - half), shape[axis] + acc)
        faces = term * (c * scale) if faces is None else faces + term * (c * scale)
    faces = faces * ham.faces[axis]
    term_sum = None
    for index, c in enumerate(coeffs):
        term = _slice_along(faces, axis, half - 1 - (index - half), shape[axis])
        term_sum = term * (c * scale) if term_sum is None else term_sum + term * (c * scale)
    return term_sum


def _orbital_filter(axis_pool, ham, row, degree: int, lower: float, upper: float, spectrum_min: float):
    """The oracle's ``chebyshev_filter`` for one orbital ``row`` (n,), the y and z axis terms of each
    application on ``axis_pool`` (or inline when it is None) while the calling thread forms the x
    term. The terms are added in the oracle's order ((x + y) + z), and h^3/omega and the potential
    are applied as in ``apply_with_potential``. The recurrence is the oracle's."""
    grid = ham.grid
    n = grid.n_points

    def apply(x):
        box = x.reshape(grid.shape)
        if axis_pool is None:
            terms = [_axis_term(ham, box, d) for d in range(3)]
        else:
            pending = [axis_pool.submit(_axis_term, ham, box, d) for d in (1, 2)]
            terms = [_axis_term(ham, box, 0)] + [f.result() for f in pending]
        div = (terms[0] + terms[1]) + terms[2]
        return div.reshape(n) * 0.5 * ham.inverse_weight + x * ham.potential

    e = 0.5 * (upper - lower)
    c = 0.5 * (upper + lower)
    sigma = e / (spectrum_min - c)
    sigma1 = sigma
    y = (apply(row) - c * row) * (sigma1 / e)
    previous = row
    for _ in range(2, degree + 1):
        sigma2 = 1.0 / (2.0 / sigma1 - sigma)
        y_new = (apply(y) - c * y) * (2.0 * sigma2 / e) - (sigma * sigma2) * previous
        previous, y = y, y_new
        sigma = sigma2
    return y


def _threaded_filter(ham, block, degree: int, lower: float, upper: float, spectrum_min: float, threads: int):
    """The oracle's ``chebyshev_filter`` of a block on up to ``threads`` host threads: one thread per
    orbital (the orbitals are independent until Rayleigh--Ritz) and, with at least three threads per
    orbital, the y and z axis terms of each application on a second pool (numpy releases the GIL in
    its array operations). Bit-identical to ``oracle.eigen.chebyshev_filter``. Returns (result,
    threads used)."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np

    k = block.shape[0]
    outer = max(1, min(k, threads))
    # the axis pool only when every orbital's y and z terms can run at once: with fewer threads the
    # extra synchronisation per application cost more than it gained (measured on 8 and 16 cores)
    inner = 2 * k if threads >= 3 * k else 0
    axis_pool = ThreadPoolExecutor(inner) if inner else None
    try:
        with ThreadPoolExecutor(outer) as pool:
            rows = list(pool.map(lambda o: _orbital_filter(axis_pool, ham, block[o], degree, lower, upper,
                                                           spectrum_min), range(k)))
    finally:
        if axis_pool is not None:
            axis_pool.shutdown()
    return np.stack(rows), outer + inner


def _chunked_xc(evaluate, pool, parts: int):
    """``oracle.xc.evaluate`` on ``parts`` slices of the points at once (the functionals are
    point-wise, so the result is bit-identical to one call on all points)."""
    import numpy as np

    def run(name, density, sigma=None):
        density = np.asarray(density, dtype=np.float64)
        sig = None if sigma is None else np.asarray(sigma, dtype=np.float64)
        cuts = [c for c in np.array_split(np.arange(density.shape[0]), parts) if c.size]
        res = list(pool.map(lambda c: evaluate(name, density[c], None if sig is None else sig[c]), cuts))
        v_sigma = None if res[0][2] is None else np.concatenate([r[2] for r in res])
        return np.concatenate([r[0] for r in res]), np.concatenate([r[1] for r in res]), v_sigma

    return run


class _RowBlocks:
    """A sparse matrix split into row blocks whose products with a vector or an (n, k) array run on a
    thread pool (scipy releases the GIL in its sparse products). Rows are independent, so the
    product is bit-identical to the whole matrix's."""

    def __init__(self, matrix, pool, parts: int):
        import numpy as np

        m = matrix.tocsr()
        cuts = np.linspace(0, m.shape[0], max(1, parts) + 1).round().astype(int)
        self.blocks = [m[a:b] for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
        self.pool = pool
        self.shape = m.shape

    def __matmul__(self, v):
        import numpy as np

        return np.concatenate(list(self.pool.map(lambda block: block @ v, self.blocks)), axis=0)


class HostThreads:
    """The oracle's own solve with its independent parts on the host's threads, bit for bit.

    Inside the context, for the geometry ``(grid, factor, quadrature)``:

    - the Chebyshev filter runs one orbital per thread, with each application's y and z axis terms
      on further threads when the host has them (``_threaded_filter``: the recurrence of every
      orbital is independent until Rayleigh--Ritz);
    - every other block application's axis terms ``D_d^T[w_d D_d phi]`` run one task per (orbital,
      axis) (``_axis_term``: the oracle's element-wise operations in its order; the terms are added
      ``(x + y) + z`` as the oracle's ``weighted_divergence`` does);
    - the point-wise XC evaluations run as slices of the points (``_chunked_xc``);
    - the interpolant and the lift run as row blocks of the sparse matrices (``_RowBlocks``);
    - the Poisson FFTs use scipy's FFT of the same transforms on every thread.

    numpy and scipy release the GIL in these operations. The rest of the solve (small sums, dense
    solves, the SCF control flow) runs on the calling thread. ``seconds`` accumulates the time spent
    in the block applications and the potential evaluations, as a breakdown of the solve.
    """

    def __init__(self, geometry, cores: int) -> None:
        self.grid, self.factor, self.quadrature = geometry
        self.cores = max(1, int(cores))
        self.seconds = {"applications": 0.0, "potentials": 0.0}
        self.counts = {"applications": 0, "potentials": 0}

    def __enter__(self):
        from concurrent.futures import ThreadPoolExecutor

        import numpy as np

        from oracle import operators as oops
        from oracle import scf as oscf
        from oracle import xc as oxc

        from oracle import eigen as oeigen

        self._pool = ThreadPoolExecutor(self.cores)
        pool, cores, box_shape = self._pool, self.cores, self.grid.shape
        self._saved = (oxc.evaluate, self.quadrature.L, self.quadrature.LT, oops.CoulombCutoffPoisson.solve,
                       oops.CuspHamiltonian.kinetic_apply, oscf.KohnShamStep.potentials, oeigen.chebyshev_filter)
        serial_xc, _, _, serial_poisson, _, serial_potentials, serial_filter = self._saved
        seconds, counts = self.seconds, self.counts

        def chebyshev_filter(ham, block, degree, lower, upper, spectrum_min):
            if type(ham) is not oops.CuspHamiltonian:  # e.g. a level-shifted operator: the serial filter
                return serial_filter(ham, block, degree, lower, upper, spectrum_min)
            if upper <= lower:
                raise ValueError(f"filter interval is empty: lower={lower}, upper={upper}")
            t = time.perf_counter()
            out, _ = _threaded_filter(ham, block, degree, lower, upper, spectrum_min, cores)
            ham.apply_count += degree
            seconds["applications"] += time.perf_counter() - t
            counts["applications"] += degree
            return out

        def kinetic_apply(ham, phi):
            t = time.perf_counter()
            n = ham.grid.n_points
            rows = phi.reshape(-1, n)
            pending = [[pool.submit(_axis_term, ham, rows[r].reshape(box_shape), d) for d in range(3)]
                       for r in range(rows.shape[0])]
            out = np.empty_like(rows)
            for r, futures in enumerate(pending):
                terms = [f.result() for f in futures]
                out[r] = ((terms[0] + terms[1]) + terms[2]).reshape(n) * 0.5 * ham.inverse_weight
            seconds["applications"] += time.perf_counter() - t
            counts["applications"] += 1
            return out.reshape(phi.shape)

        def poisson_solve(solver, density):
            solver.fft_workers = cores
            return serial_poisson(solver, density)

        def potentials(step, density):
            t = time.perf_counter()
            out = serial_potentials(step, density)
            seconds["potentials"] += time.perf_counter() - t
            counts["potentials"] += 1
            return out

        oxc.evaluate = _chunked_xc(serial_xc, pool, cores)
        self.quadrature.L = _RowBlocks(self._saved[1], pool, cores)
        self.quadrature.LT = _RowBlocks(self._saved[2], pool, cores)
        oops.CoulombCutoffPoisson.solve = poisson_solve
        oops.CuspHamiltonian.kinetic_apply = kinetic_apply
        oscf.KohnShamStep.potentials = potentials
        oeigen.chebyshev_filter = chebyshev_filter
        return self

    def __exit__(self, *exc):
        from oracle import eigen as oeigen
        from oracle import operators as oops
        from oracle import scf as oscf
        from oracle import xc as oxc

        (oxc.evaluate, self.quadrature.L, self.quadrature.LT, oops.CoulombCutoffPoisson.solve,
         oops.CuspHamiltonian.kinetic_apply, oscf.KohnShamStep.potentials, oeigen.chebyshev_filter) = self._saved
        self._pool.shutdown()
        return False


def oracle_solve(system, geometry, cores: int) -> tuple[dict, float, dict]:
    """One whole SCF solve of the CPU restatement (``oracle.scf.solve_self_consistent``) on ``cores``
    host threads (:class:`HostThreads`), geometry already built. Returns (result, seconds, breakdown)."""
    from oracle import scf as oscf

    with HostThreads(geometry, cores) as threads:
        t = time.perf_counter()
        result = oscf.solve_self_consistent(system, geometry)
        seconds = time.perf_counter() - t
    breakdown = {"block_applications": threads.counts["applications"],
                 "block_application_s": threads.seconds["applications"],
                 "potential_evaluations": threads.counts["potentials"],
                 "potential_evaluation_s": threads.seconds["potentials"]}
    return result, seconds, breakdown


def oracle_warmup(system, geometry, cores: int) -> None:
    """First-call costs of the CPU solve (thread pools, FFT plans, page faults): one potential
    evaluation and one block application, not timed."""
    import numpy as np

    from oracle import scf as oscf
    from oracle.operators import CuspHamiltonian

    grid, factor, quad = geometry
    with HostThreads(geometry, cores):
        step = oscf.KohnShamStep(system, grid, factor, quad)
        p = step.potentials(oscf.initial_density(step))
        ham = CuspHamiltonian(grid, factor, quad, extra_potential=p["effective"], bare=step.bare)
        ham.apply(np.random.default_rng(0).standard_normal((5, grid.n_points)))


#: Seconds of CPU solves the reference arm times at most (it always times one whole solve).
REFERENCE_BUDGET_S = 150.0


def _solve_text(result, seconds: float, cores: int, breakdown: dict, what: str = "whole SCF solves") -> str:
    return (f"{what} of the numpy restatement of the reference (oracle.scf.solve_self_consistent) on "
            f"{cores} host threads: {result['scf_iterations']} SCF iterations, "
            f"{breakdown['block_applications']} block applications ({breakdown['block_application_s']:.1f} s), "
            f"{breakdown['potential_evaluations']} potential evaluations ({breakdown['potential_evaluation_s']:.1f} s), "
            f"{seconds:.1f} s per solve; geometry build excluded (cached, as the reference caches it)")


def run_reference(args) -> None:
    """The reference's CPU path (the oracle restatement) on this host: whole solves of the workload.

    Every timed step is one complete SCF solve. A solve takes about a minute even on all host
    threads, so the arm times ``min(--steps, n)`` solves, n the count that fits
    ``REFERENCE_BUDGET_S`` (at least one), and reports the count it timed as ``steps``; the warm-up
    is one potential evaluation and one block application rather than whole solves.
    """
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import scf as oscf

    cores = os.cpu_count() or 1
    system = oscf.he_lda()
    geometry = oscf.build_geometry(system)
    golden = _golden()
    if args.warmup > 0:
        oracle_warmup(system, geometry, cores)
    times, errors = [], []
    text = ""
    requested = max(1, args.steps)
    while len(times) < requested:
        result, seconds, breakdown = oracle_solve(system, geometry, cores)
        times.append(seconds)
        errors.append(abs(result["energies"]["total"] - golden["total"]))
        text = _solve_text(result, seconds, cores, breakdown)
        if sum(times) + statistics.mean(times) > REFERENCE_BUDGET_S:
            break
    total = sum(times)
    value = len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(times), "steps_requested": requested, "warmup": 1 if args.warmup > 0 else 0,
        "warmup_kind": "one potential evaluation and one block application",
        "ms_per_step": total * 1e3 / len(times), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (the He atom system itself; no dataset)",
        "config": {"workload": "He-LDA 65^3 SCF solve (box 16 bohr, h 0.25, linear mixing 0.3)", "l2": "n/a (CPU)",
                   "energy_error_vs_reference_cpu_fp64_ha": max(errors), "solve_seconds": times},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": text},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _breakdown(solve, n0) -> None:
    """Print the device time of every kernel of one solve (torch.profiler's CUDA activity)."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    t = time.perf_counter()
    solve(n0)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    with profile(activities=[ProfilerActivity.CPU, ProfilerActivity.CUDA]) as prof:
        solve(n0)
        torch.cuda.synchronize()
    rows = [k for k in prof.key_averages() if k.self_device_time_total > 0]
    busy = sum(k.self_device_time_total for k in rows) / 1e3
    print(f"wall {wall * 1e3:.0f} ms per step, GPU busy {busy:.1f} ms")
    for k in sorted(rows, key=lambda r: -r.self_device_time_total)[:30]:
        print(f"{k.self_device_time_total / 1e3:9.2f} ms  {k.count:7d}  {k.key[:110]}")
    last = getattr(solve, "last", None)
    if last is not None:
        ms = last.measurements
        print("scf iterations", last.scf_iterations)
        print("float64 refinement from iteration", ms.get("fp64_refinement_from_iteration"))


def replica_seeds(rank: int, batch: int) -> list[int]:
    """Seeds of the independent systems one replica solves: disjoint across ranks."""
    return [rank * batch + k for k in range(batch)]


def max_over_ranks(seconds: float, dist, device) -> float:
    """The slowest rank's time (all-reduce MAX); the local time without a process group."""
    if dist is None:
        return seconds
    import torch

    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, batch: int, steps: int, seconds: float) -> float:
    """Solves per second of the whole job: every rank solves `batch` systems per step."""
    return world * batch * steps / seconds


def main() -> None:
    args = _args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.kernel_only:
        run_kernel_only(args)
        return
    if args.workload == "h2plus-scan":
        run_scan(args)
        return
    if args.workload == "adjoint":
        run_adjoint(args)
        return
    import torch

    import __graft_entry__

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and world > 1:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE {world}")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)

    pkg = __graft_entry__.package()
    lib = pkg._lib.library()
    system = pkg.systems.he_lda()
    grid = pkg.UniformGrid.box(system.box_lengths, system.spacing, system.anchor, device=dev)
    geometry = pkg.build_cusp_geometry(grid, system.charges, system.positions)
    precision = torch.float32 if args.form == "mixed" else torch.float64
    batch = args.batch if args.batch is not None else (128 if args.form == "mixed" else 1)
    mixing = pkg.MixingConfig(scheme="linear", alpha=0.3)
    golden = _golden()
    flush = torch.empty(256 * 2 ** 20 // 4, dtype=torch.float32, device=dev)
    if batch == 1:
        step = pkg.KohnShamStep(geometry, "lda_vwn", system.n_electrons, filter_precision=precision)
        n0 = pkg.initial_density(step)

        def solve(initial):
            out = pkg.solve_self_consistent(step, mixing, initial_density_override=initial)
            return [out.energies["total"]], out.density, out.scf_iterations, out.applications
    else:
        # independent systems: the same atom from different seeded random starts (seed = rank * batch + b)
        seeds = replica_seeds(rank, batch)
        step = pkg.batch.BatchedKohnShamStep(geometry, "lda_vwn", system.n_electrons, batch, seeds=seeds,
                                             filter_precision=precision)
        n0 = step.initial_density()

        def solve(initial):
            out = pkg.batch.solve_self_consistent_batch(step, mixing, initial_density=initial)
            solve.last = out
            return ([e["total"] for e in out.energies], out.density, max(out.scf_iterations), out.applications)

    for _ in range(max(0, args.warmup)):
        solve(n0)
    torch.cuda.synchronize()
    if args.breakdown:
        _breakdown(solve, n0)
        return

    # --- K timed steps. Each step copies its input density from pinned host memory (event e0 -> e1),
    # solves from it, resident in HBM (e1 -> e2), and reads the converged density back (e2 -> e3).
    # value: the solves alone (e1 -> e2); e2e: the whole step through the public API (e0 -> e3).
    host_in = n0.cpu().pin_memory()
    host_out = torch.empty(n0.shape, dtype=torch.float64).pin_memory()
    bytes_in = host_in.numel() * host_in.element_size()
    bytes_out = host_out.numel() * host_out.element_size() + 8 * 12 * batch  # density + the energy terms
    sampler = ClockSampler(local)
    sampler.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.cdftb_launch_count()
    solve_ms = e2e_ms = 0.0
    energies = []
    stream = torch.cuda.current_stream()
    iterations = applications = None
    for _ in range(args.steps):
        flush.fill_(1.0)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        dev_in = host_in.to(dev, non_blocking=True)
        ev[1].record(stream)
        totals, density, iterations, applications = solve(dev_in)
        ev[2].record(stream)
        host_out.copy_(density.reshape(host_out.shape), non_blocking=True)
        ev[3].record(stream)
        ev[3].synchronize()
        solve_ms += ev[1].elapsed_time(ev[2])
        e2e_ms += ev[0].elapsed_time(ev[3])
        energies.extend(totals)
    torch.cuda.synchronize()
    launches = lib.cdftb_launch_count() - launches0
    pkg._lib.check_device_status("the timed steps")
    if dist is not None:
        dist.barrier()
    clocks = sampler.stop()
    seconds = max_over_ranks(solve_ms / 1e3, dist, dev)
    value = whole_job_rate(world, batch, args.steps, seconds)
    e2e_s = max_over_ranks(e2e_ms / 1e3, dist, dev)
    e2e_value = whole_job_rate(world, batch, args.steps, e2e_s)
    error = max(abs(e - golden["total"]) for e in energies)

    # --- the plain FP64 drop-in (one system, float64 throughout) on the same box, for the metric's ratio
    plain = None
    if batch > 1 or precision != torch.float64:
        step64 = pkg.KohnShamStep(geometry, "lda_vwn", system.n_electrons, filter_precision=torch.float64)
        n64 = pkg.initial_density(step64)
        out64 = pkg.solve_self_consistent(step64, mixing, initial_density_override=n64)  # warm-up
        plain_steps = 5
        plain_ms = 0.0
        plain_errors = []
        for _ in range(plain_steps):
            flush.fill_(1.0)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            out64 = pkg.solve_self_consistent(step64, mixing, initial_density_override=n64)
            end.record(stream)
            end.synchronize()
            plain_ms += start.elapsed_time(end)
            plain_errors.append(abs(out64.energies["total"] - golden["total"]))
        pkg._lib.check_device_status("the plain FP64 solves")
        plain_s = max_over_ranks(plain_ms / 1e3, dist, dev)
        plain_value = whole_job_rate(world, 1, plain_steps, plain_s)
        plain = {"value": plain_value, "unit": UNIT, "steps": plain_steps, "ms_per_step": plain_s * 1e3 / plain_steps,
                 "energy_error_vs_reference_cpu_fp64_ha": max(plain_errors), "scf_iterations": out64.scf_iterations,
                 "form": "plain float64 drop-in, one system per solve (scf.solve_self_consistent)"}
        # the same solves with every Chebyshev filter replayed from a CUDA graph (one engine for all)
        stepg = pkg.KohnShamStep(geometry, "lda_vwn", system.n_electrons, filter_precision=torch.float64, graphs=True)
        outg = pkg.solve_self_consistent(stepg, mixing, initial_density_override=n64)  # warm-up and capture
        graphed_ms = 0.0
        graphed_errors = []
        for _ in range(plain_steps):
            flush.fill_(1.0)
            start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            outg = pkg.solve_self_consistent(stepg, mixing, initial_density_override=n64)
            end.record(stream)
            end.synchronize()
            graphed_ms += start.elapsed_time(end)
            graphed_errors.append(abs(outg.energies["total"] - golden["total"]))
        pkg._lib.check_device_status("the graphed plain FP64 solves")
        graphed_s = max_over_ranks(graphed_ms / 1e3, dist, dev)
        record = outg.measurements["cuda_graphs"]
        plain["graphed"] = {"value": whole_job_rate(world, 1, plain_steps, graphed_s),
                            "ms_per_step": graphed_s * 1e3 / plain_steps,
                            "energy_error_vs_reference_cpu_fp64_ha": max(graphed_errors),
                            "graph_captures": record["captures"], "graph_replays": record["replays"],
                            "graph_used": record["used"]}
        plain["ratio_against"] = "the faster of the direct and the graphed plain solve"

    # --- roofline of the dominant kernel: one fused Chebyshev step (apply + recurrence) over the batch ---
    effective = (step.potentials(n0).effective if batch == 1 else step.potentials(n0).effective)
    if batch == 1:
        ham = step.hamiltonian(step.potentials(n0), dtype=precision)
        per_launch_s, algorithmic = filter_step_roofline(pkg, dev, grid, ham, 5, precision)
    else:
        bham = step.hamiltonian(effective, dtype=precision)
        per_launch_s, algorithmic = batched_filter_roofline(pkg, dev, grid, bham, 5, precision)
    achieved = algorithmic / per_launch_s / 1e9
    peak, peak_kind = _peaks()
    # one shared geometry: the wide-lane kernel (four float32 or two float64 orbitals per lane point)
    tag = "f32x4" if precision == torch.float32 else "f64x2"
    pipe_frac, pipe_batch = _profile_pipe(tag, batch)

    result = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": seconds * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32-filter/f64" if precision == torch.float32 else "f64",
        "data": "synthetic (the He atom system itself; no dataset)",
        "config": {"workload": "He-LDA 65^3 SCF solve (box 16 bohr, h 0.25, linear mixing 0.3)",
                   "form": args.form, "systems_per_gpu": batch, "l2": "flushed (256 MiB write) before every step",
                   "parallelism": f"replicas{world}", "energy_error_vs_reference_cpu_fp64_ha": error,
                   "scf_iterations": iterations, "applications_per_system": applications / batch,
                   "value_timing": "device events around each solve, input already copied to HBM",
                   "e2e_timing": "device events around host-to-device copy + solve + device-to-host read, same steps"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_in, "d2h_bytes_per_step": bytes_out},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": _profile_traffic(f"{tag},batch={batch}"),
                     "kernel": f"slab_filter_wide_kernel<{tag}> (one Chebyshev step, {batch} systems x 5 orbitals)",
                     "algorithmic_bytes_per_launch": algorithmic, "us_per_launch": per_launch_s * 1e6,
                     "peak_kind": peak_kind,
                     "fp32_pipe_frac" if tag == "f32x4" else "fp64_pipe_frac": pipe_frac,
                     "pipe_source": (f"ncu {'sm__pipe_fma' if tag == 'f32x4' else 'sm__pipe_fp64'}_cycles_active / "
                                     f"elapsed, one launch at {pipe_batch} systems (profiles/slab_filter_wide_he65.txt)"
                                     if pipe_frac is not None else None)},
        "clocks": clocks,
    }
    if rank == 0 and world == 1:
        # config 4 beside the headline: the 48-system bond scan, every system on its own grid
        scan = scan_figures(pkg, dev, precision, warmup=1, one_by_one=False)
        errors = scan_errors([scan["totals"][k] for k in range(len(SCAN_BONDS))])
        result["h2plus_scan"] = {k: scan[k] for k in ("value", "unit", "batched_solve_s", "geometry_build_s")}
        result["h2plus_scan"].update({"max_energy_error_vs_reference_ha": max(errors) if errors else None,
                                      "reference_members_checked": len(errors)})
        result["h2plus_scan"]["workload"] = "bare H2+ bond scan, 48 systems on their own grids (49x49x52..73)"
    if plain is not None:
        result["plain_fp64"] = plain
        result["batched_mixed_over_plain_fp64"] = value / (world * max(plain["value"], plain["graphed"]["value"]))
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        from oracle import scf as oscf  # the CPU baseline leg: the oracle's own system and solve

        cores = os.cpu_count() or 1
        cpu_system = oscf.he_lda()
        cpu_geometry = oscf.build_geometry(cpu_system)
        oracle_warmup(cpu_system, cpu_geometry, cores)
        cpu_result, cpu_s, breakdown = oracle_solve(cpu_system, cpu_geometry, cores)
        result["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": UNIT, "cores": cores, "kind": "port",
                                  "sample": _solve_text(cpu_result, cpu_s, cores, breakdown, "one whole SCF solve"),
                                  "energy_error_vs_reference_cpu_fp64_ha":
                                      abs(cpu_result["energies"]["total"] - golden["total"])}
    if rank == 0:
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
