#!/usr/bin/env python3
"""Time-step throughput of the ParaCFD per-timestep solver path on B200.

Workload: the 4-level ~16 M leaf-cell paraglider case (``paraglider16m``, FP32 flow state, FP64
pressure, projection to 1e-8 relative residual, surface loads integrated every step) on its
cut-cell grid.  The grid (brick hierarchy, cut-cell embedded-boundary atlas, composite pressure
system) is the reference's own host preprocessing of the closed wing surface, compiled from its
sources (oracle/_ref); it reaches this library through ``pcfd_topology``, the drop-in boundary,
before any timed region.  ``--grid staircase`` uses this library's own solid-cell builder
(``pcfd_topology_build``) instead.  A step is one ``pcfd_core_step`` (CFL -> MUSCL transport ->
Smagorinsky diffusion -> smooth wall -> flux reconstruction -> boundaries -> projection ->
pressure traction) plus ``pcfd_core_loads``.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Arms
  ours       value = steps/s over K steps with the state resident in HBM (CUDA events on the
             system stream, max over ranks); e2e = steps/s over K more steps through the public
             API with host buffers: per step the X-min inflow profile is copied from pinned host
             memory and the loads are read back.  Every resident vector (19 M-DOF FP64 pressure
             vectors, 0.16 GB each) is larger than the 126 MB L2.
  reference  whole time steps of the reference's host implementation on this machine's cores:
             its CPU twins of every operator (oracle/_ref, single-threaded as written) in
             ExternalAeroCore::step's order, with the projection solved to 1e-8 by the FP64
             OpenMP restatement of its solver (the reference has no CPU solver).  A CPU step of
             the 16 M-cell grid takes minutes, so each timed step is a whole step of the same
             wing on the 1.1 M-cell grid (paraglider1m) and the value is scaled to 16 M cells by
             the cell count (see CpuStepper).  Beside it, the reference's own sm_100a build
             (its device classes in ExternalAeroCore's step sequence) runs K whole steps of the
             full workload: ``reference_sm100a``.  This arm never loads libparacfd_b200.so.
Multi-GPU: independent replicas, one per rank (the path has no exchange step).

Solver defaults of the ours arm: the composite multigrid cycle in FP32 with FP16 stage
coefficients (Chebyshev stage smoothing, Chebyshev-Richardson fine steps, exact coarsest stage),
flexible GMRES with delayed CGS2 and no recycled subspace; --mg-cycle reference --mg fp64
--delayed 0 --recycle 0 selects the reference's solver configuration.  The line also carries a
short learned-preconditioner comparison (skip with --no-learned).  Other modes:
  --learned     the learned-preconditioner measurement (harvest, train, re-solve each step's
                projection under each preconditioner)
  --sweep       the batched angle sweep (16 wing instances, 4 concurrent batches)
  --kernel-only the small per-component command that ncu captures
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

A_P_BYTES_PER_DOF = 18   # FP64 7-point operator: p 8 + Ap 8 + active 1 + cut mask 1
CLOCK_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                "clocks_event_reasons.sw_power_cap")


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default="paraglider16m")
    ap.add_argument("--grid", choices=("cutcell", "staircase"), default="cutcell",
                    help="cutcell: the reference's own preprocessing of the surface (brick hierarchy, cut-cell EB "
                         "atlas, composite system); staircase: this library's solid-cell builder")
    ap.add_argument("--mg", choices=("fp64", "fp32"), default="fp32",
                    help="multigrid preconditioner precision (the composite stages; fine sweeps and Krylov stay FP64)")
    ap.add_argument("--restart", type=int, default=0, help="GCRO columns per cycle (0: the reference's 24)")
    ap.add_argument("--mg-cycle", choices=("reference", "corrected", "composite"), default="composite",
                    help="coarse-correction weighting of the multigrid cycle (pcfd_mg_cycle)")
    ap.add_argument("--stage-sweeps", type=int, default=4,
                    help="composite cycle: smoothing steps per stage before and after its correction (0: the library's 6)")
    ap.add_argument("--chebyshev", type=int, default=20,
                    help="composite stages: r >= 2 = Chebyshev smoothing on [2/r, 2], 1 = damped Jacobi, 0: r = 30")
    ap.add_argument("--fine-chebyshev", type=int, default=0,
                    help="composite fine sweeps: r >= 2 = Chebyshev-Richardson steps on [2/r, 2], 1 = damped Jacobi, 0: r = 10")
    ap.add_argument("--delayed", type=int, default=1, choices=(0, 1),
                    help="1: GCRO columns orthogonalised by delayed CGS2 (two passes instead of three); 0: CGS2")
    ap.add_argument("--stage-fp16", type=int, default=1, choices=(0, 1),
                    help="1: FP16 storage of the composite stages' coefficients (FP32 multigrid); 0: FP32")
    ap.add_argument("--recycle", type=int, default=-1,
                    help="GCRO recycled pairs kept between solves: 1..3, -1 none (default), 0: the reference's 3")
    ap.add_argument("--block-iterations", type=int, default=0,
                    help="composite cycle: Chebyshev iterations of the brick block pre-smoother (0: Jacobi pre-sweeps)")
    ap.add_argument("--initial-guess", choices=("previous", "extrapolated", "quadratic"), default="extrapolated",
                    help="step projections start from the last pressure (the reference's warm start) or from "
                         "2 p_n - p_(n-1) of the last two")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU sample of the ours arm")
    ap.add_argument("--no-reference-gpu", action="store_true", help="reference arm: skip the sm_100a reference run")
    ap.add_argument("--profile-region", type=int, default=0, help="PCFD_PROFILE_* region timed per launch")
    ap.add_argument("--kernel-only", type=int, default=None,
                    help="build the workload, time one pcfd_time_kernel component (a few launches) and exit; "
                         "the small command an ncu capture of that component runs")
    ap.add_argument("--kernel-iterations", type=int, default=1)
    ap.add_argument("--learned", action="store_true",
                    help="the learned-preconditioner measurement: harvest brick pairs from seeded naca0012_slab / "
                         "naca4412_wing runs, train, then time projections to 1e-8 with the learned forms against "
                         "the multigrid on the same right-hand sides of the naca4412_wing case")
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--no-learned", action="store_true", help="skip the short learned-preconditioner comparison")
    ap.add_argument("--no-sweep-summary", action="store_true", help="skip the one-batch angle-sweep summary")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default brick-pipeline launch shape")
    ap.add_argument("--sweep", action="store_true",
                    help="batched angle sweep: 16 naca4412_wing instances (AoA -4..11 deg, seeded refinement bands) in "
                         "4 batches of 4, each batch stepped sequentially and then concurrently (one host thread and "
                         "stream per instance); reports instance-steps/s of both")
    ap.add_argument("--harvest-runs", type=int, default=4, help="seeded harvest runs (alternating the two cases)")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------ ranks
class Ranks:
    """One process per GPU; the collective (NCCL on GPUs, gloo for the CPU tests) only carries the
    barrier and the max over ranks -- the replicas share no data."""

    def __init__(self, collective: bool, backend: str = "nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cpu"
        if self.world > 1 and collective:
            import datetime

            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = f"cuda:{self.local}"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.dist, self.torch = dist, torch

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, value: float) -> float:
        if not self.dist:
            return value
        t = self.torch.tensor([value], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


def replica_throughput(world: int, steps: int, slowest_ms: float) -> float:
    """Whole-job steps/s of `world` independent replicas that each ran `steps` steps, timed by the
    slowest rank (weak scaling: per-GPU work fixed)."""
    return world * steps / (slowest_ms * 1e-3)


# ------------------------------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    def __init__(self, device: int, path: str | None = None):
        self.device = device
        self.proc = None
        self.path = path or os.path.join(tempfile.gettempdir(), f"pcfd_clocks_{os.getpid()}_{device}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.file = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={CLOCK_FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.file.close()

    def summary(self) -> dict:
        out = self._read()
        if self.proc:
            try:
                os.remove(self.path)
            except OSError:
                pass
        return out

    def _read(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        visible = os.environ.get("CUDA_VISIBLE_DEVICES")
        index = str(self.device)
        if visible and visible.split(",")[self.device:self.device + 1]:
            index = visible.split(",")[self.device].strip()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                cols = [c.strip() for c in line.split(",")]
                if len(cols) < 9 or cols[0] != index:
                    continue
                try:
                    sm.append(float(cols[1]))
                    smax.append(float(cols[2]))
                except ValueError:
                    continue
                for name, flag in zip(names, cols[5:9]):
                    if flag.lower() == "active":
                        reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------ helpers
def measured_peak_gbs() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def non_covered_bricks(topology) -> int:
    from paracfd_b200 import capi
    count = 0
    for l in range(topology.level_count):
        lev = topology.levels[l]
        flags = np.ctypeslib.as_array(lev.flags, shape=(lev.brick_count,))
        count += int(((flags & capi.BRICK_COVERED) == 0).sum())
    return count


def inflow_face_centres(topology, slots: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(y, z) of every X-min inflow face in pcfd_core_inflow_layout order."""
    bs = topology.brick_size
    starts = np.cumsum([0] + [topology.levels[l].brick_count for l in range(topology.level_count)])
    y = np.empty((len(slots), bs, bs))
    z = np.empty((len(slots), bs, bs))
    jk = (np.arange(bs) + 0.5)
    for n, slot in enumerate(slots):
        l = int(np.searchsorted(starts, slot, side="right") - 1)
        lev = topology.levels[l]
        b = int(slot - starts[l])
        oy, oz = lev.origin[3 * b + 1], lev.origin[3 * b + 2]
        y[n] = oy + jk[None, :] * lev.h          # [k][j]
        z[n] = oz + jk[:, None] * lev.h
    return y.ravel(), z.ravel()


def inflow_profile(speed: float, centres, step: int) -> np.ndarray:
    """Deterministic gusting X-min inflow: a +-2 % smooth travelling modulation of the freestream."""
    y, z = centres
    return (speed * (1.0 + 0.02 * np.sin(0.6 * y + 0.4 * z + 0.1 * step))).astype(np.float32)


# DRAM bytes (read + write) per launch of the roofline kernel, from one ncu capture of
# `bench.py --kernel-only <k> --workload <w>` (--metrics dram__bytes_read.sum,dram__bytes_write.sum,
# one pass); keyed by (workload, grid, kernel-only component[, first stage brick-structured]).  A bench run cannot measure DRAM
# traffic itself; absent entries report null.  Stage-1 Chebyshev step on the 16 M-cell cut-cell
# grid as CSR: two captured launches read 113.36 MB each and wrote 7.61 and 4.01 MB (mean taken);
# the algorithmic figure is 129.4 MB, the difference the part of the 2.0 M-row stage the L2 keeps
# between launches.  The same stage in brick-structured form: 71.91 MB read, 2.69 and 1.16 MB
# written (mean taken) against 89.9 MB algorithmic.
DRAM_BYTES_PER_LAUNCH: dict = {("paraglider16m", "cutcell", 17, False): 119_170_000,
                               ("paraglider16m", "cutcell", 17, True): 73_834_752}


# ------------------------------------------------------------------------------------------ grids
class Grid:
    """A workload's grid: the topology view handed to the library plus what the line reports.

    ``cutcell`` is the reference's own preprocessing of the workload's closed surface (brick
    hierarchy, cut-cell embedded-boundary atlas, composite pressure system; oracle/_ref), the
    input the drop-in boundary receives from the reference's caller.  ``staircase`` is this
    library's own solid-cell builder (pcfd_topology_build)."""

    def __init__(self, spec, kind: str = "cutcell"):
        self.kind = kind
        self.spec = spec
        if kind == "cutcell":
            from oracle import ref
            self.holder = ref.workload_case(spec)
            self.topology = self.holder.topology
            s = self.holder.summary
            self.storage_size = int(s["storage"])
            bs3 = spec.brick_size ** 3
            structured = sum(self.topology.levels[l].brick_count for l in range(self.topology.level_count)) * bs3
            active = self.holder.active.astype(bool)
            self.leaf_cells = int(active[:structured].sum())
            self.counts = {"grid": "cut-cell (reference preprocessing)", "eb_fragments": int(self.storage_size - structured),
                           "active_dofs": int(s["active"]), "coarse_fine_edges": int(s["coarse_fine"]),
                           "embedded_edges": int(s["embedded"]), "wls_gradient_nodes": int(s["gradient_nodes"]),
                           "surface_patches": int(s["patches"])}
            self.min_volume_fraction = spec.min_volume_fraction
        else:
            self.holder = spec.build()
            self.topology = self.holder.topology
            self.storage_size = self.holder.storage_size
            self.leaf_cells = self.holder.leaf_cells
            self.counts = {"grid": "staircase (pcfd_topology_build)"}
            self.min_volume_fraction = 0.0

    def close(self):
        if self.holder is not None:
            self.holder.close()
            self.holder = None


# ------------------------------------------------------------------------------------------ CPU steps
# Whole CPU steps of a 16 M-cell grid take minutes each, so the CPU timings run whole steps of the
# same wing on a smaller grid of the same family and scale by the DOF count.
CPU_SAMPLE = {"paraglider16m": "paraglider1m", "paraglider5m": "paraglider1m"}


class CpuStepper:
    """Whole time steps of the reference's host implementation on one grid.

    ExternalAeroCore::step's sequence (external_aero_core.cpp:304-328) with the reference's own CPU
    twins (oracle/_ref, single-threaded as written): outflow-rate CFL reduction, MUSCL transport,
    Smagorinsky diffusion, smooth wall, cell-to-face reconstruction, the external boundaries of
    amr_fields.cu:86-118 (X-min inflow, Y/Z free slip; restated below on the compact faces),
    projection RHS, the pressure solve, flux correction, pressure traction, surface loads.  The
    reference has no CPU pressure solver: the solve to the case tolerance is the FP64 OpenMP
    restatement of its own solver (reference multigrid cycle, flexible GCRO; oracle/pcfd_oracle.cpp),
    warm-started from the previous pressure like the reference's.  ``initialize`` follows
    ExternalAeroCore::initialize (external_aero_core.cpp:245-302)."""

    def __init__(self, grid: Grid):
        from oracle import port
        self.grid, self.spec = grid, grid.spec
        self.rc = grid.holder
        self.ps = port.PortSystem(grid.topology)
        self.threads = port.threads()
        t = grid.topology
        self.bs = bs = t.brick_size
        self.h = t.levels[t.level_count - 1].h
        flags = np.concatenate([np.ctypeslib.as_array(t.levels[l].flags, shape=(t.levels[l].brick_count,))
                                for l in range(t.level_count)])
        from paracfd_b200 import capi
        live = (flags & capi.BRICK_COVERED) == 0
        per = (bs + 1) * bs * bs
        a, b = np.meshgrid(np.arange(bs), np.arange(bs), indexing="ij")
        a, b = a.ravel(), b.ravel()

        def faces(mask, index):
            slots = np.nonzero(live & ((flags & mask) != 0))[0]
            return (slots[:, None] * per + index[None, :]).ravel()
        # compact layouts: u (k*bs+j)*(bs+1)+i, v (k*(bs+1)+j)*bs+i, w (k*bs+j)*bs+i
        self.xmin = faces(capi.BRICK_XMIN, (b * bs + a) * (bs + 1))
        self.ywall = np.concatenate([faces(capi.BRICK_YMIN, (b * (bs + 1)) * bs + a),
                                     faces(capi.BRICK_YMAX, (b * (bs + 1) + bs) * bs + a)])
        self.zwall = np.concatenate([faces(capi.BRICK_ZMIN, a * bs + b),
                                     faces(capi.BRICK_ZMAX, bs * bs * bs + a * bs + b)])
        self.n = self.rc.n
        self.pressure = np.zeros(self.n)
        self.faces = None
        self.state = None

    def close(self):
        self.ps.close()

    def boundaries(self, faces):
        u, v, w, cf, eb = faces
        u[self.xmin] = self.spec.speed
        v[self.ywall] = 0.0
        w[self.zwall] = 0.0
        return u, v, w, cf, eb

    def initialize(self) -> dict:
        rc, spec, case = self.rc, self.spec, self.spec.case
        t = self.grid.topology
        active = rc.active.astype(bool)
        connected = np.ctypeslib.as_array(t.freestream_connected, shape=(self.n,)).astype(bool)
        x = np.where(active & connected, spec.speed, 0.0).astype(np.float32)
        self.state = (x, np.zeros(self.n, np.float32), np.zeros(self.n, np.float32))
        zeros = np.zeros(rc.faces, np.float32)
        self.faces = self.boundaries(rc.reconstruct(self.state, zeros, zeros, zeros))
        dt = case["cfl"] * self.h / max(1e-9, abs(spec.speed))
        return self._project(dt, warm=False)

    def _project(self, dt: float, warm: bool) -> dict:
        rc, case = self.rc, self.spec.case
        rhs = rc.rhs(*self.faces, case["rho"], dt)
        p, info = self.ps.solve(rhs, case["projection_tolerance"], case["projection_max_iterations"],
                                x0=self.pressure if warm else None)
        self.pressure = p
        self.faces = rc.correct_fluxes(p, case["rho"], dt, *self.faces)
        if info["converged"]:
            self.state = rc.impulse(p, dt, case["rho"], self.state, True)
        return dict(info, dt=dt)

    def step(self) -> dict:
        rc, spec, case = self.rc, self.spec, self.spec.case
        rate = rc.outflow_rate(*self.faces, True)
        dt = case["cfl"] / max(1e-9, abs(spec.speed) / self.h, rate)
        self.state = rc.transport(*self.faces, dt, self.state, True, spec.speed)
        self.state = rc.diffuse_smagorinsky(self.state, case["nu"], case["smagorinsky_cs"], dt)
        self.state, _ = rc.wall(self.state, case["nu"], dt, case["rho"])
        self.faces = self.boundaries(rc.reconstruct(self.state, *self.faces[:3]))
        info = self._project(dt, warm=True)
        info["loads"] = rc.pressure_loads(self.pressure)
        return info


def cpu_steps(spec, warmup: int, steps: int) -> dict:
    """Times whole CPU steps (CpuStepper) on the workload's CPU sample grid; the value is scaled to
    the workload's DOF count.  Returns the cpu_baseline fields."""
    from paracfd_b200.workloads import WORKLOADS
    sample_name = CPU_SAMPLE.get(spec.name, spec.name)
    sample = Grid(WORKLOADS[sample_name], "cutcell")
    stepper = CpuStepper(sample)
    t0 = time.perf_counter()
    init = stepper.initialize()
    init_s = time.perf_counter() - t0
    for _ in range(warmup):
        stepper.step()
    times, iterations, converged = [], [], 0
    for _ in range(steps):
        t0 = time.perf_counter()
        info = stepper.step()
        times.append(time.perf_counter() - t0)
        iterations.append(info["iterations"])
        converged += int(info["converged"])
    stepper.close()
    sample_dofs = sample.storage_size
    sample.close()
    return {"sample_workload": sample_name, "sample_storage": sample_dofs, "step_s": times,
            "iterations": iterations, "converged_steps": converged, "init_s": init_s,
            "init_iterations": init["iterations"], "threads": stepper.threads}


# ------------------------------------------------------------------------------------------ arms
def make_system(args, grid: Grid, device: int):
    from paracfd_b200 import MG_FP32, MG_FP64, CompositeSystem
    return CompositeSystem(grid.topology, MG_FP32 if args.mg == "fp32" else MG_FP64, device=device,
                           momentum_min_volume_fraction=grid.min_volume_fraction,
                           mg_cycle={"reference": 0, "corrected": 1, "composite": 2}[args.mg_cycle],
                           gmres_restart=args.restart, mg_stage_sweeps=args.stage_sweeps,
                           mg_block_iterations=args.block_iterations, mg_stage_chebyshev=args.chebyshev,
                           mg_fine_chebyshev=args.fine_chebyshev, gmres_delayed=args.delayed,
                           gmres_recycle=args.recycle, mg_stage_fp16=args.stage_fp16)


def line_config(args, grid: Grid, n: int) -> dict:
    """The config object both arms print (same workload, same grid)."""
    spec = grid.spec
    return dict(spec.describe(), leaf_cells=grid.leaf_cells, storage=grid.storage_size, **grid.counts,
                mg=args.mg, mg_cycle=args.mg_cycle, gcro_restart=args.restart or 24,
                stage_sweeps=args.stage_sweeps or 6, block_iterations=args.block_iterations,
                stage_smoother="jacobi" if args.chebyshev == 1 else f"chebyshev 2/{args.chebyshev or 30}",
                fine_smoother="jacobi" if args.fine_chebyshev == 1 else f"chebyshev-richardson 2/{args.fine_chebyshev or 10}",
                orthogonalisation="delayed CGS2" if args.delayed else "CGS2",
                recycled_pairs=3 if args.recycle == 0 else max(args.recycle, 0),
                stage_coefficients="fp16" if args.stage_fp16 else args.mg,
                parallelism=f"replicas{n}", l2="inputs larger than L2")


METRIC = "AMR steps/s at 16M cells (projection to 1e-8, loads every step)"


def cpu_baseline_fields(spec, grid: Grid, timing: dict) -> dict:
    """cpu_baseline of a cpu_steps() timing: steps/s scaled from the sample grid to the workload."""
    mean_s = statistics.mean(timing["step_s"])
    scale = grid.storage_size / timing["sample_storage"]
    return {
        "value": round(1.0 / (mean_s * scale), 6), "unit": "steps/s", "cores": timing["threads"], "kind": "reference",
        "sample": (f"{len(timing['step_s'])} whole CPU time steps (after the initial projection and the warm-up "
                   f"steps) of the same wing on the {timing['sample_workload']} cut-cell grid "
                   f"({timing['sample_storage']} DOFs): the reference's CPU twins of every stage (1 thread) and "
                   f"its solver restated in FP64 OpenMP ({timing['threads']} threads) to the case tolerance; "
                   f"mean {mean_s:.3f} s per step scaled by the DOF ratio {scale:.2f} to this grid (the "
                   f"solver's iteration count grows with the grid, so the scaled CPU figure is optimistic)"),
        "sample_step_s": round(mean_s, 4), "sample_iterations_per_step": round(statistics.mean(timing["iterations"]), 2),
        "sample_converged_steps": timing["converged_steps"]}


def run_ours(args, ranks: Ranks):
    from paracfd_b200.workloads import WORKLOADS

    spec = WORKLOADS[args.workload]
    grid = Grid(spec, args.grid)
    bricks = non_covered_bricks(grid.topology)
    system = make_system(args, grid, ranks.local)
    system.configure(speed=spec.speed, **spec.case)
    system.set_initial_guess({"previous": 0, "extrapolated": 1, "quadratic": 2}[args.initial_guess])
    tune = system.autotune(5) if not args.no_autotune else None
    slots = system.inflow_layout()
    faces = len(slots) * spec.brick_size ** 2
    centres = inflow_face_centres(grid.topology, slots)
    system.set_inflow(inflow_profile(spec.speed, centres, 0))
    init = system.initialize()
    stats = []
    failed = 0

    def one_step():
        nonlocal failed
        st = system.step()
        system.loads()
        failed += 0 if st["pressure"]["converged"] else 1
        return st

    for _ in range(args.warmup):
        one_step()
    # ---- device-timed region: state resident in HBM
    capacity = 1 << 16
    ranks.barrier()
    system.synchronize()
    launches0 = system.launch_count()
    system.profile_begin(args.profile_region, capacity)
    with ClockSampler(ranks.local) as clocks:
        system.event_record(0)
        for _ in range(args.steps):
            stats.append(one_step())
        system.event_record(1)
        system.synchronize()
    elapsed_ms = system.event_elapsed(0, 1)
    per_launch = system.profile_end(capacity)
    launches = system.launch_count() - launches0
    ranks.barrier()
    elapsed_ms = ranks.max(elapsed_ms)
    # ---- end-to-end through the public API with host buffers
    import torch
    pinned = torch.empty(max(faces, 1), dtype=torch.float32, pin_memory=True)
    host_inflow = pinned.numpy()
    profiles = [inflow_profile(spec.speed, centres, s + 1) for s in range(args.steps)]
    loads_out = []
    ranks.barrier()
    system.synchronize()
    t0 = time.perf_counter()
    for s in range(args.steps):
        host_inflow[:faces] = profiles[s]
        system.set_inflow(host_inflow[:faces])
        st = system.step()
        loads_out.append(system.loads(reference_area=1.0))
        failed += 0 if st["pressure"]["converged"] else 1
    system.synchronize()
    e2e_s = ranks.max(time.perf_counter() - t0)

    # the dominant kernel (the composite cycle's first-stage Chebyshev smoothing, launched from a
    # captured graph in the timed steps): per-launch CUDA events over a few more whole steps with
    # the stage chain launched uncaptured, so each of its launches gets an event pair
    stage_launches = np.zeros(0)
    if args.mg_cycle == "composite":
        system.profile_begin(2, capacity)
        for _ in range(min(3, args.steps)):
            one_step()
        stage_launches = system.profile_end(capacity)
    stage_bytes = system.profile_bytes(2) if len(stage_launches) else 0.0
    stage_kernel = ("brick_stage_chebyshev_kernel (first composite stage, 64 rows per 8^3 brick, one Chebyshev step)"
                    if system.stage_brick_structured else
                    "algebraic_chebyshev_kernel (first composite stage as CSR, one Chebyshev step)")

    # isolated per-component device times on the same resident system (not part of the timed region)
    components = {0: "apply_full", 1: "apply_orthogonal", 2: "preconditioner", 3: "divergence", 4: "flux_correction",
                  5: "dot", 6: "mg_presmooth", 7: "mg_coarse_correction", 8: "mg_postsmooth", 9: "gcro_column_orth_m16",
                  10: "fused_presmooth", 11: "fused_restrict", 12: "mg_hierarchy", 13: "fused_prolong_postsmooth",
                  14: "gcro_column_orth_m8", 15: "gcro_column_orth_m27"}
    kernel_ms = {}
    for which, name in components.items():
        try:
            kernel_ms[name] = round(system.time_kernel(which, 10), 4)
        except Exception:
            pass

    n = ranks.world
    value = replica_throughput(n, args.steps, elapsed_ms)
    peak, peak_kind = measured_peak_gbs()
    region_names = {0: "brick_pipe_kernel<2> (FP64 structured 7-point operator)", 1: "MG preconditioner application"}
    roofline, roofline_operator = None, None
    region_ms = round(float(np.mean(per_launch)), 4) if len(per_launch) else None
    if len(per_launch) and args.profile_region == 0:
        avg_ms = float(np.mean(per_launch))
        algorithmic = A_P_BYTES_PER_DOF * bricks * spec.brick_size ** 3
        achieved = algorithmic / (avg_ms * 1e-3) / 1e9
        roofline_operator = {"bound": "hbm", "kernel": region_names[0], "achieved": round(achieved, 1), "peak": peak,
                             "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                             "traffic": DRAM_BYTES_PER_LAUNCH.get((args.workload, args.grid, 1)),
                             "algorithmic_bytes_per_launch": algorithmic, "launches_timed": int(len(per_launch)),
                             "avg_launch_us": round(avg_ms * 1e3, 2)}
    if len(stage_launches):
        avg_ms = float(np.mean(stage_launches))
        achieved = stage_bytes / (avg_ms * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": stage_kernel,
                    "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                    "peak_kind": peak_kind,
                    "traffic": DRAM_BYTES_PER_LAUNCH.get((args.workload, args.grid, 17, system.stage_brick_structured)),
                    "algorithmic_bytes_per_launch": int(stage_bytes), "launches_timed": int(len(stage_launches)),
                    "avg_launch_us": round(avg_ms * 1e3, 2),
                    "timing": "CUDA events around each launch over 3 whole steps after the timed region (stage chain "
                              "launched uncaptured)"}
    # the Krylov orthogonalisation (a quarter of the step): one delayed-CGS2 column against 13 basis
    # vectors on the resident system, its algorithmic bytes from the library
    roofline_orthogonalisation = None
    try:
        column_ms = system.time_kernel(18, 10)
        column_bytes = system.profile_bytes(3)
        achieved = column_bytes / (column_ms * 1e-3) / 1e9
        roofline_orthogonalisation = {
            "bound": "hbm", "kernel": "delayed CGS2 column against 13 basis vectors (dcgs_dot_kernel, dcgs_final_kernel, "
                                      "dcgs_update_kernel)",
            "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "peak_kind": peak_kind, "algorithmic_bytes_per_launch": int(column_bytes), "avg_launch_us": round(column_ms * 1e3, 2),
            "timing": "CUDA events over 10 back-to-back columns on resident vectors, after the timed region"}
    except Exception:
        pass
    line = {
        "metric": METRIC,
        "value": round(value, 4), "unit": "steps/s", "n_gpus": n, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(elapsed_ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 state / f64 pressure", "data": "synthetic analytic geometry",
        "config": line_config(args, grid, n),
        "projection_ms": round(statistics.mean(s["projection_ms"] for s in stats), 3),
        "iterations_per_step": round(statistics.mean(s["pressure"]["iterations"] for s in stats), 2),
        "initial_guess": {"previous": "last pressure (the reference's warm start)",
                          "extrapolated": "2 p_n - p_(n-1) of the last two converged pressures",
                          "quadratic": "3 p_n - 3 p_(n-1) + p_(n-2) of the last three converged pressures"}[args.initial_guess],
        "final_residual_max": max(s["pressure"]["relative_residual"] for s in stats),
        "unconverged_steps": failed,
        "init_projection": {"iterations": init["pressure"]["iterations"], "ms": round(init["projection_ms"], 3)},
        "clocks": clocks.summary(),
        "e2e": {"value": round(n * args.steps / e2e_s, 4), "unit": "steps/s", "h2d_bytes_per_step": 4 * faces,
                "d2h_bytes_per_step": 12 * 8},
        "gpu_launches": int(launches),
        "launches_before_timed": int(launches0),
        "component_ms": kernel_ms,
        "roofline": roofline,
        "roofline_operator": roofline_operator,
        "roofline_orthogonalisation": roofline_orthogonalisation,
        "profiled_region": {"region": region_names.get(args.profile_region), "launches": int(len(per_launch)),
                            "avg_ms": region_ms},
        "cpu_baseline": None,
        "autotune": tune,
    }
    system.close()
    if ranks.rank == 0 and n == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline_fields(spec, grid, cpu_steps(spec, 1, 3))
        except Exception as exc:   # the CPU sample must not hide the GPU result
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    grid.close()
    if ranks.rank == 0 and n == 1 and not args.no_sweep_summary:
        # one batch of the angle sweep (4 instances) beside the headline
        try:
            short = argparse.Namespace(**{**vars(args), "steps": 3, "warmup": 1})
            line["sweep"] = run_sweep(short, ranks, batches=1)
        except Exception as exc:
            line["sweep"] = {"error": str(exc)[:200]}
    if ranks.rank == 0 and n == 1 and not args.no_learned:
        # the learned-preconditioner comparison (a short --learned run) beside the headline
        try:
            short = argparse.Namespace(**{**vars(args), "harvest_runs": 2, "train_steps": 1500, "steps": 2, "warmup": 2})
            line["learned"] = run_learned(short, ranks)
        except Exception as exc:
            line["learned"] = {"error": str(exc)[:200]}
    return line


def run_kernel_only(args):
    from paracfd_b200.workloads import WORKLOADS
    spec = WORKLOADS[args.workload]
    grid = Grid(spec, args.grid)
    system = make_system(args, grid, 0)
    ms = system.time_kernel(args.kernel_only, args.kernel_iterations)
    line = {"kernel_only": args.kernel_only, "workload": args.workload, "grid": args.grid, "ms_per_launch": ms,
            "iterations": args.kernel_iterations, "launches": system.launch_count()}
    system.close()
    grid.close()
    return line


def run_reference(args, ranks: Ranks):
    """The reference arm: whole CPU time steps of the reference's host implementation (CpuStepper
    on the workload's CPU sample grid, scaled to the workload), and whole steps of the reference's
    own sm_100a build on the full workload.  Loads only oracle/_ref libraries."""
    from paracfd_b200.workloads import WORKLOADS
    if ranks.rank != 0:
        return None
    spec = WORKLOADS[args.workload]
    if args.grid != "cutcell":
        raise SystemExit("the reference arm runs on the reference's own cut-cell grid (--grid cutcell)")
    grid = Grid(spec, "cutcell")
    case = spec.case
    gpu = None
    if not args.no_reference_gpu:
        try:
            from oracle import ref
            core = ref.RefDeviceCore(grid.holder, spec.speed, case["rho"], case["nu"], case["cfl"], case["smagorinsky_cs"],
                                     case["projection_tolerance"], case["projection_max_iterations"],
                                     grid.min_volume_fraction)
            init = core.initialize()
            for _ in range(args.warmup):
                core.step()
            t0 = time.perf_counter()
            st = [core.step() for _ in range(args.steps)]
            wall_s = time.perf_counter() - t0
            core.close()
            step_ms = statistics.mean(s["gpu_step_ms"] for s in st)
            gpu = {"steps_per_s": round(args.steps / wall_s, 4), "ms_per_step": round(1e3 * wall_s / args.steps, 3),
                   "gpu_step_ms": round(step_ms, 3), "steps": args.steps, "warmup": args.warmup,
                   "projection_ms": round(statistics.mean(s["projection_ms"] for s in st), 3),
                   "iterations_per_step": round(statistics.mean(s["iterations"] for s in st), 2),
                   "converged_steps": sum(bool(s["converged"]) for s in st),
                   "init_iterations": init["iterations"],
                   "timing": "host clock around K whole synchronous steps (the reference synchronises every stage)",
                   "build": "reference sources compiled for sm_100a (oracle/_ref): its DeviceAmrFields, "
                            "DeviceCompositeAmrProjection and DeviceCompositeCellMomentumTransport in "
                            "ExternalAeroCore::step's sequence"}
        except Exception as exc:
            gpu = {"unavailable": str(exc)[:200]}
    t0 = time.perf_counter()
    timing = cpu_steps(spec, args.warmup, args.steps)
    cpu_wall = time.perf_counter() - t0
    cpu = cpu_baseline_fields(spec, grid, timing)
    sample_ms = 1e3 * statistics.mean(timing["step_s"])
    line = {
        "metric": METRIC, "impl": "reference",
        "value": cpu["value"], "unit": "steps/s", "n_gpus": ranks.world, "steps": args.steps, "warmup": args.warmup,
        # each timed step is a whole step of the sample grid: ms_per_step x steps is the timed CPU region
        "ms_per_step": round(sample_ms, 1),
        "full_grid_ms_per_step_equivalent": round(1e3 / cpu["value"], 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state / f64 pressure", "data": "synthetic analytic geometry",
        "config": line_config(args, grid, ranks.world),
        "cpu_baseline": cpu,
        "cpu_wall_s": round(cpu_wall, 1),
        "e2e": {"value": cpu["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_sm100a": gpu,
    }
    grid.close()
    return line


# Network FLOPs per brick as the oracle defines it (oracle/unet.py LAYERS): 2*27*Cin*Cout per
# output voxel of every convolution, plus the 16-wide head.
LEARNED_FLOPS_PER_BRICK = 2 * 27 * (16 * 16 * 512 + 16 * 32 * 64 + 32 * 64 * 8 + 96 * 32 * 64 + 48 * 16 * 512) + 2 * 16 * 512


def measured_peak_tflops() -> tuple[float, str]:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def run_learned(args, ranks: Ranks):
    """Projection time to 1e-8 under the learned preconditioner forms against the multigrid one,
    on the same right-hand sides (state snapshots of the naca4412_wing run)."""
    from paracfd_b200 import (LEARNED_TARGET_BRICK_SOLVE, MG_CYCLE_COMPOSITE, PRECONDITIONER_LEARNED,
                              PRECONDITIONER_LEARNED_MULTIGRID, PRECONDITIONER_MULTIGRID, CompositeSystem)
    from paracfd_b200.workloads import WORKLOADS, with_aoa

    rng = np.random.default_rng(20261203)
    harvest = []
    t0 = time.time()
    pairs_per_run = 4000 // max(args.harvest_runs, 1)
    for k in range(args.harvest_runs):
        name = ("naca0012_slab", "naca4412_wing")[k % 2]
        spec = with_aoa(name, float(rng.uniform(0.0, 10.0)))
        built = Grid(spec, args.grid)
        with CompositeSystem(built.topology, device=ranks.local, mg_cycle=MG_CYCLE_COMPOSITE,
                             momentum_min_volume_fraction=built.min_volume_fraction) as system:
            system.configure(speed=spec.speed, **spec.case)
            system.initialize()
            system.harvest_begin(capacity_pairs=4000, bricks_per_pair=32, seed=1000 + k, target=LEARNED_TARGET_BRICK_SOLVE)
            before = system.harvest_stop()
            system.harvest_begin(capacity_pairs=4000, bricks_per_pair=32, seed=1000 + k, target=LEARNED_TARGET_BRICK_SOLVE)
            steps = 0
            while steps < 400:
                system.step()
                steps += 1
                if system.harvest_stop() - before >= pairs_per_run * 32:
                    break
                system.harvest_begin(capacity_pairs=4000, bricks_per_pair=32, seed=1000 + k, target=LEARNED_TARGET_BRICK_SOLVE)
            samples = system.harvest_stop()
        harvest.append({"case": name, "aoa": round(spec.aoa, 3), "steps": steps, "samples": samples - before})
        built.close()
    harvest_s = time.time() - t0

    spec = WORKLOADS["naca4412_wing"]
    built = Grid(spec, args.grid)
    system = CompositeSystem(built.topology, device=ranks.local, mg_cycle=MG_CYCLE_COMPOSITE,
                             momentum_min_volume_fraction=built.min_volume_fraction)
    system.configure(speed=spec.speed, **spec.case)
    system.initialize()
    t0 = time.time()
    loss = system.train(args.train_steps, batch=64, learning_rate=2e-3, seed=7)
    system.synchronize()
    train_s = time.time() - t0
    forward_ms = system.time_kernel(16, 10)
    bricks = non_covered_bricks(built.topology)
    peak, peak_kind = measured_peak_tflops()
    achieved = LEARNED_FLOPS_PER_BRICK * bricks / (forward_ms * 1e-3) / 1e12

    kinds = {"multigrid": PRECONDITIONER_MULTIGRID, "learned_multigrid": PRECONDITIONER_LEARNED_MULTIGRID,
             "learned": PRECONDITIONER_LEARNED}
    results = {k: {"ms": [], "iterations": [], "residual": [], "fallbacks": 0} for k in kinds}
    system.keep_projection_start(True)
    for step in range(args.warmup + args.steps):
        system.step()
        if step < args.warmup:
            continue
        # the step's own projection solved again from its saved start (same right-hand side, warm
        # start and recycled subspace) under each preconditioner
        for name, kind in kinds.items():
            system.set_preconditioner(kind)
            ms, res = system.resolve_projection(1e-8, 600)
            r = results[name]
            r["ms"].append(ms)
            r["iterations"].append(res["iterations"])
            r["residual"].append(res["relative_residual"])
            r["fallbacks"] += res["fallback_solves"]
        system.set_preconditioner(PRECONDITIONER_MULTIGRID)
        system.resolve_projection(1e-8, 600)   # leave the multigrid solve's pressure and subspace
    summary = {k: {"projection_ms": round(statistics.mean(v["ms"]), 3), "iterations": round(statistics.mean(v["iterations"]), 2),
                   "final_residual_max": max(v["residual"]), "fallbacks": v["fallbacks"]} for k, v in results.items()}
    mg_ms = summary["multigrid"]["projection_ms"]
    line = {
        "metric": "projection time to 1e-8 relative residual, learned (NN) vs multigrid preconditioner",
        "value": summary["learned_multigrid"]["projection_ms"], "unit": "ms", "higher_is_better": False,
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "vs_multigrid": round(mg_ms / summary["learned_multigrid"]["projection_ms"], 3),
        "dtype": "bf16 network / f64 Krylov", "data": "synthetic analytic geometry",
        "config": dict(spec.describe(), leaf_cells=built.leaf_cells, **built.counts, bricks=bricks, mg_cycle="composite",
                       harvest_target="brick solve", train_steps=args.train_steps, batch=64),
        "preconditioners": summary,
        "harvest": harvest, "harvest_s": round(harvest_s, 1), "train_s": round(train_s, 1), "train_loss": loss,
        "network": {"forward_ms": round(forward_ms, 3), "flops_per_brick": LEARNED_FLOPS_PER_BRICK,
                    "roofline": {"bound": "tensor", "achieved": round(achieved, 1), "peak": peak, "unit": "TFLOP/s",
                                 "frac": round(achieved / peak, 4), "peak_kind": peak_kind}},
    }
    system.close()
    built.close()
    return line


def run_sweep(args, ranks: Ranks, batches: int = 4):
    """BASELINE config 5 on one GPU: the angle-of-attack sweep as batches of concurrent instances
    (the first `batches` of the 4 batches of 4)."""
    from concurrent.futures import ThreadPoolExecutor

    from paracfd_b200 import MG_CYCLE_COMPOSITE, MG_FP32, CompositeSystem
    from paracfd_b200.workloads import sweep_instances

    specs = sweep_instances()[:4 * batches]
    batches = []
    for first in range(0, len(specs), 4):
        batch = specs[first:first + 4]
        builts = [Grid(sp, args.grid) for sp in batch]
        systems = [CompositeSystem(b.topology, MG_FP32, device=ranks.local, mg_cycle=MG_CYCLE_COMPOSITE,
                                   momentum_min_volume_fraction=b.min_volume_fraction,
                                   mg_stage_sweeps=args.stage_sweeps, mg_stage_chebyshev=args.chebyshev,
                                   mg_fine_chebyshev=args.fine_chebyshev, gmres_delayed=args.delayed,
                             gmres_recycle=args.recycle, mg_stage_fp16=args.stage_fp16) for b in builts]
        tuned = []
        for sp, sy in zip(batch, systems):
            sy.configure(speed=sp.speed, **sp.case)
            tuned.append(sy.autotune(3)["chosen"] if not args.no_autotune else None)
            sy.initialize()
            for _ in range(args.warmup):
                sy.step()
            sy.synchronize()

        def run(sy):
            its = 0
            for _ in range(args.steps):
                its += sy.step()["pressure"]["iterations"]
            sy.synchronize()
            return its

        sequential = []
        for sy in systems:
            t0 = time.perf_counter()
            run(sy)
            sequential.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=len(systems)) as pool:
            iterations = list(pool.map(run, systems))
        concurrent = time.perf_counter() - t0
        batches.append({"aoa": [sp.aoa for sp in batch], "leaf_cells": [b.leaf_cells for b in builts],
                        "sequential_s": round(sum(sequential), 3), "concurrent_s": round(concurrent, 3),
                        "iterations_per_step": [round(i / args.steps, 2) for i in iterations],
                        "autotuned_ctas_per_sm": tuned})
        for sy in systems:
            sy.close()
        for b in builts:
            b.close()
    instance_steps = len(specs) * args.steps
    seq = sum(b["sequential_s"] for b in batches)
    conc = sum(b["concurrent_s"] for b in batches)
    return {
        "metric": f"batched angle sweep: instance-steps/s over {len(specs)} naca4412_wing instances "
                  f"({len(batches)} batch{'es' if len(batches) > 1 else ''} of 4)",
        "value": round(instance_steps / conc, 3), "unit": "instance-steps/s", "higher_is_better": True, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "sequential": round(instance_steps / seq, 3),
        "speedup_vs_sequential": round(seq / conc, 3), "timing": "host wall clock around synchronised step loops",
        "config": {"workload": "naca4412_wing sweep", "aoa": [-4, 11], "seed": 20261203, "mg": "fp32",
                   "leaf_cells_per_batch": [sum(b["leaf_cells"]) for b in batches]},
        "batches": batches,
    }


def main():
    args = parse_args()
    ranks = Ranks(collective=args.impl == "ours")
    try:
        if args.learned:
            line = run_learned(args, ranks) if ranks.rank == 0 else None
        elif args.sweep:
            line = run_sweep(args, ranks) if ranks.rank == 0 else None
        elif args.kernel_only is not None:
            line = run_kernel_only(args)
        elif args.impl == "reference":
            line = run_reference(args, ranks)
        else:
            line = run_ours(args, ranks)
        if ranks.rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
