#!/usr/bin/env python3
"""Time-step throughput of the ParaCFD per-timestep solver path on B200.

Workload: the 4-level ~16 M leaf-cell paraglider case (``paraglider16m``, FP32 flow state, FP64
pressure, projection to 1e-8 relative residual, surface loads integrated every step).  A step
is one ``pcfd_core_step`` (CFL -> MUSCL transport -> Smagorinsky diffusion -> smooth wall ->
flux reconstruction -> boundaries -> projection -> pressure traction) plus ``pcfd_core_loads``.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Arms
  ours       value = steps/s over K steps with the state resident in HBM (CUDA events on the
             system stream, max over ranks); e2e = steps/s over K more steps through the public
             API with host buffers: per step the X-min inflow profile is copied from pinned host
             memory and the loads are read back.  Every resident vector (19 M-DOF FP64 pressure
             vectors, 0.2 GB each) is larger than the 126 MB L2.
  reference  the reference's own host implementation of the step on this machine's cores
             (oracle/_ref: its CPU twins of every operator, timed at full size) with the
             projection from the FP64 OpenMP restatement of its solver; see cpu_step_sample.
Multi-GPU: independent replicas, one per rank (the path has no exchange step).

Solver defaults of the ours arm: the composite multigrid cycle in FP32 with FP16 stage
coefficients (Chebyshev stage smoothing, Chebyshev-Richardson fine steps, exact coarsest stage),
flexible GMRES with delayed CGS2 and no recycled subspace; --mg-cycle reference --mg fp64
--delayed 0 --recycle 0 selects the reference's solver configuration.  The line also carries a short learned-preconditioner
comparison (skip with --no-learned).  Other modes:
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
    ap.add_argument("--mg", choices=("fp64", "fp32"), default="fp32",
                    help="multigrid preconditioner precision (the composite stages; fine sweeps and Krylov stay FP64)")
    ap.add_argument("--restart", type=int, default=0, help="GCRO columns per cycle (0: the reference's 24)")
    ap.add_argument("--mg-cycle", choices=("reference", "corrected", "composite"), default="composite",
                    help="coarse-correction weighting of the multigrid cycle (pcfd_mg_cycle)")
    ap.add_argument("--stage-sweeps", type=int, default=0,
                    help="composite cycle: smoothing steps per stage before and after its correction (0: 6)")
    ap.add_argument("--chebyshev", type=int, default=0,
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
        self.path = path or os.path.join(ROOT, "gpurun_out", f"clocks_rank{device}.csv")

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


def ncu_traffic(workload: str) -> float | None:
    """DRAM bytes (read + write) per launch of the structured operator kernel, from the committed
    ncu summary ``profiles/brick_apply_<workload>.md`` (line ``bytes_per_launch: N``), if present."""
    path = os.path.join(ROOT, "profiles", f"brick_apply_{workload}.md")
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith("bytes_per_launch:"):
                    return float(line.split(":", 1)[1].strip().split()[0])
    except (OSError, ValueError):
        pass
    return None


# ------------------------------------------------------------------------------------------ CPU sample
class CpuReference:
    """The reference's host implementation of one time step on the full workload.

    Every operator of the step is the reference's own CPU twin (oracle/_ref, single-threaded as
    the reference wrote it): outflow-rate reduction, MUSCL transport, Smagorinsky diffusion,
    smooth wall, flux reconstruction, projection RHS, flux correction, pressure traction and
    surface loads.  The reference has no CPU pressure solver; the projection is the FP64 OpenMP
    restatement of its solver (oracle/pcfd_oracle.cpp).  Stages run on fixed inputs derived
    from the freestream initial state (their cost does not depend on the values).
    """

    STAGES = ("outflow_rate", "transport", "diffusion", "wall", "reconstruct", "rhs", "correct", "impulse", "loads")

    def __init__(self, topology, spec):
        from oracle import port, ref
        self.spec = spec
        self.rc = rc = ref.import_topology(topology)
        self.ps = port.PortSystem(topology)
        self.threads = port.threads()
        n = rc.n
        active = rc.active.astype(bool)
        connected = np.ctypeslib.as_array(topology.freestream_connected, shape=(n,)).astype(bool)
        x = np.where(active & connected, spec.speed, 0.0).astype(np.float32)
        self.state = (x, np.zeros(n, np.float32), np.zeros(n, np.float32))
        zeros = np.zeros(rc.faces, np.float32)
        self.faces = rc.reconstruct(self.state, zeros, zeros, zeros)
        rate = rc.outflow_rate(*self.faces, True)
        h = topology.levels[topology.level_count - 1].h
        self.dt = spec.case["cfl"] / max(1e-9, spec.speed / h, rate)
        self.rhs = rc.rhs(*self.faces, spec.case["rho"], self.dt)
        self.pressure = np.zeros(n)
        self.per_iteration_s = None
        self.solver_iterations = None

    def close(self):
        self.ps.close()
        self.rc.close()

    def time_solver(self, max_iterations: int) -> dict:
        """Restated FP64 solve of the step's RHS from zero, capped at ``max_iterations``."""
        case = self.spec.case
        t0 = time.perf_counter()
        self.pressure, info = self.ps.solve(self.rhs, case["projection_tolerance"], max_iterations)
        elapsed = time.perf_counter() - t0
        self.per_iteration_s = elapsed / max(1, info["iterations"])
        self.solver_iterations = info["iterations"]
        return dict(info, seconds=elapsed)

    def stage(self, name: str) -> float:
        rc, case, (u, v, w, cf, eb), st = self.rc, self.spec.case, self.faces, self.state
        nu, rho, dt = case["nu"], case["rho"], self.dt
        calls = {
            "outflow_rate": lambda: rc.outflow_rate(u, v, w, cf, eb, True),
            "transport": lambda: rc.transport(u, v, w, cf, eb, dt, st, True, self.spec.speed),
            "diffusion": lambda: rc.diffuse_smagorinsky(st, nu, case["smagorinsky_cs"], dt),
            "wall": lambda: rc.wall(st, nu, dt, rho),
            "reconstruct": lambda: rc.reconstruct(st, u, v, w),
            "rhs": lambda: rc.rhs(u, v, w, cf, eb, rho, dt),
            "correct": lambda: rc.correct_fluxes(self.pressure, rho, dt, u, v, w, cf, eb),
            "impulse": lambda: rc.impulse(self.pressure, dt, rho, st, True),
            "loads": lambda: rc.pressure_loads(self.pressure),
        }
        t0 = time.perf_counter()
        calls[name]()
        return time.perf_counter() - t0


# ------------------------------------------------------------------------------------------ arms
def run_ours(args, ranks: Ranks):
    import ctypes as C

    from paracfd_b200 import MG_FP32, MG_FP64, CompositeSystem
    from paracfd_b200.workloads import WORKLOADS

    spec = WORKLOADS[args.workload]
    built = spec.build()
    bricks = non_covered_bricks(built.topology)
    system = CompositeSystem(built.topology, MG_FP32 if args.mg == "fp32" else MG_FP64, device=ranks.local,
                             mg_cycle={"reference": 0, "corrected": 1, "composite": 2}[args.mg_cycle],
                             gmres_restart=args.restart, mg_stage_sweeps=args.stage_sweeps,
                             mg_block_iterations=args.block_iterations, mg_stage_chebyshev=args.chebyshev,
                             mg_fine_chebyshev=args.fine_chebyshev, gmres_delayed=args.delayed,
                             gmres_recycle=args.recycle, mg_stage_fp16=args.stage_fp16)
    system.configure(speed=spec.speed, **spec.case)
    slots = system.inflow_layout()
    faces = len(slots) * spec.brick_size ** 2
    centres = inflow_face_centres(built.topology, slots)
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
    roofline = None
    region_ms = round(float(np.mean(per_launch)), 4) if len(per_launch) else None
    if len(per_launch) and args.profile_region == 0:
        avg_ms = float(np.mean(per_launch))
        algorithmic = A_P_BYTES_PER_DOF * bricks * spec.brick_size ** 3
        achieved = algorithmic / (avg_ms * 1e-3) / 1e9
        traffic = ncu_traffic(args.workload)
        roofline = {"bound": "hbm", "kernel": region_names[0], "achieved": round(achieved, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                    "traffic": traffic, "algorithmic_bytes_per_launch": algorithmic,
                    "launches_timed": int(len(per_launch)), "avg_launch_us": round(avg_ms * 1e3, 2)}
    line = {
        "metric": "AMR steps/s at 16M cells (projection to 1e-8, loads every step)",
        "value": round(value, 4), "unit": "steps/s", "n_gpus": n, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(elapsed_ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 state / f64 pressure", "data": "synthetic analytic geometry",
        "config": dict(spec.describe(), leaf_cells=built.leaf_cells, storage=built.storage_size,
                       mg=args.mg, mg_cycle=args.mg_cycle, gcro_restart=args.restart or 24,
                       stage_sweeps=args.stage_sweeps or 6, block_iterations=args.block_iterations,
                       stage_smoother="jacobi" if args.chebyshev == 1 else f"chebyshev 2/{args.chebyshev or 30}",
                       fine_smoother="jacobi" if args.fine_chebyshev == 1 else f"chebyshev-richardson 2/{args.fine_chebyshev or 10}",
                       orthogonalisation="delayed CGS2" if args.delayed else "CGS2",
                       recycled_pairs=3 if args.recycle == 0 else max(args.recycle, 0),
                       stage_coefficients="fp16" if args.stage_fp16 else args.mg,
                       parallelism=f"replicas{n}",
                       l2="inputs larger than L2"),
        "projection_ms": round(statistics.mean(s["projection_ms"] for s in stats), 3),
        "iterations_per_step": round(statistics.mean(s["pressure"]["iterations"] for s in stats), 2),
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
        "profiled_region": {"region": region_names.get(args.profile_region), "launches": int(len(per_launch)),
                            "avg_ms": region_ms},
        "cpu_baseline": None,
    }
    if ranks.rank == 0 and n == 1 and not args.no_cpu_baseline:
        try:
            cpu = CpuReference(built.topology, spec)
            stages = {name: cpu.stage(name) for name in CpuReference.STAGES}
            cpu.time_solver(2)
            iters = max(1, int(round(line["iterations_per_step"])))
            stages["projection_solve"] = cpu.per_iteration_s * iters
            cpu.close()
            step_s = sum(stages.values())
            line["cpu_baseline"] = {
                "value": round(1.0 / step_s, 6), "unit": "steps/s", "cores": cpu.threads, "kind": "reference",
                "sample": (f"one full-size step: each operator once through the reference CPU twins (1 thread); "
                           f"solve = FP64 OpenMP restated solver ({cpu.threads} threads), time of its first 2 "
                           f"Krylov iterations per iteration x {iters} (this run's GPU count; early iterations are "
                           f"the cheapest, so the CPU figure is optimistic)"),
                "stages_s": {k: round(t, 4) for k, t in stages.items()}}
        except Exception as exc:   # the CPU sample must not hide the GPU result
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    system.close()
    built.close()
    if ranks.rank == 0 and n == 1 and not args.no_learned:
        # the learned-preconditioner comparison (a short --learned run) beside the headline
        try:
            short = argparse.Namespace(**{**vars(args), "harvest_runs": 2, "train_steps": 1500, "steps": 2, "warmup": 2})
            line["learned"] = run_learned(short, ranks)
        except Exception as exc:
            line["learned"] = {"error": str(exc)[:200]}
    return line


def run_kernel_only(args):
    from paracfd_b200 import MG_FP32, MG_FP64, CompositeSystem
    from paracfd_b200.workloads import WORKLOADS
    spec = WORKLOADS[args.workload]
    built = spec.build()
    system = CompositeSystem(built.topology, MG_FP32 if args.mg == "fp32" else MG_FP64,
                             mg_cycle={"reference": 0, "corrected": 1, "composite": 2}[args.mg_cycle],
                             gmres_restart=args.restart, mg_stage_sweeps=args.stage_sweeps,
                             mg_block_iterations=args.block_iterations, mg_stage_chebyshev=args.chebyshev,
                             mg_fine_chebyshev=args.fine_chebyshev, gmres_delayed=args.delayed,
                             gmres_recycle=args.recycle, mg_stage_fp16=args.stage_fp16)
    ms = system.time_kernel(args.kernel_only, args.kernel_iterations)
    line = {"kernel_only": args.kernel_only, "workload": args.workload, "ms_per_launch": ms,
            "iterations": args.kernel_iterations, "launches": system.launch_count()}
    system.close()
    built.close()
    return line


def run_reference(args, ranks: Ranks):
    """The reference's CPU implementation of the step on this machine's cores.

    Setup (untimed): the reference imports the topology; its solver restatement solves the first
    step's RHS to 1e-8 once, which gives the per-iteration cost and, without a GPU, the iteration
    count.  With a GPU, the reference's own sm_100a device classes run the same workload
    (ExternalAeroCore's step sequence) and their mean iterations per step are used, and reported
    beside.  Each timed step then times one stage of the step in rotation (all stages are covered
    after len(STAGES) steps; any left over are timed after the loop), so a run stays within a few
    minutes; value = 1 / (sum of the mean stage times + per-iteration time x iterations).
    """
    from paracfd_b200.workloads import WORKLOADS
    spec = WORKLOADS[args.workload]
    if ranks.rank != 0:
        return None
    built = spec.build()
    case = spec.case
    gpu = None
    iterations = None
    if not args.no_reference_gpu:
        try:
            from oracle import ref
            rc = ref.import_topology(built.topology)
            core = ref.RefDeviceCore(rc, spec.speed, case["rho"], case["nu"], case["cfl"], case["smagorinsky_cs"],
                                     case["projection_tolerance"], case["projection_max_iterations"], 0.0)
            core.initialize()
            for _ in range(args.warmup):
                core.step()
            st = [core.step() for _ in range(args.steps)]
            core.close()
            rc.close()
            step_ms = statistics.mean(s["gpu_step_ms"] for s in st)
            iterations = max(1, int(round(statistics.mean(s["iterations"] for s in st))))
            gpu = {"steps_per_s": round(1000.0 / step_ms, 4), "step_ms": round(step_ms, 3),
                   "projection_ms": round(statistics.mean(s["projection_ms"] for s in st), 3),
                   "iterations_per_step": iterations, "converged_steps": sum(bool(s["converged"]) for s in st),
                   "timing": "reference ExternalAeroStepStats host clock around its synchronous stages",
                   "build": "reference sources compiled for sm_100a (oracle/_ref)"}
        except Exception as exc:
            gpu = {"unavailable": str(exc)[:200]}
    cpu = CpuReference(built.topology, spec)
    solve = cpu.time_solver(case["projection_max_iterations"])
    if iterations is None:
        iterations = max(1, solve["iterations"])
    names = CpuReference.STAGES
    for q in range(args.warmup):
        cpu.stage(names[q % len(names)])
    times = {name: [] for name in names}
    for q in range(args.steps):
        name = names[q % len(names)]
        times[name].append(cpu.stage(name))
    for name in names:
        if not times[name]:
            times[name].append(cpu.stage(name))
    cpu.close()
    stages = {name: statistics.mean(t) for name, t in times.items()}
    stages["projection_solve"] = cpu.per_iteration_s * iterations
    step_s = sum(stages.values())
    value = 1.0 / step_s
    sample = (f"per step one stage of the reference CPU twins (1 thread) at full size, in rotation; solve = FP64 "
              f"OpenMP restated solver ({cpu.threads} threads): {solve['iterations']} iterations to "
              f"{solve['relative_residual']:.2e} in {solve['seconds']:.1f} s, per-iteration time x {iterations} iterations")
    line = {
        "metric": "AMR steps/s at 16M cells (projection to 1e-8, loads every step)", "impl": "reference",
        "value": round(value, 6), "unit": "steps/s", "n_gpus": ranks.world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(step_s * 1e3, 1), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 state / f64 pressure", "data": "synthetic analytic geometry",
        "config": dict(spec.describe(), leaf_cells=built.leaf_cells, storage=built.storage_size),
        "cpu_baseline": {"value": round(value, 6), "unit": "steps/s", "cores": cpu.threads, "kind": "reference",
                         "sample": sample, "stages_s": {k: round(t, 4) for k, t in stages.items()}},
        "e2e": {"value": round(value, 6), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_sm100a": gpu,
    }
    built.close()
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
        built = spec.build()
        with CompositeSystem(built.topology, device=ranks.local, mg_cycle=MG_CYCLE_COMPOSITE) as system:
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
    built = spec.build()
    system = CompositeSystem(built.topology, device=ranks.local, mg_cycle=MG_CYCLE_COMPOSITE)
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
        "config": dict(spec.describe(), leaf_cells=built.leaf_cells, bricks=bricks, mg_cycle="composite",
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


def run_sweep(args, ranks: Ranks):
    """BASELINE config 5 on one GPU: the angle-of-attack sweep as batches of concurrent instances."""
    from concurrent.futures import ThreadPoolExecutor

    from paracfd_b200 import MG_CYCLE_COMPOSITE, MG_FP32, CompositeSystem
    from paracfd_b200.workloads import sweep_instances

    specs = sweep_instances()
    batches = []
    for first in range(0, len(specs), 4):
        batch = specs[first:first + 4]
        builts = [sp.build() for sp in batch]
        systems = [CompositeSystem(b.topology, MG_FP32, device=ranks.local, mg_cycle=MG_CYCLE_COMPOSITE,
                                   mg_stage_sweeps=args.stage_sweeps, mg_stage_chebyshev=args.chebyshev,
                                   mg_fine_chebyshev=args.fine_chebyshev, gmres_delayed=args.delayed,
                             gmres_recycle=args.recycle, mg_stage_fp16=args.stage_fp16) for b in builts]
        for sp, sy in zip(batch, systems):
            sy.configure(speed=sp.speed, **sp.case)
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
                        "iterations_per_step": [round(i / args.steps, 2) for i in iterations]})
        for sy in systems:
            sy.close()
        for b in builts:
            b.close()
    instance_steps = len(specs) * args.steps
    seq = sum(b["sequential_s"] for b in batches)
    conc = sum(b["concurrent_s"] for b in batches)
    return {
        "metric": "batched angle sweep: instance-steps/s over 16 naca4412_wing instances (4 batches of 4)",
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
