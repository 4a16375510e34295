#!/usr/bin/env python
"""Benchmark of the 3D IISPH timestep (neighborhood search + IISPH step) on
one or more B200s; prints one JSON line.

Workload (default): the 1M-fluid breaking dam -- a 100 x 100 x 100 block with
+-1 % seeded jitter in a single-layer tank (256,624 boundary particles), cubic
spline kernel with support 2 x spacing, relaxed Jacobi omega 0.5, gamma 0.7,
<= 0.1 % average density error, 2..100 iterations, viscosity 0.01, single-layer
gamma_1 1.1. The scene is in the reference's own units (particle size 1, rest
density 1, dt 0.005; see fluidsolver_b200/scenes.py). A "step" is one
Simulator step: search + IISPH step over the whole scene. The metric counts
fluid particles: fluid particle-steps per second.

  python bench.py [--gpus N --steps K --warmup W]     # this implementation
  python bench.py --impl reference ...                # the reference's CPU code

Under torchrun with N ranks every rank advances its own replica of the scene
on its own GPU (independent scenes, no exchange): weak scaling.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D IISPH fluid particle-steps/s (1M breaking dam), <= 0.1% avg density error"
UNIT = "fluid particle-steps/s"

# algorithmic bytes (compulsory SoA traffic per phase; neighbor gathers are
# on-chip reuse and neighbor lists are not counted)
BYTES_SEARCH = 144   # per active particle: keys, 2 radix passes, permute pos/vel/rho/tag, cell ranges
BYTES_L1 = 76        # per fluid particle: read pos4 vel4 rho, write rho v*4 a_np4 p
BYTES_L2 = 44        # per fluid particle: read pos4 v*4 rho, write s a_ii
BYTES_ITER = 84      # per fluid particle and iteration: pressure acceleration 36 + update 48
BYTES_INTEGRATE = 96  # per active particle: read pos4 v*4 a_np4 a4, write pos4 vel4
PHASES = ["search", "iisph_l1", "iisph_l2", "pressure_iterations", "integration"]
PHASE_KERNELS = ["neighborhood search (sort, reorder, cell table, k_build_tiles)", "k_tile_iisph3d_l1",
                 "k_tile_iisph3d_l2 (with the first pressure iteration)",
                 "pressure iteration 2..I: k_tile_iisph3d_pressure_acc + k_tile_iisph3d_pressure_update",
                 "k_cfl + k_iisph3d_integrate"]
PHASE_UNITS = ["step", "launch", "launch", "iteration (two launches)", "step"]
# The timed window starts PREROLL_STEPS steps into the dam's run, inside its
# collapse, so that it needs as many pressure iterations per step as the
# configuration's whole run of FULL_RUN_STEPS steps does on average (its
# first steps, from rest, need the minimum of 2).
PREROLL_STEPS = 1000
FULL_RUN_STEPS = 2000


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML every
    few milliseconds while the timed region runs (read-only queries)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device: int, period_s: float = 0.004):
        self.device, self.period = device, period_s
        self.samples, self.max_mhz, self.handle = [], None, None
        self.nvml = None
        self.stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            self.handle = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.handle, pynvml.NVML_CLOCK_SM)
            self.nvml = pynvml
        except Exception:
            self.nvml = None
            return self
        self.sample()
        self.thread = threading.Thread(target=self.loop, daemon=True)
        self.thread.start()
        return self

    def sample(self):
        N = self.nvml
        try:
            mhz = N.nvmlDeviceGetClockInfo(self.handle, N.NVML_CLOCK_SM)
            bits = N.nvmlDeviceGetCurrentClocksEventReasons(self.handle)
        except Exception:
            return
        self.samples.append((mhz, bits))

    def loop(self):
        while not self.stop.wait(self.period):
            self.sample()

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
            self.sample()

    def summary(self):
        if self.nvml is None or not self.samples:
            return None
        N = self.nvml
        reasons = sorted({name for _, bits in self.samples for name, attr in self.REASONS
                          if hasattr(N, attr) and bits & getattr(N, attr)})
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, 4 ms period"}


def configure_iisph(s, rest_density=1.0, particle_size=1.0):
    """The benchmark's IISPH parameters (reference units, see scenes.py)."""
    from fluidsolver_b200.scenes import REFERENCE_UNITS_DT
    s.parameters.rest_density = rest_density
    s.parameters.gravity = 9.81
    s.parameters.particle_size = particle_size
    s.settings.viscosity = 0.01
    s.settings.single_layer_boundary = True
    s.settings.single_layer_boundary_gamma_1 = 1.1
    s.settings.max_density_error_allowed = 0.001
    s.settings.min_number_of_iterations = 2
    s.settings.max_number_of_iterations = 100
    s.settings.omega = 0.5
    s.settings.gamma = 0.7
    s.timestep_generator.settings.timestep = REFERENCE_UNITS_DT


def make_solver(scene, device, precision="fp32-kahan", eager=False):
    from fluidsolver_b200 import IISPHFluidSolver3D
    s = IISPHFluidSolver3D(search="hashed-3d", precision=precision, device=device, sync_each_iteration=eager)
    configure_iisph(s, scene.rest_density, scene.particle_size)
    s.data.collection = scene.collection
    return s


def reference_settings():
    from oracle import ref_oracle as R
    from fluidsolver_b200.scenes import REFERENCE_UNITS_DT
    return ((1.0, 9.81, 1.0), R.iisph3d_settings(max_err=0.001, min_it=2, max_it=100, omega=0.5, gamma=0.7,
                                                   viscosity=0.01, single_layer=True, gamma1=1.1),
            (REFERENCE_UNITS_DT, 0.4, 0.25))


def ref_variant():
    from oracle import ref_oracle as R
    return "omp" if R.available("omp") else ("serial" if R.available("serial") else None)


def variant_text(variant):
    return "OpenMP over its 16-particle chunks" if variant == "omp" else "as built, serial"


def cpu_baseline_from_state(state, n_fluid, seconds_budget=20.0):
    """The reference's own CPU code (oracle/_ref, all host cores) continuing
    from the GPU's state at the end of the timed window: one untimed step
    first (the reference's first search sorts the whole collection and builds
    its grid, HashedNeighborhoodSearch3D.cpp:82-131, 187-217), then timed
    steps until the budget is spent (at least one, at most three)."""
    from oracle import ref_oracle as R
    variant = ref_variant()
    if variant is None:
        return None
    params, settings, gen = reference_settings()
    ref = R.RefSolver("iisph-3d", "hashed-3d", state, params, settings, gen, variant=variant)
    t_cold = time.perf_counter()
    ref.step()
    t_cold = time.perf_counter() - t_cold
    steps, t0 = 0, time.perf_counter()
    iters = []
    while True:
        iters.append(ref.step()["iterations"])
        steps += 1
        el = time.perf_counter() - t0
        if el > seconds_budget / 2 or steps >= 3:
            break
    ref.close()
    cores = os.cpu_count() if variant == "omp" else 1
    return {"value": n_fluid * steps / el, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{steps} timed step(s) of the same 1M-fluid scene continuing from the GPU state at the end of "
                      f"the timed window, after 1 untimed step ({t_cold:.1f} s: the first search's sort and grid "
                      f"build); reference libFluid IISPHFluidSolver3D<CubicSplineKernel3D, HashedNeighborhoodSearch3D> "
                      f"({variant_text(variant)}), iterations {iters}, {el:.1f} s timed"}


# iterations per step assumed for every scene when the batched scenes are
# dealt out (the cost estimate of scene_cost; the measured means lie near 2-4)
COST_ITERATIONS = 3.0


def scene_cost(n_fluid: int, n_boundary: int, iterations: float = COST_ITERATIONS) -> float:
    """Estimated cost of one step of a scene: its algorithmic bytes
    (144 per active particle for the search, 216 + 84 I per fluid particle
    for the IISPH phases), i.e. F * I plus the terms that do not iterate."""
    return BYTES_SEARCH * (n_fluid + n_boundary) + n_fluid * (BYTES_L1 + BYTES_L2 + BYTES_INTEGRATE + BYTES_ITER * iterations)


def shard(items, rank: int, world: int, cost=None) -> list:
    """The items that rank `rank` of `world` takes: longest processing time
    first. Items go in order of decreasing cost (ties by index) to the rank
    with the least cost so far (ties by rank), so every rank's total is at
    most the mean plus the largest item's cost. Without costs every item
    costs 1. The assignment depends on the items only, so every rank computes
    the same split without exchanging anything."""
    costs = [1.0] * len(items) if cost is None else [float(cost(x)) for x in items]
    order = sorted(range(len(items)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        load[r] += costs[i]
        if r == rank:
            mine.append(i)
    return [items[i] for i in sorted(mine)]


def max_reducer(world: int, device):
    """max over ranks of a float (torch.distributed, tensors on `device`)."""
    def reduce(x: float) -> float:
        if world == 1:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return reduce


def run_ours(args):
    import torch
    import torch.distributed as dist
    from fluidsolver_b200 import _lib as F
    from fluidsolver_b200 import scenes

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    max_over_ranks = max_reducer(world, "cuda")

    scene = scenes.dam_1m(seed=5 + rank)
    n_active = scene.n_fluid + scene.n_boundary
    solver = make_solver(scene, local, args.precision, args.eager)
    L = F.lib()
    # the fast mode's launch shapes, chosen on a copy of this scene (fs_autotune)
    tuning = None if args.no_autotune else solver.autotune()
    # advance the dam into its collapse, where a run of the configuration's
    # length spends its steps, before warming up and timing
    run_its = []
    for _ in range(args.preroll):
        run_its.append(int(solver.step().iterations))
    for _ in range(args.warmup):
        run_its.append(int(solver.step().iterations))
    ctx = solver.ctx
    stream = torch.cuda.ExternalStream(L.fs_stream(ctx), device=torch.device("cuda", local))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = L.fs_launch_count(ctx)
    phase = np.zeros(5)
    iters, errs = [], []
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            st = solver.step()
            phase += np.array(solver.phase_times())
            iters.append(int(st.iterations))
            errs.append(float(st.avg_density_error_fp64))
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    launches = L.fs_launch_count(ctx) - launches0
    value = scene.n_fluid * args.steps * world / (ms / 1e3)

    # roofline of the dominant phase (algorithmic bytes / its event-timed duration)
    F_, N_ = scene.n_fluid, n_active
    it_total = float(sum(iters))
    # the second loop runs the first pressure iteration too (it needs no
    # neighbor sums: every pressure is 0 when the loop starts), so that phase
    # carries one iteration's bytes and the loop phase the others
    phase_bytes = [BYTES_SEARCH * N_ * args.steps, BYTES_L1 * F_ * args.steps,
                   (BYTES_L2 + BYTES_ITER) * F_ * args.steps, BYTES_ITER * F_ * (it_total - args.steps),
                   BYTES_INTEGRATE * N_ * args.steps]
    dom = int(np.argmax(phase))
    peak, peak_kind = measured_peak()
    achieved = phase_bytes[dom] / (phase[dom] / 1e3) / 1e9
    step_bytes = sum(phase_bytes) / args.steps
    # the unit the roofline kernel's bytes and traffic are quoted per
    units = [args.steps, args.steps, args.steps, max(it_total - args.steps, 1.0), args.steps]
    per_launch = phase_bytes[dom] / units[dom]
    traffic, winst = None, None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        traffic = tj.get(PHASES[dom])
        winst = tj.get("warp_instructions", {}).get(PHASES[dom])

    run_its += iters
    # the state at the end of the window: where the end-to-end run and the
    # CPU baseline continue from
    window_state = solver.collection()
    # the rest of a run of the configuration's length, for its mean iteration count
    while len(run_its) < args.full_run:
        run_its.append(int(solver.step().iterations))
    # end to end through the public API: pinned host state in, step, state out
    e2e = run_e2e(solver, window_state, scene.n_fluid, min(args.steps, 10), local, max_over_ranks)
    solver_state = window_state if (rank == 0 and world == 1 and not args.no_cpu_baseline) else None
    solver.close()
    batched = None if args.no_batched else run_batched(args, local, rank, world, max_over_ranks, barrier, tuning)
    ns_micro = run_ns_microbench(args, local) if (rank == 0 and world == 1 and not args.no_batched) else None
    configs = run_configs(args, local) if (rank == 0 and world == 1 and not args.no_batched) else None

    cpu = None
    if solver_state is not None:
        cpu = cpu_baseline_from_state(solver_state, scene.n_fluid)

    clocks = clk.summary()
    # the same kernel against the SMs' instruction issue rate (one warp
    # instruction per scheduler and cycle, 4 schedulers per SM, at the SM clock
    # sampled in the timed region), which is what bounds it
    issue = None
    if winst and clocks and clocks.get("sm_mhz"):
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        unit_s = phase[dom] / 1e3 / units[dom]
        peak_issue = sms * 4 * clocks["sm_mhz"] * 1e6
        issue = {"issue_achieved": winst / unit_s / 1e9, "issue_peak": peak_issue / 1e9,
                 "issue_unit": "G warp instructions/s", "issue_frac": winst / unit_s / peak_issue,
                 "warp_instructions_per_unit": winst, "sms": sms, "sm_mhz": clocks["sm_mhz"],
                 "issue_source": "warp instructions per unit from profiles/traffic.json (ncu "
                                 "smsp__inst_executed.sum); the duration event-timed here"}
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (Kahan-compensated sums, FP64 residual)" if args.precision ==
            "fp32-kahan" else args.precision, "data": "synthetic (seeded breaking-dam scenes)",
            "config": {"workload": "3D IISPH breaking dam, 1,000,000 fluid + 256,624 boundary particles, "
                       "hashed-3d neighbor contract, dt 0.005 (reference units), single-layer boundary",
                       "fluid_particles_per_gpu": scene.n_fluid, "boundary_particles_per_gpu": scene.n_boundary,
                       "parallelism": f"replicas x{world} (independent scenes)",
                       "mode": "eager (host-driven pressure loop, profiling only)" if args.eager else
                       "whole step as one CUDA graph (pressure loop: conditional WHILE node)",
                       "l2": "inputs larger than L2 (~0.5 GB of particle state and lists per step)",
                       "tuning": tuning,
                       "preroll_steps": args.preroll,
                       "window": f"steps {args.preroll + args.warmup + 1}-{args.preroll + args.warmup + args.steps} "
                                 f"of the dam (after {args.preroll} pre-roll and {args.warmup} warm-up steps)",
                       "iterations_mean": it_total / args.steps,
                       "iterations_mean_full_run": float(np.mean(run_its)), "full_run_steps": len(run_its),
                       "avg_density_error_max": max(errs),
                       "phase_ms_per_step": dict(zip(PHASES, (phase / args.steps).round(4).tolist())),
                       "algorithmic_bytes_per_step": step_bytes,
                       "step_fraction_of_hbm_roofline": step_bytes / (ms / args.steps / 1e3) / 1e9 / peak},
            "roofline": dict({"bound": "hbm", "kernel": PHASE_KERNELS[dom], "achieved": achieved, "peak": peak,
                              "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                              "algorithmic_bytes_per_launch": per_launch, "per": PHASE_UNITS[dom],
                              "traffic_source": "profiles/traffic.json (ncu dram__bytes_read.sum + "
                                                "dram__bytes_write.sum)"}, **(issue or {})),
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
            "batched": batched, "ns_microbench": ns_micro, "other_configs": configs,
        }
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()


def run_batched(args, device, rank, world, max_over_ranks, barrier, tuning=None):
    """The batched breaking dams (256 scenes, seed 6, dealt out over the ranks
    by estimated cost, see shard): all of a rank's scenes in one batched context, timed with CUDA
    events on the context's stream around fs_batch_run; at N = 1 the same
    scenes also run one at a time through the single-scene path (fs_run of
    the same steps per scene, events around each), the plain per-scene form."""
    import torch
    from fluidsolver_b200 import BatchedIISPHFluidSolver3D
    from fluidsolver_b200 import _lib as F
    from fluidsolver_b200 import scenes
    L = F.lib()
    allsc = scenes.batched_dams(256, seed=6)
    mine = shard(allsc, rank, world, cost=lambda sc: scene_cost(sc.n_fluid, sc.n_boundary))
    batch = BatchedIISPHFluidSolver3D([s.collection for s in mine], device=device)
    configure_iisph(batch)
    if tuning and tuning["tuned"]:   # the shapes the 1M dam chose
        batch.set_tuning(tuning["first_loop_prefetch"], tuning["pressure_prefetch"], tuning["tile_cap"],
                         tuning["block_size"], tuning["pressure_threads_per_owner"])
    batch.run(args.warmup)
    stream = torch.cuda.ExternalStream(L.fs_stream(batch.ctx), device=torch.device("cuda", device))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    ev0.record(stream)
    st = batch.run(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    fluid_all = sum(s.n_fluid for s in allsc)
    out = {"workload": f"{len(allsc)} breaking dams (seed 6): fluid {min(s.n_fluid for s in allsc):,}-"
                       f"{max(s.n_fluid for s in allsc):,} per scene, {fluid_all:,} fluid + "
                       f"{sum(s.n_boundary for s in allsc):,} boundary in total, one batched context per GPU",
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
           "value": fluid_all * args.steps / (ms / 1e3), "unit": UNIT,
           "iterations_last_step": {"min": int(min(x.iterations for x in st)), "max": int(max(x.iterations for x in st))},
           "avg_density_error_max": float(max(x.avg_density_error_fp64 for x in st))}
    batch.close()
    if world == 1:
        total_ms = 0.0
        for sc in allsc:
            solver = make_solver(sc, device)
            if tuning and tuning["tuned"]:
                solver.set_tuning(tuning["first_loop_prefetch"], tuning["pressure_prefetch"], tuning["tile_cap"],
                                  tuning["block_size"], tuning["pressure_threads_per_owner"])
            solver.run(args.warmup)
            s2 = torch.cuda.ExternalStream(L.fs_stream(solver.ctx), device=torch.device("cuda", device))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(s2)
            solver.run(args.steps)
            b.record(s2)
            torch.cuda.synchronize()
            total_ms += a.elapsed_time(b)
            solver.close()
        out["plain_per_scene_value"] = fluid_all * args.steps / (total_ms / 1e3)
        out["plain_per_scene_ms_per_step"] = total_ms / args.steps
        out["speedup_vs_plain_per_scene"] = out["value"] / out["plain_per_scene_value"]
        if not args.no_cpu_baseline:
            out["cpu"] = batched_cpu_baseline(allsc)
    return out


def batched_cpu_baseline(allsc, sample=16, steps=2):
    """The reference scene by scene (it has no batching; one
    IISPHFluidSolver3D per scene, oracle/_ref on all host cores) on a
    sample of the batched dams: `sample` scenes evenly spaced in fluid count,
    each 1 untimed + `steps` timed steps. The value is the sample's fluid
    particle-steps over its total time; the 256 scenes' time follows from it
    (their fluid total over that rate)."""
    from oracle import ref_oracle as R
    variant = ref_variant()
    if variant is None:
        return None
    params, settings, gen = reference_settings()
    order = sorted(range(len(allsc)), key=lambda i: allsc[i].n_fluid)
    pick = [order[int(round(q * (len(order) - 1) / (sample - 1)))] for q in range(sample)]
    fluid_steps, el = 0, 0.0
    for i in pick:
        sc = allsc[i]
        ref = R.RefSolver("iisph-3d", "hashed-3d", sc.collection, params, settings, gen, variant=variant)
        ref.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            ref.step()
        el += time.perf_counter() - t0
        fluid_steps += sc.n_fluid * steps
        ref.close()
    rate = fluid_steps / el
    fluid_all = sum(x.n_fluid for x in allsc)
    return {"value": rate, "unit": UNIT, "ms_per_step_all_scenes": fluid_all / rate * 1e3,
            "cores": os.cpu_count() if variant == "omp" else 1, "kind": "reference",
            "sample": f"{sample} of the {len(allsc)} scenes, evenly spaced in fluid count "
                      f"({min(allsc[i].n_fluid for i in pick):,}-{max(allsc[i].n_fluid for i in pick):,}), "
                      f"scene by scene, 1 untimed + {steps} timed steps each, {el:.1f} s timed",
            "variant": variant_text(variant)}


def ref_search_time(kind, pts, radius, calls=10, budget_s=15.0):
    """The reference's own search (oracle/_ref) on the same points: one
    untimed call (the first builds the grid and, for hashed-3d, sorts the
    collection), then up to `calls` timed find_neighbors calls within the
    budget; ms per call (wall clock) and the calls made."""
    from oracle import ref_oracle as R
    variant = ref_variant()
    if variant is None:
        return None
    rs = R.RefSearch(kind, pts, radius, variant=variant)
    t_cold = time.perf_counter()
    ok = rs.find()
    t_cold = time.perf_counter() - t_cold
    if not ok:
        rs.close()
        return {"error": "the reference's search threw (a list above its capacity)"}
    k, t0 = 0, time.perf_counter()
    while k < calls and (k == 0 or time.perf_counter() - t0 < budget_s):
        rs.find()
        k += 1
    el = time.perf_counter() - t0
    rs.close()
    return {"ms_per_search": el / k * 1e3, "calls": k, "first_call_s": t_cold,
            "points_per_s": len(pts) / (el / k), "cores": os.cpu_count() if variant == "omp" else 1,
            "kind": "reference", "variant": variant_text(variant)}


def run_ns_microbench(args, device):
    """The 3D search microbenchmark: 10^6 points in the unit cube, r = 0.02,
    uniform (seed 2) and 64 Gaussian blobs (sigma 0.03, seed 3). (1) The
    device search as a solver step runs it (sort, reorder, cell table and the
    neighbor lists of every point), timed with the library's own events over
    --steps searches: the fast mode's tile lists on the uniform points; on
    the blobs, whose cores hold over a thousand neighbors per point, the
    32-bit lists of the FP32 mode. (2) The contract's neighbor sets exported
    in host index space (fs_get_neighbors_csr, both calls, wall clock).
    (3) The reference's own searches on the same points (oracle/_ref):
    HashedNeighborhoodSearch3D on both sets, CompressedNeighborhoodSearch on
    the uniform points (it throws above 97 neighbors, which the blobs' cores
    exceed). Byte model: 96 B per point (keys, sort, permute of the
    positions) + (4 n + 8) B of lists per point."""
    from fluidsolver_b200 import IISPHFluidSolver3D, NeighborhoodSearch, ParticleCollection
    sc = scenes_mod()
    peak, kind = measured_peak()
    out = {}
    for case, pts in (("uniform", sc.ns_points_uniform()), ("blobs", sc.ns_points_blobs())):
        col = ParticleCollection(position=pts)
        s = IISPHFluidSolver3D(search="hashed-3d", precision="fp32-kahan" if case == "uniform" else "fp32",
                               device=device)
        s.parameters.particle_size = 0.01
        s.data.collection = col
        for _ in range(args.warmup):
            s.execute_neighborhood_search()
        ms = []
        for _ in range(args.steps):
            s.execute_neighborhood_search()
            ms.append(s.phase_times()[0])
        s.close()
        ns = NeighborhoodSearch("hashed-3d", 0.02, device=device)
        ns.data.collection = col
        ns.find_neighbors()
        t0 = time.perf_counter()
        off, idx = ns.neighbor_lists()
        export_s = time.perf_counter() - t0
        ns.close()
        nbar = len(idx) / len(pts)
        nmax = int(np.max(np.diff(off)))
        del off, idx
        per = statistics.median(ms)
        bytes_ = (96 + 4 * nbar + 8) * len(pts)
        r = {"workload": f"10^6 {'uniform points' if case == 'uniform' else 'points in 64 Gaussian blobs (sigma 0.03)'}"
                         f" in [0,1)^3 (seed {2 if case == 'uniform' else 3}), r = 0.02, hashed-3d contract",
             "neighbors_mean": nbar, "neighbors_max": nmax, "search_with_lists_ms": per,
             "lists": "tile lists (fast mode)" if case == "uniform" else "32-bit lists (FP32 mode)",
             "points_per_s": len(pts) / (per / 1e3), "algorithmic_bytes": bytes_,
             "achieved_gbs": bytes_ / (per / 1e3) / 1e9, "frac_of_hbm_peak": bytes_ / (per / 1e3) / 1e9 / peak,
             "csr_export_s": export_s, "csr_export_path": "fs_get_neighbors_csr, sets in host index space, wall clock"}
        if not args.no_cpu_baseline:
            r["cpu_hashed_3d"] = ref_search_time("hashed-3d", pts, 0.02)
            if case == "uniform":
                r["cpu_compressed_3d"] = ref_search_time("compressed-3d", pts, 0.02)
        out[case] = r
    return out


def run_configs(args, device):
    """The other configurations, each next to the reference's own CPU code
    (oracle/_ref, bounded samples): the 2D SESPH dam (hashed-2d), the 100k 3D
    IISPH dam, and the 1M dam in the two other precisions (plain FP32 in the
    reference's operation order, FP64). GPU times are CUDA events around
    fs_run on the library's stream."""
    import torch
    from fluidsolver_b200 import SESPHFluidSolver
    from fluidsolver_b200 import _lib as F
    from fluidsolver_b200.scenes import REFERENCE_UNITS_DT
    sc = scenes_mod()
    L = F.lib()

    def gpu_time(solver, steps):
        solver.run(args.warmup)
        st = torch.cuda.ExternalStream(L.fs_stream(solver.ctx), device=torch.device("cuda", device))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        stats = solver.run(steps)
        b.record(st)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps, stats

    def ref_time(solver_kind, search, scene, params, settings, gen, steps, budget_s):
        from oracle import ref_oracle as R
        variant = "omp" if R.available("omp") else ("serial" if R.available("serial") else None)
        if variant is None:
            return None
        ref = R.RefSolver(solver_kind, search, scene.collection, params, settings, gen, variant=variant)
        ref.step()
        t0, k = time.perf_counter(), 0
        while k < steps and time.perf_counter() - t0 < budget_s:
            ref.step()
            k += 1
        el = time.perf_counter() - t0
        ref.close()
        return {"ms_per_step": el / k * 1e3, "steps": k, "cores": os.cpu_count() if variant == "omp" else 1,
                "kind": "reference", "variant": "OpenMP over its 16-particle chunks" if variant == "omp" else "as built"}

    out = {}
    # 2D SESPH dam: 50 x 50 fluid, 3 boundary layers, k 1000, nu 0.01, dt 0.001 (no CFL clamp in 2D SESPH)
    d2 = sc.breaking_dam_2d()
    s2 = SESPHFluidSolver(search="hashed-2d", device=device)
    s2.parameters.rest_density, s2.parameters.gravity, s2.parameters.particle_size = 1.0, 9.81, 1.0
    s2.settings.StiffnessK, s2.settings.Viscosity = 1000.0, 0.01
    s2.timestep_generator.settings.timestep = 0.001
    s2.data.collection = d2.collection
    ms2, _ = gpu_time(s2, 200)
    s2.close()
    out["sesph2d_dam"] = {"workload": f"2D SESPH dam, {d2.n_fluid} fluid + {d2.n_boundary} boundary, hashed-2d, "
                                      "k 1000, nu 0.01, dt 0.001", "gpu_ms_per_step": ms2,
                          "gpu_particle_steps_per_s": d2.n_fluid / (ms2 / 1e3),
                          "cpu": None}

    def dam2d_ms(precision, reference_order, one_kernel_steps):
        s = SESPHFluidSolver(search="hashed-2d", device=device, precision=precision,
                             reference_order=reference_order, one_kernel_steps=one_kernel_steps)
        s.parameters.rest_density, s.parameters.gravity, s.parameters.particle_size = 1.0, 9.81, 1.0
        s.settings.StiffnessK, s.settings.Viscosity = 1000.0, 0.01
        s.timestep_generator.settings.timestep = 0.001
        s.data.collection = d2.collection
        ms, _ = gpu_time(s, 200)
        blocks = int(L.fs_small_blocks(s.ctx))
        s.close()
        return ms, blocks

    # the same dam in the bit-exact reference-order mode, and both modes in
    # the small-scene cluster kernel (FS_FLAG_ONE_KERNEL_STEPS: whole steps
    # in one launch of one thread-block cluster)
    ms2x, _ = dam2d_ms("fp32", True, False)
    ms2c, blocks = dam2d_ms("fp32-kahan", False, True)
    ms2cx, _ = dam2d_ms("fp32", True, True)
    out["sesph2d_dam"].update({"gpu_ms_per_step_reference_order": ms2x, "cluster_kernel_ms_per_step": ms2c,
                               "cluster_kernel_ms_per_step_reference_order": ms2cx, "cluster_blocks": blocks})
    if not args.no_cpu_baseline:
        from oracle import ref_oracle as R
        cpu = ref_time("sesph-2d", "hashed-2d", d2, (1.0, 9.81, 1.0), R.sesph2d_settings(1000.0, 0.01),
                       (0.001, 0.4, 0.25), 200, 10.0)
        out["sesph2d_dam"]["cpu"] = cpu
    # the same dam on the quadratic-dynamic-allocated contract (every pair tested)
    s2q = SESPHFluidSolver(search="quadratic-2d", device=device)
    s2q.parameters.rest_density, s2q.parameters.gravity, s2q.parameters.particle_size = 1.0, 9.81, 1.0
    s2q.settings.StiffnessK, s2q.settings.Viscosity = 1000.0, 0.01
    s2q.timestep_generator.settings.timestep = 0.001
    s2q.data.collection = d2.collection
    ms2q, _ = gpu_time(s2q, 200)
    s2q.close()
    out["sesph2d_dam_quadratic"] = {"workload": f"2D SESPH dam, {d2.n_fluid} fluid + {d2.n_boundary} boundary, "
                                                "quadratic-2d (QuadraticNeighborhoodSearchDynamicAllocated), k 1000, "
                                                "nu 0.01, dt 0.001", "gpu_ms_per_step": ms2q,
                                    "gpu_particle_steps_per_s": d2.n_fluid / (ms2q / 1e3), "cpu": None}
    if not args.no_cpu_baseline:
        out["sesph2d_dam_quadratic"]["cpu"] = ref_time(
            "sesph-2d", "quadratic-2d", d2, (1.0, 9.81, 1.0), R.sesph2d_settings(1000.0, 0.01),
            (0.001, 0.4, 0.25), 100, 10.0)
    # 3D IISPH 100k dam
    d3 = sc.dam_100k()
    s3 = make_solver(d3, device)
    ms3, st3 = gpu_time(s3, 20)
    s3.close()
    out["iisph3d_dam_100k"] = {"workload": f"3D IISPH dam, {d3.n_fluid} fluid + {d3.n_boundary} boundary, hashed-3d, "
                                           f"dt {REFERENCE_UNITS_DT}", "gpu_ms_per_step": ms3,
                               "gpu_particle_steps_per_s": d3.n_fluid / (ms3 / 1e3),
                               "iterations_last_step": int(st3.iterations), "cpu": None}
    if not args.no_cpu_baseline:
        params, settings, gen = reference_settings()
        out["iisph3d_dam_100k"]["cpu"] = ref_time("iisph-3d", "hashed-3d", d3, params, settings, gen, 5, 15.0)
    # the other solvers at a glance: 3D SESPH on the 100k dam, 2D IISPH on the 2D dam
    from fluidsolver_b200 import IISPHFluidSolver, SESPHFluidSolver3D
    s5 = SESPHFluidSolver3D(search="hashed-3d", device=device)
    s5.parameters.rest_density, s5.parameters.gravity, s5.parameters.particle_size = 1.0, 9.81, 1.0
    s5.settings.StiffnessK, s5.settings.Viscosity = 1000.0, 0.01
    s5.settings.single_layer_boundary = True
    s5.timestep_generator.settings.timestep = 0.001
    s5.data.collection = d3.collection
    ms5, _ = gpu_time(s5, 20)
    s5.close()
    out["sesph3d_dam_100k"] = {"workload": "3D SESPH on the 100k dam, hashed-3d, k 1000, nu 0.01, dt 0.001 (CFL-clamped)",
                               "gpu_ms_per_step": ms5, "gpu_particle_steps_per_s": d3.n_fluid / (ms5 / 1e3)}
    d1m = sc.dam_1m(seed=5)
    s5 = SESPHFluidSolver3D(search="hashed-3d", device=device)
    s5.parameters.rest_density, s5.parameters.gravity, s5.parameters.particle_size = 1.0, 9.81, 1.0
    s5.settings.StiffnessK, s5.settings.Viscosity = 1000.0, 0.01
    s5.settings.single_layer_boundary = True
    s5.timestep_generator.settings.timestep = 0.001
    s5.data.collection = d1m.collection
    ms7, _ = gpu_time(s5, 20)
    s5.close()
    out["sesph3d_dam_1m"] = {"workload": "3D SESPH on the 1M dam, hashed-3d, k 1000, nu 0.01, dt 0.001 (CFL-clamped)",
                             "gpu_ms_per_step": ms7, "gpu_particle_steps_per_s": d1m.n_fluid / (ms7 / 1e3)}
    s6 = IISPHFluidSolver(search="hashed-2d", device=device)
    s6.parameters.rest_density, s6.parameters.gravity, s6.parameters.particle_size = 1.0, 9.81, 1.0
    s6.settings.Viscosity = 0.01
    s6.timestep_generator.settings.timestep = 0.001
    s6.data.collection = d2.collection
    ms6, st6 = gpu_time(s6, 100)
    s6.close()
    out["iisph2d_dam"] = {"workload": f"2D IISPH dam, {d2.n_fluid} fluid + {d2.n_boundary} boundary, hashed-2d, dt 0.001",
                          "gpu_ms_per_step": ms6, "gpu_particle_steps_per_s": d2.n_fluid / (ms6 / 1e3),
                          "iterations_last_step": int(st6.iterations)}
    # 1M dam in the other precisions
    d4 = sc.dam_1m(seed=5)
    for prec in ("fp32", "fp64"):
        s4 = make_solver(d4, device, prec)
        if prec == "fp32":
            s4.reference_order = True
        ms4, st4 = gpu_time(s4, 5)
        s4.close()
        out[f"iisph3d_dam_1m_{prec}"] = {
            "workload": "the 1M dam" + (" in FP32 with the reference's operation order and list order" if prec ==
                                        "fp32" else " in FP64 (the error reference)"),
            "gpu_ms_per_step": ms4, "gpu_particle_steps_per_s": d4.n_fluid / (ms4 / 1e3),
            "iterations_last_step": int(st4.iterations), "avg_density_error_last_step": float(st4.avg_density_error_fp64)}
    out["error_vs_fp64"] = error_vs_fp64(sc.dam_1m(seed=5), device)
    return out


def error_vs_fp64(scene, device, steps=5):
    """The state after `steps` steps of the 1M dam in the fast mode (FP32 + compensated sums) and in
    FP32 with the reference's operation order, each against FP64 from the same start: the largest
    position deviation (in particle sizes) and the largest relative density deviation."""
    def run(prec, reference_order=False):
        s = make_solver(scene, device, prec)
        s.reference_order = reference_order
        for _ in range(steps):
            s.step()
        c = s.collection()
        s.close()
        return c
    ref = run("fp64")
    out = {"steps": steps, "scene": "the 1M dam from its initial state"}
    for name, (prec, order) in {"fast_mode": ("fp32-kahan", False), "reference_arithmetic_fp32": ("fp32", True)}.items():
        c = run(prec, order)
        fluid = ref.type == 0
        out[name] = {
            "position_max_abs": float(np.abs(c.position[fluid] - ref.position[fluid]).max() / scene.particle_size),
            "density_max_rel": float((np.abs(c.density[fluid].astype(np.float64) - ref.density[fluid]) /
                                      np.abs(ref.density[fluid].astype(np.float64))).max())}
    return out


def scenes_mod():
    from fluidsolver_b200 import scenes
    return scenes


def run_e2e(solver, src, n_fluid, steps, device, max_over_ranks):
    """Per step: upload the state from pinned host memory, search + step,
    download the state to pinned host memory (the host collection stays
    authoritative, as when entities or sensors touch it every step). src:
    the collection the run starts from."""
    import torch
    from fluidsolver_b200 import _lib as F
    L = F.lib()
    n = len(src)

    def pinned(shape, dtype):
        return torch.empty(shape, dtype=dtype, pin_memory=True).numpy()

    inp = {"position": pinned((n, 3), torch.float32), "velocity": pinned((n, 3), torch.float32),
           "mass": pinned((n,), torch.float32), "density": pinned((n,), torch.float32),
           "type": pinned((n,), torch.uint8)}
    for k, a in inp.items():
        a[...] = getattr(src, k)
    # the step's results land in the same pinned arrays the next upload reads
    out = {"position": inp["position"], "velocity": inp["velocity"], "density": inp["density"],
           "pressure": pinned((n,), torch.float32)}
    fin = F.FsParticles()
    fin.n = n
    for k, a in inp.items():
        setattr(fin, k, a.ctypes.data)
    fout = F.FsParticles()
    fout.n = n
    for k, a in out.items():
        setattr(fout, k, a.ctypes.data)
    h2d = sum(a.nbytes for a in inp.values())
    d2h = sum(a.nbytes for a in out.values())
    ctx = solver.ctx
    stats = F.FsStepStats()

    def one():
        F.check(L.fs_upload(ctx, ctypes.byref(fin)))
        F.check(L.fs_step(ctx, ctypes.c_float(0.0), ctypes.byref(stats)))
        F.check(L.fs_download(ctx, ctypes.byref(fout)))

    one()   # untimed: one-time costs of the first host round trip after the device-timed run
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        one()
    el = max_over_ranks(time.perf_counter() - t0)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    return {"value": n_fluid * steps * world / el, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": steps,
            "path": "fs_upload (pinned host) -> fs_step -> fs_download (pinned host), wall clock"}


def run_reference(args):
    """The reference's own CPU implementation (libFluid sources compiled
    unmodified in oracle/_ref) on all host cores, on the benchmark's own
    scene: the 1M-fluid breaking dam with the same parameters, through the
    reference's solver interface (RefSolver drives its
    execute_neighborhood_search + execute_simulation_step). Each step is a
    whole reference step; the run is bounded in time: the first warm-up step
    (the first search sorts the whole collection and builds the grid) and at
    most 60 s of further warm-up steps, then timed steps until --steps or
    150 s, whichever comes first. The reference starts from the dam at rest,
    where a step needs the fewest pressure iterations (this arm's window lies
    earlier in the run than the GPU arm's, which favours the reference)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import ref_oracle as R
    from fluidsolver_b200 import scenes
    variant = ref_variant()
    if variant is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (needs the reference "
                          "checkout at build time)"}))
        return
    scene = scenes.dam_1m() if args.scene == "1m" else scenes.dam_100k()
    params, settings, gen = reference_settings()
    ref = R.RefSolver("iisph-3d", "hashed-3d", scene.collection, params, settings, gen, variant=variant)
    t_w = time.perf_counter()
    warm = 0
    for _ in range(args.warmup):
        ref.step()
        warm += 1
        if time.perf_counter() - t_w > 60.0:
            break
    iters = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        iters.append(ref.step()["iterations"])
        if time.perf_counter() - t0 > 150.0:   # keep the run within a few minutes
            break
    el = time.perf_counter() - t0
    ref.close()
    done = len(iters)
    value = scene.n_fluid * done / el
    cores = os.cpu_count() if variant == "omp" else 1
    desc = (f"{scene.n_fluid:,}-fluid breaking dam ({scene.n_boundary:,} boundary), steps {warm + 1}-{warm + done} "
            f"from rest: {done} of {args.steps} timed steps (150 s budget) after {warm} of {args.warmup} warm-up "
            f"steps (60 s budget), mean iterations {np.mean(iters):.2f}")
    print(json.dumps({
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": done, "warmup": warm, "ms_per_step": el / done * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded breaking-dam scenes)",
        "impl": "reference",
        "config": {"workload": "3D IISPH breaking dam, " + (
                       "1,000,000 fluid + 256,624 boundary particles (the benchmark's scene)" if args.scene == "1m"
                       else "100,000 fluid + 59,684 boundary particles") +
                   ", hashed-3d neighbor contract, dt 0.005 (reference units), single-layer boundary",
                   "same_config": args.scene == "1m",
                   "implementation": "libFluid IISPHFluidSolver3D<CubicSplineKernel3D, HashedNeighborhoodSearch3D>, "
                                     + variant_text(variant)},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32-kahan", choices=["fp32", "fp32-kahan", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 256-scene batched measurement")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes of the fast mode")
    ap.add_argument("--preroll", type=int, default=PREROLL_STEPS,
                    help="steps the dam advances before the warm-up (into its collapse)")
    ap.add_argument("--full-run", type=int, default=FULL_RUN_STEPS,
                    help="steps of the whole run whose mean iteration count is reported (untimed)")
    ap.add_argument("--scene", default="1m", choices=["1m", "100k"],
                    help="reference arm only: the dam it times (1m: the benchmark's own scene)")
    ap.add_argument("--eager", action="store_true",
                    help="host-driven pressure loop instead of the whole-step CUDA graph: for kernel-level profiling "
                         "(ncu cannot profile the kernels of a graph with conditional nodes); slower, not a bench value")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
