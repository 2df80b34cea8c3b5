#!/usr/bin/env python
"""Throughput of the B200-native FLIP/APIC substep on the 256^3 sparse dam break + falling sphere.

Workload (default `dam_break_sphere_256`): 256^3 cells (h = 1/256, 8^3 bricks, storage budget 1.0),
liquid block x < 0.3, y < 0.5 plus a liquid sphere of radius 0.12 at (0.7, 0.75, 0.5) falling at
2 m/s, 8 jittered particles per fluid cell (seed 1): 20,583,872 particles, 48-byte records (0.99 GB,
far larger than the 126 MB L2, so no L2 flush is needed between steps). APIC, gravity -9.81 y,
CFL 1, frame dt 1/120 s, pressure by FP32 MGPCG to a relative residual of 1e-6, spatial sort every 4
frames, two-sided density projection on the last substep of each frame (the plugin's defaults).

A step is one frame: the CFL substeps of 1/120 s plus the frame's sort and readback. The metric is
substeps per second (whole job; with --gpus N each rank advances its own replica of the tank, no
data-path collective, "weak" scaling). `value` is timed with CUDA events on the simulation stream;
`e2e` is the same loop timed on the host through the C ABI (slosh_step_frame with host frame input,
host results readback), with the bytes the library copied each way.

`--impl reference` times the reference path's CPU restatement (the C++ oracle, OpenMP over all host
cores) on the same workload, one substep per step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FLIP substeps/s at 256^3 ~16M particles; pressure-solve ms to 1e-6 rel residual"
HBM_FALLBACK_GBS = 6650.0
# The preconditioner the GPU arm runs by default: the reference's MGPCG (same V-cycle structure, same stopping
# test) with each coarse-grid correction scaled by 1.9, which makes up for the piecewise-constant prolongation,
# two red-black sweep pairs per smoothing and 4 coarsest-level iterations (the coarsest solve's accuracy does
# not change the iteration count) and the finest level's sweeps over-relaxed by 1.15.
# `--mg-correction 1 --mg-sweeps 1 --mg-coarse-iterations 16 --mg-smoother-weight 1` runs the reference's V-cycle
# exactly; the line's "reference_vcycle" object times it on the same box.
PRECOND = {"mg_correction_scale": 1.9, "mg_smoothing_sweeps": 2, "pcg_flexible": 0, "mg_coarse_iterations": 4,
           "mg_smoother_weight": 1.15}


def apply_precond(settings, args):
    settings.mg_correction_scale = args.mg_correction
    settings.mg_smoothing_sweeps = args.mg_sweeps
    settings.pcg_flexible = args.pcg_flexible
    settings.mg_coarse_iterations = args.mg_coarse_iterations
    settings.mg_smoother_weight = args.mg_smoother_weight
    return {"mg_correction_scale": args.mg_correction, "mg_smoothing_sweeps": args.mg_sweeps,
            "pcg_flexible": bool(args.pcg_flexible), "mg_coarse_iterations": args.mg_coarse_iterations,
            "mg_smoother_weight": args.mg_smoother_weight}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["slosh", "reference"], default="slosh")
    # dam_break_sphere_<n>: the same scene on an n^3 grid (256 is the benchmark; 192 is the small
    # profiling case, 8.7M particles, about 2 GB on the device)
    ap.add_argument("--workload", default="dam_break_sphere_256",
                    help="dam_break_sphere_<n> (n multiple of 8, 32..256), dam_break_64, boxes_512 (512x256x256, 34.5M particles, "
                         "3 static spheres) or tanks_64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # skip the second timed run with the reference's V-cycle (reported as "reference_vcycle")
    ap.add_argument("--no-reference-vcycle", action="store_true")
    # mgpcg: MGPCG to a relative residual of 1e-6 (the benchmark); rbgs: red-black SOR, omega 1.9, 200 iterations
    ap.add_argument("--solver", choices=["mgpcg", "rbgs"], default="mgpcg")
    # storage of the V-cycle's coarse levels (precision_mode); the CG vectors and level 0 stay FP32
    ap.add_argument("--precision", choices=["fp32", "fp16", "bf16"], default="fp32")
    # tanks_64: 64 independent tanks (32^3-128^3), LPT-partitioned over the ranks; each step is one frame of
    # every tank, overlapped on the device by slosh_step_frames, and the same frames are then timed sequentially
    ap.add_argument("--tanks", type=int, default=64)
    # autotune the brick passes' CTAs per SM (slosh_autotune) during warm-up: candidates 2-16, one timed
    # frame each; results do not depend on the choice
    ap.add_argument("--autotune", action="store_true")
    # fixed CTAs per SM of the brick passes (0: the library default)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    # fixed CTAs per SM of the level-0 MGPCG passes (0: the library default)
    ap.add_argument("--mg-ctas-per-sm", type=int, default=0)
    # multigrid preconditioner: scale of each coarse-grid correction (1 = the reference's V-cycle),
    # red-black sweep pairs per smoothing, flexible PCG, coarsest-level iterations
    ap.add_argument("--mg-correction", type=float, default=PRECOND["mg_correction_scale"])
    ap.add_argument("--mg-sweeps", type=int, default=PRECOND["mg_smoothing_sweeps"])
    ap.add_argument("--pcg-flexible", type=int, default=PRECOND["pcg_flexible"])
    ap.add_argument("--mg-coarse-iterations", type=int, default=PRECOND["mg_coarse_iterations"])
    ap.add_argument("--mg-smoother-weight", type=float, default=PRECOND["mg_smoother_weight"])
    return ap.parse_args()


def make_scene(workload, default_fn, solver="mgpcg"):
    from slosh_b200 import _abi as A
    from slosh_b200 import scenes
    sv = A.SOLVER_RBGS if solver == "rbgs" else A.SOLVER_MGPCG
    if workload == "dam_break_64":
        sc = scenes.dam_break(default_fn, n=64, solver=sv)
        sc["settings"].sort_interval = 4
        sc["settings"].sor_weight = 1.9
        sc["settings"].pressure_iterations = 200
    elif workload == "boxes_512":
        sc = scenes.boxes_512(default_fn)
    elif workload.startswith("dam_break_sphere_") and workload[17:].isdigit() and int(workload[17:]) % 8 == 0 \
            and 32 <= int(workload[17:]) <= 256:
        sc = scenes.dam_break_sphere(default_fn, n=int(workload[17:]), solver=sv, sor_iterations=200)
    else:
        raise SystemExit(f"unknown workload {workload!r} (tanks_64 runs the batched tanks)")
    sc["settings"].max_substeps = 16  # CFL 1 holds; the plugin's default cap of 4 would exceed it
    return sc


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        rows = [r for r in self.rows if r[0] == str(self.index)] or self.rows
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def cpu_baseline_sample(workload, solver="mgpcg"):
    """One substep of the same workload by the C++ oracle on all host cores (bounded: ~10-30 s)."""
    from oracle import oracle as O
    from slosh_b200 import _abi as A
    O.build()
    cores = O.set_threads(os.cpu_count() or 1)
    sc = make_scene(workload, O.settings_default, solver)
    o = O.Oracle(sc["settings"])
    o.set_emit_seed(sc["seed"])
    fi = A.frame_input(sc["settings"], emits=sc["emits"], colliders=sc.get("colliders", []))
    n, _ = o.begin_frame(fi)
    t0 = time.perf_counter()
    o.substep(0)
    el = time.perf_counter() - t0
    o.close()
    return {"value": 1.0 / el, "unit": "substeps/s", "cores": cores, "kind": "port",
            "sample": f"1 substep (frame 1, substep 0 of {n}) of {sc['name']}, {sc['particles']} particles, "
                      f"C++ oracle with OpenMP, {el:.2f} s"}


def run_reference(args):
    """The reference path's CPU restatement on all host cores, over the same window as the GPU arm: the
    emission frame and max(W, 3) - 1 more frames untimed (the GPU arm's warm-up), then `steps` substeps of
    the frames that follow, timed one by one. The reference runs its own V-cycle (correction scale 1)."""
    world, rank, _ = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
    if rank != 0:
        return
    from oracle import oracle as O
    from slosh_b200 import _abi as A
    O.build()
    cores = O.set_threads(os.cpu_count() or 1)
    sc = make_scene(args.workload, O.settings_default, args.solver)
    o = O.Oracle(sc["settings"])
    o.set_emit_seed(sc["seed"])
    cols = sc.get("colliders", [])
    o.step_frame(A.frame_input(sc["settings"], emits=sc["emits"], colliders=cols))  # frame 1: scene creation
    fi = A.frame_input(sc["settings"], colliders=cols)
    warm_frames = max(args.warmup, 3) - 1
    for _ in range(warm_frames):
        o.step_frame(fi)
    pending = []
    iters = []
    state = {"open": False}

    def next_substep():
        if not pending:
            if state["open"]:
                o.end_frame()
            n, _ = o.begin_frame(fi)
            pending.extend(range(n))
            state["open"] = True
        o.substep(pending.pop(0))
        iters.append(o.results().last_solve_iterations)

    el = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        next_substep()
        el += time.perf_counter() - t0
    value = args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "substeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": sc["name"], "grid": list(sc["settings"].grid_dim), "particles": sc["particles"],
                   "solver": "MGPCG" if args.solver == "mgpcg" else "RBGS omega 1.9 x200",
                   "tolerance": 1e-6 if args.solver == "mgpcg" else None, "transfer": "APIC", "cfl": 1.0,
                   "frame_dt": 1.0 / 120.0, "sort_interval": 4, "parallelism": "host threads",
                   "step": "one substep (the GPU arm's step is one frame; both report substeps/s)",
                   "window": f"frames 1-{warm_frames + 1} untimed, then {args.steps} substeps from frame {warm_frames + 2}",
                   "preconditioner": {"mg_correction_scale": 1.0, "mg_smoothing_sweeps": 1, "pcg_flexible": False,
                                      "mg_coarse_iterations": 16, "mg_smoother_weight": 1.0}},
        "pressure_iterations_mean": statistics.mean(iters) if iters else None,
        "cpu_baseline": {"value": value, "unit": "substeps/s", "cores": cores, "kind": "port",
                         "sample": f"{args.steps} substeps of {sc['name']} from frame {warm_frames + 2}, C++ oracle with OpenMP"},
        "e2e": {"value": value, "unit": "substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    o.close()
    print(json.dumps(line), flush=True)


def _timed_frames(sim, fi, steps, stream, phases):
    """Steps `steps` frames on the simulation's stream: device time (CUDA events on that stream), host
    wall time around the public calls, and per-frame solver statistics."""
    import torch
    out = {"phase": {k: 0.0 for k in phases}, "substeps": 0, "iters": [], "rels": [], "trues": [], "active": 0}
    l0 = sim.launch_count()
    h0, d0 = sim.transfer_bytes()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ev0.record(stream)
    for _ in range(steps):
        sim.step_frame(fi)
        r = sim.results()
        out["substeps"] += r.substeps
        out["iters"].append(r.last_solve_iterations)
        out["rels"].append(r.last_solve_rel_residual)
        out["trues"].append(r.last_solve_true_rel_residual)
        out["active"] = max(out["active"], int(r.raw_stats[7]))
        for k, v in sim.phase_ms().items():
            out["phase"][k] += v
    ev1.record(stream)
    torch.cuda.synchronize()
    out["wall_ms"] = (time.perf_counter() - t0) * 1000.0
    out["dev_ms"] = ev0.elapsed_time(ev1)
    out["launches"] = sim.launch_count() - l0
    h1, d1 = sim.transfer_bytes()
    out["h2d"], out["d2h"] = h1 - h0, d1 - d0
    return out


def _scene_sim(args, S, A, local, settings_fn=None):
    """The workload's simulation on its own stream, stepped through the emission frame (frame 1)."""
    import torch
    sc = make_scene(args.workload, S.settings_default, args.solver)
    sc["settings"].precision_mode = {"fp32": A.PRECISION_FP32, "fp16": A.PRECISION_FP16_STORAGE,
                                     "bf16": A.PRECISION_BF16_STORAGE}[args.precision]
    precond = apply_precond(sc["settings"], args)
    if settings_fn:
        precond = settings_fn(sc["settings"], precond)
    sim = S.Simulation(sc["settings"], device=local)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.set_emit_seed(sc["seed"])
    if args.ctas_per_sm > 0:
        sim.set_ctas_per_sm(args.ctas_per_sm)
    if args.mg_ctas_per_sm > 0:
        sim.set_mg_ctas_per_sm(args.mg_ctas_per_sm)
    cols = sc.get("colliders", [])
    sim.step_frame(A.frame_input(sc["settings"], emits=sc["emits"], colliders=cols))  # scene creation (frame 1)
    return sc, sim, stream, A.frame_input(sc["settings"], colliders=cols), precond


def run_slosh(args):
    world, rank, local = dist_setup(args.gpus)
    import torch

    import slosh_b200 as S
    from slosh_b200 import _abi as A
    from slosh_b200.replicas import reduce_run
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
    sc, sim, stream, fi, precond = _scene_sim(args, S, A, local)
    tuned = None
    if args.autotune:
        r = sim.autotune(fi, frames=1)
        tuned = {"ctas_per_sm": int(r.best_ctas_per_sm), "brick_ctas": int(r.brick_ctas),
                 "ms_per_substep": {int(r.ctas_per_sm[k]): round(float(r.ms_per_substep[k]), 4) for k in range(r.num_candidates)}}
    for _ in range(max(args.warmup, 3) - 1):
        sim.step_frame(fi)
    sim.enable_phase_timing(True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    run = _timed_frames(sim, fi, args.steps, stream, S.PHASES)
    clk = clocks.stop()
    sim.close()
    substeps, phase, iters, rels, trues, active = (run["substeps"], run["phase"], run["iters"], run["rels"], run["trues"],
                                                   run["active"])
    launches = run["launches"]
    total_substeps, dev_ms, wall_ms = reduce_run(substeps, run["dev_ms"], run["wall_ms"])
    # The same workload with the reference's V-cycle (correction scale 1, one sweep pair, plain PCG), timed
    # the same way on a fresh simulation: what the preconditioner options change.
    ref_vc = None
    if args.solver == "mgpcg" and not args.no_reference_vcycle:
        def ref_settings(st, _):
            st.mg_correction_scale, st.mg_smoothing_sweeps, st.pcg_flexible, st.mg_coarse_iterations = 1.0, 1, 0, 16
            st.mg_smoother_weight = 1.0
            return None
        _, sim2, stream2, fi2, _ = _scene_sim(args, S, A, local, ref_settings)
        for _ in range(max(args.warmup, 3) - 1):
            sim2.step_frame(fi2)
        sim2.enable_phase_timing(True)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        run2 = _timed_frames(sim2, fi2, args.steps, stream2, S.PHASES)
        sim2.close()
        t2, dev2, _ = reduce_run(run2["substeps"], run2["dev_ms"], run2["wall_ms"])
        ref_vc = {"value": t2 / (dev2 * 1e-3), "unit": "substeps/s",
                  "pressure_solve_ms": run2["phase"]["pressure"] / max(run2["substeps"], 1),
                  "pressure_iterations_mean": statistics.mean(run2["iters"]) if run2["iters"] else None,
                  "pressure_rel_residual_max": max(run2["rels"]) if run2["rels"] else None,
                  "preconditioner": {"mg_correction_scale": 1.0, "mg_smoothing_sweeps": 1, "pcg_flexible": False,
                                     "mg_coarse_iterations": 16, "mg_smoother_weight": 1.0}}
    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    n_particles = sc["particles"]
    peak, peak_kind = measured_peak()
    active_cells = active * 512
    # Roofline of the dominant single-kernel phase: algorithmic bytes per launch / event-timed duration.
    algo = {"g2p": 96.0 * n_particles + 16.0 * active_cells, "p2g": 48.0 * n_particles + 28.0 * active_cells}
    dom = max(("g2p", "p2g"), key=lambda k: phase[k])
    per_launch_ms = phase[dom] / max(substeps, 1)
    achieved = algo[dom] / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        try:
            with open(tp) as f:
                tj = json.load(f)
            if dom in tj and tj[dom].get("workload") == sc["name"]:
                traffic = tj[dom]["bytes_per_launch"]
        except Exception:
            traffic = None
    line = {
        "metric": METRIC if sc["name"] == "dam_break_sphere_256" else f"FLIP substeps/s, {sc['name']}",
        "value": total_substeps / (dev_ms * 1e-3), "unit": "substeps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": sc["name"], "grid": list(sc["settings"].grid_dim), "particles": n_particles,
                   "solver": "MGPCG" if args.solver == "mgpcg" else "RBGS omega 1.9 x200", "tolerance": 1e-6 if args.solver == "mgpcg" else None, "transfer": "APIC", "cfl": 1.0, "frame_dt": 1.0 / 120.0,
                   "sort_interval": 4, "parallelism": f"replicas{world}", "step": "one frame of CFL substeps",
                   "mg_coarse_storage": args.precision, "preconditioner": precond, "autotune": tuned,
                   "l2": f"inputs larger than L2 (particles {48.0 * n_particles / 1e9:.2f} GB)"},
        "substeps": total_substeps,
        "particle_updates_per_s": total_substeps * n_particles / (dev_ms * 1e-3),
        "pressure_solve_ms": phase["pressure"] / max(substeps, 1),
        "pressure_iterations_mean": statistics.mean(iters) if iters else None,
        "pressure_rel_residual_max": (max(rels) if rels else None) if args.solver == "mgpcg" else None,
        "pressure_true_rel_residual_max": max(trues) if trues else None,
        "reference_vcycle": ref_vc,
        "phase_ms_per_substep": {k: v / max(substeps, 1) for k, v in phase.items()},
        "clocks": clk,
        "e2e": {"value": total_substeps / (wall_ms * 1e-3), "unit": "substeps/s",
                "h2d_bytes_per_step": run["h2d"] // args.steps, "d2h_bytes_per_step": run["d2h"] // args.steps},
        "gpu_launches": launches,
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                     "algorithmic_bytes_per_launch": algo[dom]},
    }
    if world == 1 and not args.no_cpu_baseline:
        torch.cuda.synchronize()
        try:
            line["cpu_baseline"] = cpu_baseline_sample(args.workload, args.solver)
        except Exception as e:  # keep the GPU line even if the host sample fails
            line["cpu_baseline"] = {"value": None, "unit": "substeps/s", "error": str(e)[:200]}
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_tanks(args):
    """Batched tanks: every rank steps its LPT share of independent tanks, one frame each per step."""
    world, rank, local = dist_setup(args.gpus)
    import torch

    import slosh_b200 as S
    from slosh_b200 import _abi as A
    from slosh_b200 import scenes
    from slosh_b200.replicas import gather_tank_stats, lpt_partition, reduce_run
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
    tanks = scenes.tank_batch(S.settings_default, count=args.tanks)
    precond = None
    for t in tanks:
        precond = apply_precond(t["settings"], args)
    plan = lpt_partition([t["cost"] for t in tanks], world)
    mine = plan[rank]
    sims, streams = [], []
    for k in mine:
        sim = S.Simulation(tanks[k]["settings"], device=local)
        st = torch.cuda.Stream()
        sim.set_stream(st.cuda_stream)
        sim.set_emit_seed(tanks[k]["seed"])
        sims.append(sim)
        streams.append(st)
    S.step_frames(sims, [A.frame_input(tanks[k]["settings"], emits=tanks[k]["emits"]) for k in mine])
    nxt = [A.frame_input(tanks[k]["settings"]) for k in mine]
    tuned = None
    if args.autotune:  # each tank alone, one timed frame per candidate
        tuned = {}
        for sim, fi in zip(sims, nxt):
            r = sim.autotune(fi, frames=1)
            tuned[int(r.best_ctas_per_sm)] = tuned.get(int(r.best_ctas_per_sm), 0) + 1
    for _ in range(max(args.warmup, 3) - 1):
        S.step_frames(sims, nxt)

    def timed(batched):
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        join = torch.cuda.current_stream()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(join)
        for st in streams:
            st.wait_event(ev0)
        substeps = 0
        t0 = time.perf_counter()
        for _ in range(args.steps):
            if batched:
                S.step_frames(sims, nxt)
            else:
                for sim, fi in zip(sims, nxt):
                    sim.step_frame(fi)
            substeps += sum(sim.results().substeps for sim in sims)
        for st in streams:
            e = torch.cuda.Event()
            e.record(st)
            join.wait_event(e)
        ev1.record(join)
        torch.cuda.synchronize()
        wall = (time.perf_counter() - t0) * 1000.0
        return reduce_run(substeps, ev0.elapsed_time(ev1), wall)

    clocks = ClockSampler(local)
    clocks.start()
    h0 = [sim.transfer_bytes() for sim in sims]
    total, dev_ms, wall_ms = timed(True)
    h1 = [sim.transfer_bytes() for sim in sims]
    clk = clocks.stop()
    seq_total, seq_dev_ms, seq_wall_ms = timed(False)

    # Per-tank substep latency: one more frame of every tank with phase events on the tanks' own
    # streams (outside the timed region); a tank's latency is its frame's device time / its substeps,
    # batched (sharing the GPU with the other tanks) and one tank at a time.
    def latencies(batched):
        for sim in sims:
            sim.enable_phase_timing(True)
        if batched:
            S.step_frames(sims, nxt)
        else:
            for sim, fi in zip(sims, nxt):
                sim.step_frame(fi)
        out = [sum(sim.phase_ms().values()) / max(sim.results().substeps, 1) for sim in sims]
        for sim in sims:
            sim.enable_phase_timing(False)
        return out
    lat_b = latencies(True)
    lat_s = latencies(False)
    rows = gather_tank_stats([(k, sim.results().substeps, sim.results().last_solve_iterations, sim.results().fluid_cells, lb, ls)
                              for k, sim, lb, ls in zip(mine, sims, lat_b, lat_s)], width=6)
    for sim in sims:
        sim.close()
    if rank == 0:
        particles = sum(t["particles"] for t in tanks)
        h2d = sum(b[0] - a[0] for a, b in zip(h0, h1)) // args.steps
        d2h = sum(b[1] - a[1] for a, b in zip(h0, h1)) // args.steps
        line = {
            "metric": f"tank substeps/s, {args.tanks} independent tanks 32^3-128^3, batched", "value": total / (dev_ms * 1e-3),
            "unit": "substeps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"tanks_{args.tanks}", "tanks": args.tanks, "particles": particles, "solver": "MGPCG",
                       "preconditioner": precond,
                       "autotune_ctas_per_sm_counts": tuned,
                       "tolerance": 1e-6, "step": "one frame of every tank", "parallelism": f"lpt{world}",
                       "l2": "inputs larger than L2 (1.3 GB of particles)"},
            "sequential": {"value": seq_total / (seq_dev_ms * 1e-3), "ms_per_step": seq_dev_ms / args.steps},
            "tank_iterations_mean": statistics.mean(r[2] for r in rows) if rows else None,
            "tank_substep_latency_ms": {
                "batched_p50": float(np.percentile([r[4] for r in rows], 50)), "batched_p99": float(np.percentile([r[4] for r in rows], 99)),
                "sequential_p50": float(np.percentile([r[5] for r in rows], 50)),
                "sequential_p99": float(np.percentile([r[5] for r in rows], 99))},
            "clocks": clk,
            "e2e": {"value": total / (wall_ms * 1e-3), "unit": "substeps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": None, "roofline": None, "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_warm_start(args):
    """Learned warm start at 128^3: held-out randomised scenes (seeds 90000+), the first frame's pressure
    solve from a zero guess and from the trained network's guess (weights slosh_b200/warmstart_128.npz,
    trained on 20k MGPCG pairs by slosh_b200.train_warmstart); --steps scenes (default 200 here)."""
    world, rank, local = dist_setup(args.gpus)
    import torch
    from slosh_b200 import train_warmstart as TW
    torch.cuda.set_device(local)
    if rank != 0:
        return
    path = os.path.join(ROOT, "slosh_b200", "warmstart_128.npz")
    if not os.path.exists(path):
        print(json.dumps({"metric": "pressure-solve ms at 128^3, learned warm start", "unavailable": "no trained weights"}))
        return
    scenes = args.steps if args.steps != 10 else 200
    clocks = ClockSampler(local)
    clocks.start()
    ev = TW.evaluate(TW.load_weights(path), scenes=scenes, n=128)
    clk = clocks.stop()
    line = {
        "metric": "pressure-solve ms at 128^3 to 1e-6, learned warm start (zero guess beside it)",
        "value": ev["pressure_ms_learned"], "unit": "ms", "n_gpus": 1, "steps": scenes, "warmup": 0,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 network, f32 solve", "data": "synthetic",
        "config": {"workload": "warm_start_128", "grid": [128, 128, 128], "scenes": scenes, "scene_seeds": "90000+",
                   "network": "3-D U-Net, 4 levels, 16/32/64/64 channels, 3x3x3, BF16/FP32-accumulate",
                   "solver": "MGPCG", "tolerance": 1e-6},
        "evaluation": ev, "clocks": clk, "gpu_launches": None, "roofline": None, "cpu_baseline": None,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload.startswith("tanks"):
        run_tanks(args)
    elif args.workload == "warm_start_128":
        run_warm_start(args)
    else:
        run_slosh(args)


if __name__ == "__main__":
    main()
