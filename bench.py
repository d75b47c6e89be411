#!/usr/bin/env python3
"""Throughput of the per-step particle hot path on B200: particle-steps/s.

Workload: the 3D delta+-SPH dam break (sigmasph_b200.scenes.dambreak3d), 1,000,188 fluid
particles at dx = 4.762 mm, reflecting tank walls.  A step is one SPHBase.step(): the
step-start binning and neighbour search (each step's pairs are the reference's sweep
against fresh bins, filtered from candidate lists within 1.1 h that are built again, with
the reorder of every persistent field, whenever the particles' displacement since the
last build could exceed 0.05 h), the five pair passes of the delta+-SPH substep, advect,
particle shifting and the walls.  The state (>= 0.9 GB with the lists) is far larger
than the 126 MB L2, so no flush is needed between steps.  The line reports how many of
the timed steps built the lists.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload dambreak3d|tensile_bar3d|tensile_bar3d_jc|strips256] [--dx DX]

`--workload tensile_bar3d` times the hypoelastic solid step instead: the 3D round-bar
tensile test (sigmasph_b200.scenes.tensile_bar3d), about 2.3M particles at dx = 0.113 mm.
`--workload strips256` times 256 independent plane-strain strips (about 6M particles) as
packed ensembles.

Besides `value` and `e2e`, the line carries `roofline` (the dominant kernel's algorithmic
bytes over its event-timed launch, against the measured HBM copy peak, with its ncu DRAM
traffic), `issue_roofline` (the same kernel's warp instructions, from ncu, over its launch
against the GPU's instruction issue rate: the bound the pair passes sit at),
`step_roofline` (the whole step's algorithmic bytes), `fp32_bound` (the step's
estimated FP32 work against the FP32 FMA peak that `sph_fma_peak` measures on the same
GPU), `kernel_ms_per_step` (CUDA events around every kernel of eager steps on a copy of
the workload warmed up the same way: the same steps of the simulation as the timed
window), `neighbour_lists` (list builds among the timed steps), `steady_state` (200 steps
from step 400 on, or right after the timed window if that ends later: the flow is faster
there and the lists are built more often, so the build cost is amortised), `drift` (the energy balance over the timed window from the
library's FP64 reductions) and `clocks`.

Under torchrun (N > 1) every rank runs an independent replica of a single scene (it does
not shard at one-GPU scale: replicas only); the strip ensemble is sharded instead, each
rank stepping its share of the strips.  The time is the max over ranks.
`--impl reference` times the reference's algorithm on the host cores: the CPU
restatement of the reference's kernels (the reference itself is Taichi, not installed
and not installable here), float32, all host threads, on rank 0 only.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "particle-steps/s on 1 B200 (3D delta+-SPH dam break)"
METRIC_BAR = "particle-steps/s on 1 B200 (3D round-bar tensile test)"
UNIT = "particle-steps/s"
DX_1M = 0.004762
DX_BAR = 0.113

# Algorithmic (compulsory, own-particle) bytes per particle of each kernel: the fields it
# must read and write once in float32; neighbour data is assumed served on chip.
ALGO_BYTES = {
    "k_vlist_build": 16 + 16 + 4,      # pos + cell read, count write (list entries: design)
    "k_nbr_filter": 16 + 16 + 4 + 4,   # pos + cell + candidate count read, count write
    "k_cells": 16 + 16 + 16,           # pos + build pos read, coarse cell write
    "k_lam": 16 + 4 + 32,              # pos read; lam + L (8 floats) write
    "k_lamgrad_cont": 16 + 16 + 16 + 32 + 4 + 16 + 16,  # pos vel shift L lam read; lgrad, div write
    "k_eos": 16 + 4 + 4 + 16 + 4 + 16,  # pos, div, V_lo, vel.m read; pos.V, V_lo, p, acc write
    "k_force": 16 + 16 + 16 + 16 + 16 + 16,  # pos vel disp shift acc read; acc write
    "k_advect": 16 + 16 + 16 + 16 + 16 + 16 + 16,
    "k_pst": 16 + 16 + 4 + 16 + 16,   # pos vel lam lgrad read; shift write
    "k_finish": 16 * 6 + 16 * 4,
    "k_gather": 2 * (16 * 5 + 4) + 16,
    # solid passes: the compulsory own-particle bytes of the reference passes they fuse
    "k_solid_a": 56 + 64,              # grad lambda + grad v
    "k_solid_b": 144,                  # Jaumann + ALE(s, eps_p, e) + return map + e update
    "k_solid_force": 132,              # EOS + stress force + in-loop hourglass + dt pairs
    "k_solid_commit": 64,              # continuity (V) + commit of the returned state
}
# Compulsory own-particle bytes of a whole delta+-SPH particle-step (sort/reorder 168,
# lambda/L 44, grad lambda 56, continuity 64, EOS + force + dt 60, advect 84, PST 60,
# displace 60), neighbour gathers assumed served on chip.
STEP_ALGO_BYTES = 600
# The hypoelastic solid step without the sub-cycled damper: sort 340, lambda/L 44, grad
# lambda 56, grad v 64, Jaumann + ALE + return + energy 144, continuity 64, EOS + force +
# in-loop hourglass + dt 132, advect + grips 88, PST 64, displace 60.
STEP_ALGO_BYTES_SOLID = 1060
# FP32 work per particle-step (the secondary bound): five pair passes over ~80 neighbours
# at ~50 FLOP per pair (fluid, 2.6 dx); ten pair-pass equivalents over ~113 neighbours at
# ~60 FLOP (3D solid at 3 dx, in-loop damper).
STEP_FLOP_FLUID = 5 * 80 * 50
STEP_FLOP_SOLID = 10 * 113 * 60


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes per particle of one launch of the dominant kernels (ncu dram__bytes_read.sum
# + dram__bytes_write.sum over the particles of the captured case, in the workload's own
# configuration at 256k (dam break) and 219k (bar) particles: a --set full capture at full
# size is too large to run safely).  The traffic of these kernels grows in proportion to the particles, so the line
# scales them by the particle count.  Measured with the commands recorded beside the
# figures under profiles/.
NCU_DRAM_BYTES_PER_PARTICLE = {
    "dambreak3d": {"k_pst": 421.7, "k_force": 421.8, "k_lamgrad_cont": 443.3, "k_lam": 354.8,
                   "k_nbr_filter": 230.3},
    "tensile_bar3d": {"k_solid_force": 559.6, "k_solid_b": 665.3, "k_solid_a": 542.3, "k_pst": 630.5},
}


# Warp instructions per particle of one launch (ncu smsp__inst_executed.sum over the
# particles of the same captures).  The pair passes are bound by instruction issue, not by
# DRAM: the issue roofline is the GPU's SMs x 4 schedulers x one warp instruction per
# cycle at the clock sampled during the timed window.
NCU_WARP_INST_PER_PARTICLE = {
    "dambreak3d": {"k_pst": 326.0, "k_force": 341.7, "k_lamgrad_cont": 292.6, "k_lam": 127.7,
                   "k_nbr_filter": 114.2},
    "tensile_bar3d": {"k_solid_force": 593.8, "k_solid_b": 386.8, "k_solid_a": 372.5, "k_pst": 347.6},
}


def scaled_traffic(kernel, tag, n):
    per = NCU_DRAM_BYTES_PER_PARTICLE.get(tag, {}).get(kernel)
    return None if per is None else per * n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"sph_b200_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [t.strip() for t in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower() == "active":
                        reasons.add(nm)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    from sigmasph_b200.replicas import env_ranks
    return env_ranks()


def workload(args):
    """(scene, config description, profile tag) of the selected workload."""
    from sigmasph_b200.scenes import dambreak3d, tensile_bar3d
    if args.workload == "dambreak3d":
        dx = args.dx or DX_1M
        return (dambreak3d(dx=dx),
                {"workload": "3D dam break, delta+-SPH, reflecting walls", "dx_m": dx,
                 "support_dx": 2.6}, "dambreak3d")
    dx = args.dx or DX_BAR
    plast = "jc" if args.workload == "tensile_bar3d_jc" else "j2"
    return (tensile_bar3d(dx=dx, plasticity=plast),
            {"workload": "3D round-bar tensile test, hypoelastic %s, ALE + hourglass, grips"
                         % ("Johnson-Cook" if plast == "jc" else "J2 linear hardening"),
             "dx_mm": dx, "support_dx": 3.0}, "tensile_bar3d")


def cpu_baseline(ps, steps_target_s=15.0, max_steps=6, threads=None):
    """The CPU restatement (float32, all host threads) on the same workload."""
    from oracle.oracle import Oracle, state_from_sets
    from sigmasph_b200.solver import build_params
    nt = Oracle.threads(threads or os.cpu_count())
    p = build_params(ps)
    st = state_from_sets(ps.state_numpy())
    orc = Oracle(p, ps.particle_max_num, fp64=False)
    orc.set_state(st, p.CFL * p.support_radius / p.c_signal)
    orc.stage(0)
    t0 = time.perf_counter()
    orc.step(1)       # warm-up step
    t_warm = time.perf_counter() - t0
    k = max(1, min(max_steps, int(steps_target_s / max(t_warm, 1e-3))))
    t0 = time.perf_counter()
    orc.step(k)
    el = time.perf_counter() - t0
    return {"value": ps.particle_max_num * k / el, "unit": UNIT, "cores": nt,
            "kind": "port",
            "sample": f"{k} step(s) of the full {ps.particle_max_num}-particle workload after 1 "
                      f"warm-up step, CPU restatement of the reference kernels (float32, "
                      f"OpenMP, {nt} threads, every per-particle loop parallel: grid ids, sort and "
                      f"permutation, pair sweeps, advect, walls and reductions); the reference's "
                      f"own Taichi run is not installable"}


def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return 0
    from sigmasph_b200.config import SimConfig
    from sigmasph_b200.particle_system import ParticleSystem
    from oracle.oracle import Oracle, state_from_sets
    from sigmasph_b200.solver import build_params
    scene, desc, _ = workload(args)
    ps = ParticleSystem(SimConfig(scene), device="cpu")
    nt = Oracle.threads(os.cpu_count())
    p = build_params(ps)
    orc = Oracle(p, ps.particle_max_num, fp64=False)
    orc.set_state(state_from_sets(ps.state_numpy()), p.CFL * p.support_radius / p.c_signal)
    orc.stage(0)
    # A bounded sample: one warm-up step, then as many of the K steps as fit in about
    # 90 s of host time (a step of the 1M-particle workload takes about a second).
    t0 = time.perf_counter()
    orc.step(1)
    t_w = time.perf_counter() - t0
    k = max(1, min(args.steps, int(90.0 / max(t_w, 1e-3))))
    t0 = time.perf_counter()
    orc.step(k)
    el = time.perf_counter() - t0
    n = ps.particle_max_num
    val = n * k / el
    metric = METRIC if args.workload == "dambreak3d" else METRIC_BAR
    line = {"impl": "reference", "metric": metric, "value": val, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * el / k, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(desc, particles=n, parallelism="host threads"),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": nt, "kind": "port",
                             "sample": f"the full {n}-particle workload, 1 warm-up + {k} timed "
                                       f"step(s) (of the {args.steps} asked, bounded to ~90 s); "
                                       "CPU restatement of the reference kernels, float32, "
                                       "OpenMP with every per-particle loop parallel, sort "
                                       "included (the reference's Taichi is not installable here)"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_strips(args):
    """256 plane-strain Johnson-Cook strips (2k-60k particles each, ~6M in all) as packed
    size buckets with autotuned block sizes; a step is one step of every strip (each with
    its own dt), two steps per CUDA-graph launch."""
    import torch
    from sigmasph_b200.ensemble import Ensemble, shard, strip_specs, STATE_COLUMNS
    from sigmasph_b200.replicas import Replicas
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    all_specs = strip_specs(256)
    # the strips are independent: with N GPUs each steps its share (balanced by particles)
    own = shard(all_specs, ws, rank)
    specs = [all_specs[k] for k in own]
    ens = Ensemble(specs, buckets=args.buckets)
    tune = ens.autotune(candidates=(64, 128, 256), steps=4)
    ens.capture()
    for _ in range(max(args.warmup // 2, 2)):
        ens.step2()
    torch.cuda.synchronize()
    n = ens.particles
    K2 = max(args.steps // 2, 1)
    clocks = ClockSampler(local)
    rep.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(K2):
        ens.step2()
    e1.record()
    torch.cuda.synchronize()
    rep.barrier()
    ck = clocks.stop()
    ms = rep.max_over_ranks(e0.elapsed_time(e1))
    n_all = int(rep.sum_over_ranks(n))
    value = n_all * 2 * K2 / (ms / 1000.0)
    # end to end: after every launch read every strip's state (clock, dt, grip forces)
    rep.barrier()
    t0 = time.perf_counter()
    nread = 0
    for _ in range(K2):
        ens.step2()
        for b in ens.buckets:
            nread += len(b.state())
    el = rep.max_over_ranks(time.perf_counter() - t0)
    # the one exchange of the sharded ensemble: every strip's final state, in float64
    table = rep.gather_rows(ens.state_rows(), own, len(all_specs))
    from sigmasph_b200 import abi
    import ctypes as C
    d2h = C.sizeof(abi.SphInstState) * len(specs) // 2
    launches = 0
    for b in ens.buckets:                     # kernels of one step, counted on an eager step
        b.solver.profile(True)
        b.solver.profile_read()
        b.solver.step()
        launches += sum(cnt for _, cnt in b.solver.profile_read().values())
        b.solver.profile(False)
    line = {"metric": "particle-steps/s on 1 B200 (256 plane-strain strip ensemble)", "value": value,
            "unit": UNIT, "n_gpus": ws, "steps": 2 * K2, "warmup": args.warmup,
            "ms_per_step": ms / (2 * K2), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "256 plane-strain JC strips packed in %d handle(s), one graph launch per 2 steps"
                                   % len(ens.buckets),
                       "particles": n_all, "strips": len(all_specs), "buckets": tune,
                       "parallelism": ("strips sharded over %d GPUs (largest first, balanced by "
                                       "particles); no per-step collective, one float64 gather "
                                       "of the final states" % ws) if ws > 1 else "single GPU",
                       "l2": "inputs larger than L2 (state + neighbour lists > 1 GB)"},
            "e2e": {"value": n_all * 2 * K2 / el, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": d2h},
            "gathered": {"strips": int(table.shape[0]),
                         "sim_time_min": float(table[:, STATE_COLUMNS.index("sim_time")].min()),
                         "sim_time_max": float(table[:, STATE_COLUMNS.index("sim_time")].max())},
            "gpu_launches": launches * 2 * K2}
    if ck is not None:
        line["clocks"] = ck
    if rep.reporter:
        print(json.dumps(line))
    rep.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=6)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--workload", default="dambreak3d",
                    choices=("dambreak3d", "tensile_bar3d", "tensile_bar3d_jc", "strips256"))
    ap.add_argument("--buckets", type=int, default=1,
                    help="strips256: size buckets (one: every strip in one handle, measured "
                         "16.0 ms per ensemble step against 16.5 ms with four)")
    ap.add_argument("--dx", type=float, default=None)
    ap.add_argument("--jc-surrogate", default=None,
                    help="tensile_bar3d_jc only: surrogate parameters (.npy), e.g. "
                         "sigmasph_b200/data/jc_surrogate_config0.npy")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="eager profiled steps (0: as many as the timed window)")
    ap.add_argument("--steady-after", type=int, default=400,
                    help="the steady window starts at this step (or after the timed one)")
    ap.add_argument("--steady-steps", type=int, default=200,
                    help="a longer window after the timed one, for the amortised build cost")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "strips256":
        return run_strips(args)

    import torch
    from sigmasph_b200.replicas import Replicas
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    rep = Replicas("nccl")
    from sigmasph_b200 import abi
    from sigmasph_b200.config import SimConfig
    from sigmasph_b200.particle_system import ParticleSystem
    scene, desc, tag = workload(args)
    if args.jc_surrogate:
        if args.workload != "tensile_bar3d_jc":
            raise SystemExit("--jc-surrogate applies to --workload tensile_bar3d_jc")
        from sigmasph_b200.surrogate import JCSurrogate
        sur = JCSurrogate.load(args.jc_surrogate)
        desc = dict(desc, jc_surrogate=os.path.basename(args.jc_surrogate), jc_surrogate_tol=1e-3)
    W = args.warmup + (args.warmup & 1)

    def warm_solver(single_step_graph):
        """The workload's particle system and solver after W warm-up steps (the CUDA
        graphs are captured there, outside any timed region)."""
        ps_ = ParticleSystem(SimConfig(scene), device=f"cuda:{local}")
        sv = ps_.build_solver()
        if args.jc_surrogate:
            sv.enable_jc_surrogate(sur, tol=1e-3)
        sv.initialize()
        if single_step_graph:
            sv.step_many(W - 1)
            sv.step()
        else:
            sv.step_many(W)
        torch.cuda.synchronize()
        return ps_, sv

    ps, solver = warm_solver(False)
    n = ps.particle_max_num
    cpu_ps = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu_ps = ParticleSystem(SimConfig(scene), device="cpu")
    stream = torch.cuda.current_stream()

    # ---------------------------------------------------------------- timed region
    K = args.steps
    solver.list_stats(reset=True)
    bud0 = solver.energy_budget()
    clocks = ClockSampler(local)
    rep.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.step_many(K)
    e1.record(stream)
    torch.cuda.synchronize()
    rep.barrier()
    ck = clocks.stop()
    ms = rep.max_over_ranks(e0.elapsed_time(e1))
    err = solver.error_word()
    lists = solver.list_stats()
    value = rep.throughput(n * K, ms / 1000.0)
    bud1 = solver.energy_budget()

    # ---------------------------------------------------------------- steady state
    # The window above starts right after the warm-up, while the flow is slow and the
    # candidate lists are rarely built; a window that starts at step --steady-after (or
    # right after the timed one, if later) shows the build cost amortised at the rate the
    # flow sets later on.
    Ks = args.steady_steps
    steady = None
    if Ks > 0:
        done = W + K
        if args.steady_after > done:
            solver.step_many(args.steady_after - done)
            done = args.steady_after
        solver.list_stats(reset=True)
        rep.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        solver.step_many(Ks)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_s = rep.max_over_ranks(e0.elapsed_time(e1))
        ls = solver.list_stats()
        steady = {"steps": Ks, "after_steps": done, "builds": ls["builds"],
                  "ms_per_step": ms_s / Ks, "value": rep.throughput(n * Ks, ms_s / 1000.0),
                  "unit": UNIT}

    # energy balance over the timed window (the library's FP64 reductions): the fluid's
    # E_bal = ke + se + pe - visc + wall - leftover changes only by the budget's residual
    # (delta-SPH diffusion, shift, wall clamp; DSPH.py:1800-1852), the solid's total
    # (ke + ie + hg + pe - leftover) by the viscous and wall work
    def e_bal(b):
        if tag == "dambreak3d":
            return b["ke"] + b["se"] + b["pe"] - b["visc"] + b["wall"] - b["leftover"]
        return b["total"]
    scale = max(abs(bud0["pe"]), abs(bud0["ke"]) + abs(bud0.get("ie", 0.0)), 1e-300)
    if tag == "dambreak3d":
        drift = {"window_steps": K, "E_bal_start": e_bal(bud0), "E_bal_end": e_bal(bud1),
                 "E_bal_change_rel": (e_bal(bud1) - e_bal(bud0)) / scale,
                 "diffusion_work_in_window_rel": (bud1["wd"] - bud0["wd"]) / scale,
                 "scale": "max(|pe|, ke + ie) at the window's start",
                 "fp64_oracle_comparison": "tests/test_drift_gpu.py (1000 steps at 128k particles)"}
    else:
        # the grips do work on the bar that no budget term holds (the reference's neither:
        # total(t) - total(0) = -wall + residual holds for undriven decks), so the change
        # of the total over the window is the energy put in, not a drift
        drift = {"window_steps": K, "total_start": e_bal(bud0), "total_end": e_bal(bud1),
                 "E_bal_change_rel": None,
                 "note": "driven by the grips' work, which no budget term holds; the solid's "
                         "work channels are checked against the FP64 oracle in tests/test_solid_gpu.py"}

    # ---------------------------------------------------------------- e2e through the public API
    # Per step, as the reference's driver loop does (run_simulation.py:1186-1209): write
    # dt from page-locked host memory, solver.step(), read dt back (synchronises).  On a
    # second copy of the workload, warmed up the same way, so that it covers the same
    # steps of the simulation as the device-timed region.
    Ke = args.e2e_steps or K
    ps_e, solver_e = warm_solver(True)
    dt = solver_e.dt[None]
    rep.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(Ke):
        solver_e.dt[None] = dt
        solver_e.step()
        dt = solver_e.dt[None]
    torch.cuda.synchronize()
    el = rep.max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": rep.throughput(n * Ke, el), "unit": UNIT, "h2d_bytes_per_step": 4,
           "d2h_bytes_per_step": 4, "steps": Ke,
           "window": "the same steps as the device-timed region, on a second copy of the workload"}
    del solver_e, ps_e
    torch.cuda.empty_cache()

    # ---------------------------------------------------------------- per-kernel timing
    # CUDA events around every kernel of eagerly launched steps, on a third copy warmed up
    # the same way: the same steps of the simulation as the timed window.
    ps_p, solver_p = warm_solver(False)
    solver_p.profile(True)
    solver_p.profile_read()
    Kp = min(K, args.profile_steps) if args.profile_steps > 0 else K
    for _ in range(Kp):
        solver_p.step()
    prof = solver_p.profile_read()
    solver_p.profile(False)
    del solver_p, ps_p
    torch.cuda.empty_cache()
    launches_per_step = sum(c for _, c in prof.values()) / max(Kp, 1)
    per_step_ms = {k: v[0] / Kp for k, v in prof.items()}
    dom = max(prof, key=lambda k: per_step_ms[k])
    if dom not in ALGO_BYTES:
        dom = max((k for k in prof if k in ALGO_BYTES), key=lambda k: per_step_ms[k])
    dom_ms = prof[dom][0] / prof[dom][1]
    peak, peak_kind = load_peaks()
    achieved = ALGO_BYTES[dom] * n / (dom_ms / 1000.0) / 1e9
    traffic = scaled_traffic(dom, tag, n)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "algorithmic_bytes_per_particle": ALGO_BYTES[dom],
                "launch_ms": dom_ms, "traffic": traffic,
                "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                                   "the same kernel on the same workload at %s particles, scaled by "
                                   "the particle count" % ("256,000" if tag == "dambreak3d" else "218,573"))
                                  if traffic else None}
    issue_roofline = None
    wi = NCU_WARP_INST_PER_PARTICLE.get(tag, {}).get(dom)
    if wi is not None:
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        mhz = (ck or {}).get("sm_mhz") or (ck or {}).get("sm_max_mhz")
        if mhz:
            peak_i = sms * 4 * mhz * 1e6
            ach_i = wi * n / (dom_ms / 1000.0)
            issue_roofline = {"bound": "issue", "kernel": dom, "achieved": ach_i, "peak": peak_i,
                              "unit": "warp-instructions/s", "frac": ach_i / peak_i,
                              "warp_instructions_per_particle": wi,
                              "peak_source": "%d SMs x 4 schedulers x the sampled %g MHz" % (sms, mhz),
                              "source": "ncu smsp__inst_executed.sum of one launch on the same workload "
                                        "at %s particles, scaled by the particle count"
                                        % ("256,000" if tag == "dambreak3d" else "218,573")}
    import ctypes as C
    fma = C.c_double(0.0)
    abi.check(abi.lib().sph_fma_peak(C.byref(fma), None), "sph_fma_peak")
    step_flop = STEP_FLOP_FLUID if tag == "dambreak3d" else STEP_FLOP_SOLID
    fp32_bound = {"flop_per_particle_step": step_flop, "achieved_tflops": step_flop * value / 1e12,
                  "peak_tflops": fma.value, "frac": step_flop * value / 1e12 / fma.value if fma.value else None,
                  "peak_source": "measured FP32 FMA microbenchmark (sph_fma_peak)"}
    step_bytes = STEP_ALGO_BYTES if tag == "dambreak3d" else STEP_ALGO_BYTES_SOLID
    step_gbs = step_bytes * value / 1e9
    step_roofline = {"bound": "hbm", "algorithmic_bytes_per_particle_step": step_bytes,
                     "achieved": step_gbs, "peak": peak, "unit": "GB/s", "frac": step_gbs / peak,
                     "peak_source": peak_kind}

    if rank == 0:
        metric = METRIC if args.workload == "dambreak3d" else METRIC_BAR
        line = {"metric": metric, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K,
                "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(desc, particles=n,
                               parallelism="replicas" if ws > 1 else "single GPU",
                               l2="inputs larger than L2 (state + neighbour lists > 0.5 GB)",
                               graph="two-step CUDA graph replayed"),
                "e2e": e2e, "gpu_launches": int(round(launches_per_step * K)),
                "neighbour_lists": {"timed_steps": lists["steps"], "builds": lists["builds"],
                                    "shift_searches": lists["shift_searches"]},
                "steady_state": steady, "drift": drift,
                "kernel_profile_window": f"{Kp} eager steps, the same steps of the simulation as the timed window",
                "roofline": roofline, "issue_roofline": issue_roofline,
                "step_roofline": step_roofline, "fp32_bound": fp32_bound,
                "kernel_ms_per_step": {k: round(v, 5) for k, v in sorted(per_step_ms.items(),
                                                                       key=lambda t: -t[1])},
                "error_word": err}
        if ck is not None:
            line["clocks"] = ck
        if cpu_ps is not None:
            try:
                line["cpu_baseline"] = cpu_baseline(cpu_ps)
            except Exception as e:  # the baseline is reported, not required
                line["cpu_baseline"] = {"value": None, "error": str(e)}
        print(json.dumps(line))
    rep.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
