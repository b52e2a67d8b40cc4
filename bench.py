#!/usr/bin/env python
"""Benchmark of the implicit MPM snow step on B200: particle-steps/s.

Headline workload: the 4,000,032-particle snow slab (1.0 x 0.2 x 0.5 m, 2x2x2 jittered particles per cell at
h = 1/171 m, per-particle E0 log-uniform in [1e5, 2e5] Pa) on a 30 degree plane, dt = 2.5e-4 s, conjugate
residuals to a 1e-5 relative residual (max 60 iterations), FP32 state with FP64 solver reductions.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One JSON line on rank 0.  N > 1 (launched by torch.distributed.run): N independent replicas, one per GPU (the
path has no exchange step to shard), weak scaling; the timed region is bracketed by a barrier and a device
synchronise on both sides and the time is the max over ranks.

value   : device-resident particle state, K steps of the C-ABI's mpm_step with the learned warm start (the
          packaged model mpmsnow_b200/warm_start_slab.npz, trained on slab sections of other seeds), timed with
          CUDA events recorded on the library's own stream (the step is host-synchronous, so the span is the
          whole step).  The same K steps of the plain solver (the reference's uniform initial guess) on a fresh
          handle are reported under "plain", and value / plain as "learned_vs_plain"; the same guess without
          the network (p*/m plus the previous step's correction) under "guess_without_network"; all solve to the
          same relative residual.  --no-warm-start times the plain solver only.
e2e     : the same K steps on a fresh handle after the same W warm-up steps, but every step uploads the particles'
          positions and velocities from pinned host memory and reads them back (mpm_set_variable /
          mpm_get_variable), as a host-resident caller would.
The default K = 100 is the headline run's length: the solver needs more iterations once the slab settles on the
plane, so a short early window would flatter every arm.
roofline: the operator pass (the dominant kernel), algorithmic bytes (172 B per particle visit: the reference's
          per-particle state an operator application reads) over its device time from per-launch CUDA events on
          the launching stream, against the measured HBM copy bandwidth; the same at the 280 B of the operator
          record the pass actually reads is reported beside it.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s at 4M particles, learned warm-start vs plain CR @1e-5 residual"
WORKLOAD = ("snow slab 1.0x0.2x0.5 m on a 30 degree plane, jittered 2x2x2 per cell, per-particle E0 log-uniform "
            "[1e5, 2e5] Pa")
UNIT = "particle-steps/s"
# The roofline's algorithmic bytes per particle visit of the CR operator pass: the reference's per-particle state
# that one application of the force-differential operator reads (x, vol, F, R, F^-T, G^-1, J, mu, lambda in FP32:
# 172 B).  The pass reads the step's operator record instead (window base 4 B, 24 B-spline weights 96 B, the
# 45-entry upper triangle of the particle's 9x9 linearised force map 180 B: 280 B), reported beside it.
OP_ALGORITHMIC_BYTES_PER_PARTICLE = 172
OP_RECORD_BYTES_PER_PARTICLE = 280
# dram__bytes_read.sum + dram__bytes_write.sum per particle visit of the operator pass (k_op_apply) in a one-launch
# ncu capture of the 40-cell section of the slab (935,680 particles, every particle visited)
OP_TRAFFIC_PER_PARTICLE = 322.0
SOLVE_MAX_ITERS = 60
SOLVE_TOL = 1e-5


def headline_scene(length_cells=171):
    """The headline slab; a smaller length_cells keeps its cross-section, spacing and density (profiling cases)."""
    from mpmsnow_b200 import scenes as S
    if length_cells == 171:
        return S.slab()
    return S.slab(cells=(length_cells, 34, 86), h=1.0 / 171)


AVALANCHE_WORKLOAD = ("large avalanche: 2.0x0.5x1.0 m block (16M particles, jittered lattice) on a 35 degree slope "
                      "with a vertical cylinder (r = 0.1 m) standing in the snow, h = 0.005 m, dt = 2e-4 s")


def cpu_sample_scene(length_cells):
    """The headline slab's cross-section (34 x 86 cells at h = 1/171 m) over a shorter length."""
    from mpmsnow_b200 import scenes as S
    return S.slab(cells=(length_cells, 34, 86), h=1.0 / 171)


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms; the samples of the timed region are kept."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.dev = device_index
        self.proc = None

    def start(self):
        """Starts sampling and returns once the first sample is written: nvidia-smi's start-up (NVML
        initialisation) holds driver locks that stall CUDA calls, so it must finish before a timed region."""
        self.offset = 0
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 10 and os.path.getsize(self.tmp.name) == 0 and self.proc.poll() is None:
            time.sleep(0.05)
        time.sleep(0.3)

    def mark(self):
        """Only samples written after this call count (the timed region's)."""
        self.offset = os.path.getsize(self.tmp.name)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.tmp.flush()
        self.tmp.seek(self.offset)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.tmp.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        # short: a rank that never joins or dies ends the others' next collective with an error
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reduce_max(pg, value):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def run_cpu_oracle(scene, steps, warmup, threads):
    """The FP32 restatement of the reference step (the oracle) on the host cores; returns seconds per step and
    the CR iterations per step of the timed steps."""
    from oracle import oracle as O
    O.build()
    sim = O.OracleSim(scene["x"], scene["m"], scene["h"], scene["snow"], scene["colliders"], scene["gravity"],
                      prec=32, threads=threads, mu0=scene.get("mu0"), lambda0=scene.get("lambda0"))
    for _ in range(warmup):
        sim.advance(scene["dt"], SOLVE_MAX_ITERS, SOLVE_TOL)
    iters = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        iters += sum(sim.advance(scene["dt"], SOLVE_MAX_ITERS, SOLVE_TOL)["iterations"])
    return (time.perf_counter() - t0) / max(steps, 1), iters / max(steps, 1)


def bench_reference(args, world, rank, pg):
    """--impl reference: the reference's CPU step (the FP32 oracle port; the reference itself does not build
    here) on all host cores, on a bounded sample of the headline workload: a section of the slab with its
    cross-section, spacing and material, stepped from rest.  The line names the section it timed."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    scene = cpu_sample_scene(args.ref_sample_cells)
    n = scene["x"].shape[0]
    sec, iters = run_cpu_oracle(scene, args.steps, args.warmup, threads)
    value = n / sec
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD + f" (section of {args.ref_sample_cells} cells' length)",
                       "particles": n, "headline_particles": headline_particle_count(), "h": scene["h"],
                       "dt": scene["dt"], "cr_tol": SOLVE_TOL, "cr_max_iters": SOLVE_MAX_ITERS,
                       "solver": "plain CR (the reference's uniform initial guess), FP32 oracle port on the host",
                       "cr_iterations_per_step": iters, "parallelism": f"cpu threads x{threads}"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{n}-particle section (length {args.ref_sample_cells} cells) of the headline "
                                       f"slab, {args.steps} timed steps after {args.warmup} warm-up from rest, "
                                       f"{iters:.1f} CR iterations per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def headline_particle_count(length_cells=171):
    """Particles of the headline slab (2 x 2 x 2 per cell over 171 x 34 x 86 cells) without building it."""
    return 8 * length_cells * 34 * 86


def default_warm_start():
    p = os.path.join(ROOT, "mpmsnow_b200", "warm_start_slab.npz")
    return p if os.path.exists(p) else None


def time_arm(args, scene, local, pg, model=None, e2e=False, network=True):
    """One arm on a fresh handle: W warm-up steps, then K steps timed with CUDA events on the library's stream
    (max over ranks); per-phase device times from the library's profiler; optionally the e2e loop."""
    import ctypes as C

    import torch

    from mpmsnow_b200 import capi
    from mpmsnow_b200 import sim as M

    L = capi.load()
    n = scene["x"].shape[0]
    sp = capi.MpmSolveParams(SOLVE_MAX_ITERS, SOLVE_TOL)
    st = capi.MpmStepStats()

    def fresh():
        """A new handle on the scene, warmed up by W steps: both loops below cover the same K steps."""
        sim = M.from_scene(scene, device=local)
        if model is not None:
            model.install(sim._h, min_nodes=0, network=network)
        stream = torch.cuda.ExternalStream(M.stream_ptr(sim), device=local)
        return sim, stream

    def step(sim):
        rc = L.mpm_step(sim._h, float(scene["dt"]), C.byref(sp), C.byref(st))
        if rc != 0:
            raise capi.MpmError(rc, L.mpm_last_error(sim._h).decode())
        return st.kernel_launches, st.total_iterations

    clocks = ClockSampler(local)
    clocks.start()
    sim, stream = fresh()
    for _ in range(args.warmup):
        step(sim)
    M.profile_enable(sim, True)
    barrier(pg)
    torch.cuda.synchronize(local)
    clocks.mark()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    iters = []
    for _ in range(args.steps):
        k, it = step(sim)
        launches += k
        iters.append(it)
    e1.record(stream)
    torch.cuda.synchronize(local)
    clk = clocks.stop()
    barrier(pg)
    ms_max = reduce_max(pg, e0.elapsed_time(e1))
    phases = M.profile_read(sim)
    M.profile_enable(sim, False)
    del sim
    ms_e2e = None
    iters_e2e = None
    if e2e:
        # host-resident caller: positions and velocities through pinned host memory every step, on a fresh
        # handle after the same warm-up, so the K steps are the same simulated steps as the device-resident loop
        sim, stream = fresh()
        for _ in range(args.warmup):
            step(sim)
        hp = torch.empty(3 * n, dtype=torch.float32).pin_memory()
        hv = torch.empty(3 * n, dtype=torch.float32).pin_memory()
        L.mpm_get_variable(sim._h, b"p", hp.data_ptr(), 3 * n)
        L.mpm_get_variable(sim._h, b"v", hv.data_ptr(), 3 * n)
        barrier(pg)
        torch.cuda.synchronize(local)
        e2 = torch.cuda.Event(enable_timing=True)
        e3 = torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        iters_e2e = []
        for _ in range(args.steps):
            for nm, buf in ((b"p", hp), (b"v", hv)):
                rc = L.mpm_set_variable(sim._h, nm, buf.data_ptr(), 3 * n)
                assert rc == 0, rc
            iters_e2e.append(step(sim)[1])
            for nm, buf in ((b"p", hp), (b"v", hv)):
                rc = L.mpm_get_variable(sim._h, nm, buf.data_ptr(), 3 * n)
                assert rc == 0, rc
        e3.record(stream)
        torch.cuda.synchronize(local)
        barrier(pg)
        ms_e2e = reduce_max(pg, e2.elapsed_time(e3))
        del sim
    return {"ms": ms_max, "iters": iters, "launches": launches, "phases": phases, "clocks": clk, "ms_e2e": ms_e2e,
            "iters_e2e": iters_e2e}


def bench_b200(args, world, rank, local, pg):
    import numpy as np

    from mpmsnow_b200 import build

    build.build()
    if args.workload == "avalanche":
        from mpmsnow_b200 import scenes as S
        scene = S.avalanche()
    else:
        scene = headline_scene(args.slab_length_cells)
    n = scene["x"].shape[0]
    model, model_path = None, None
    if not args.no_warm_start:
        model_path = args.warm_start or default_warm_start()
        if model_path:
            from mpmsnow_b200.learned import WarmStartNet
            model = WarmStartNet(seed=0, device=f"cuda:{local}")
            model.load_state_dict(dict(np.load(model_path)))
    # plain arm (the reference's uniform initial guess), then the learned warm start on a fresh handle
    plain = time_arm(args, scene, local, pg, None, e2e=(model is None and not args.no_e2e))
    arm = plain
    bare = None
    if model is not None:
        arm = time_arm(args, scene, local, pg, model, e2e=not args.no_e2e)
        # the same guess without the network (p*/m and the history): the network's own share of the gain
        bare = time_arm(args, scene, local, pg, model, e2e=False, network=False)
    phases, clk, ms_max, ms_e2e = arm["phases"], arm["clocks"], arm["ms"], arm["ms_e2e"]

    # --- CPU baseline (rank 0, N = 1 only) ------------------------------------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cs = cpu_sample_scene(args.cpu_sample_cells)
        cn = cs["x"].shape[0]
        sec, cit = run_cpu_oracle(cs, args.cpu_steps, 0, threads)
        sec1, cit1 = run_cpu_oracle(cs, 1, 0, 1)
        cpu = {"value": cn / sec, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"FP32 oracle (the reference's step restated, 8-colour parallel splats, serial elsewhere), "
                         f"{cn}-particle section (length {args.cpu_sample_cells} cells) of the headline slab, "
                         f"{args.cpu_steps} steps from rest",
               "cr_iterations_per_step": cit,
               "value_1_thread": cn / sec1, "sample_1_thread": "the same section, its first step, one thread"}

    if rank != 0:
        return
    op = next(p for p in phases if p["name"] == "op_apply")
    op_launches = op["launches"]
    op_ms = op["ms"]
    achieved = (op["particles"] * OP_ALGORITHMIC_BYTES_PER_PARTICLE) / (op_ms * 1e-3) / 1e9 if op_ms > 0 else 0.0
    achieved_rec = (op["particles"] * OP_RECORD_BYTES_PER_PARTICLE) / (op_ms * 1e-3) / 1e9 if op_ms > 0 else 0.0
    peak, peak_kind = measured_hbm_peak()
    per_launch_particles = op["particles"] / max(op_launches, 1)
    traffic = (OP_TRAFFIC_PER_PARTICLE * per_launch_particles) if OP_TRAFFIC_PER_PARTICLE else None
    total_ms = sum(p["ms"] for p in phases)
    value = world * n * args.steps / (ms_max * 1e-3)
    plain_value = world * n * args.steps / (plain["ms"] * 1e-3)
    solver = "plain CR (the reference's uniform initial guess)"
    if model is not None:
        solver = (f"learned warm start ({os.path.basename(model_path)}: BF16 tcgen05 3-D conv network trained on "
                  f"slab sections by this project's kernels, on top of p*/m and the previous step's correction) + CR "
                  f"to the same residual")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": AVALANCHE_WORKLOAD if args.workload == "avalanche" else WORKLOAD, "particles": n,
                   "h": scene["h"],
                   "dt": scene["dt"], "cr_tol": SOLVE_TOL, "cr_max_iters": SOLVE_MAX_ITERS, "solver": solver,
                   "l2": f"inputs larger than L2 (particle state {n * 240 / 1e9:.1f} GB per replica)",
                   "parallelism": f"replicas x{world}",
                   "cr_iterations_per_step": sum(arm["iters"]) / len(arm["iters"])},
        "plain": {"value": plain_value, "ms_per_step": plain["ms"] / args.steps,
                  "cr_iterations_per_step": sum(plain["iters"]) / len(plain["iters"]),
                  "phases_ms_per_step": {p["name"]: round(p["ms"] / args.steps, 4) for p in plain["phases"]
                                         if p["launches"]}},
        "learned_vs_plain": value / plain_value if model is not None else None,
        "guess_without_network": None if bare is None else {
            "value": world * n * args.steps / (bare["ms"] * 1e-3), "ms_per_step": bare["ms"] / args.steps,
            "cr_iterations_per_step": sum(bare["iters"]) / len(bare["iters"]),
            "phases_ms_per_step": {p["name"]: round(p["ms"] / args.steps, 4) for p in bare["phases"] if p["launches"]}},
        "roofline": {"kernel": "k_op_apply (CR operator pass: gather 64 nodes -> linearised 9x9 force map -> "
                               "cell-run scatter)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if peak else None, "traffic": traffic,
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "bytes_per_particle": OP_ALGORITHMIC_BYTES_PER_PARTICLE,
                     "record_bytes_per_particle": OP_RECORD_BYTES_PER_PARTICLE, "achieved_at_record_bytes": achieved_rec,
                     "frac_at_record_bytes": achieved_rec / peak if peak else None,
                     "launches": op_launches, "particles_per_launch": per_launch_particles,
                     "avg_launch_ms": op_ms / max(op_launches, 1)},
        "cpu_baseline": cpu,
        "clocks": clk,
        "e2e": None if ms_e2e is None else {"value": world * n * args.steps / (ms_e2e * 1e-3), "unit": UNIT,
                                            "h2d_bytes_per_step": 24 * n, "d2h_bytes_per_step": 24 * n,
                                            "cr_iterations_per_step": sum(arm["iters_e2e"]) / len(arm["iters_e2e"])},
        "gpu_launches": arm["launches"],
        "phases_ms_per_step": {p["name"]: round(p["ms"] / args.steps, 4) for p in phases if p["launches"]},
        "phases_share": {p["name"]: round(p["ms"] / total_ms, 4) for p in phases if p["launches"] and total_ms > 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-cells", type=int, default=10)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--ref-sample-cells", type=int, default=4)
    ap.add_argument("--slab-length-cells", type=int, default=171,
                    help="profiling cases: a shorter slab with the headline cross-section (171 = the headline)")
    ap.add_argument("--workload", default="slab", choices=["slab", "avalanche"],
                    help="slab: the headline 4M slab; avalanche: the 16M avalanche with its cylinder (the plain, "
                         "learned and network-free arms as for the slab)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--warm-start", default=None, help="learned warm-start model (.npz); default: the packaged one")
    ap.add_argument("--no-warm-start", action="store_true", help="time the plain solver only")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local, pg = dist_setup()
    try:
        if args.impl == "reference":
            bench_reference(args, world, rank, pg)
        else:
            bench_b200(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
