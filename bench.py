#!/usr/bin/env python
"""Throughput of the DSMC timestep on B200: atom-steps/s at 1e7 atoms.

Workload: the full trapped step (1e7 Rb-87 atoms, linear quadrupole B' = 2.5 T/m, 50 uK,
128^3 cells over +-5 thermal radii, dt = 1e-6 s, NTC collisions, Larmor precession,
Majorana loss, energy knife 6 -> 4 kT over 1e5 steps), FP32 state with exact fixed-point
diagnostics.  One bench "step" = one DSMC timestep of the whole cloud.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--atoms N]

Under torchrun (N > 1) every rank simulates its own cloud (different seed): the clouds are
independent, so the GPUs share no data and the scaling is weak.  ``--impl reference`` times
the CPU restatement of the same step (the reference has no CPU code path; its CUDA kernels
target sm_30) on all host cores.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s @1e7 atoms"
UNIT = "atom-steps/s"
WORKLOAD = "trapped-quadrupole-1e7-atoms-128cubed-cells-fp32"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--atoms", type=int, default=10_000_000)
    ap.add_argument("--cpu-steps", type=int, default=10, help="timed steps of the CPU baseline sample")
    ap.add_argument("--cpu-warmup", type=int, default=2, help="untimed steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-steps", type=int, default=50)
    ap.add_argument("--batched", action="store_true",
                    help="time the 256-cloud batched ensemble instead, sharded over the ranks (torchrun)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-drift", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--fp64-steps", type=int, default=20)
    ap.add_argument("--drift-steps", type=int, default=200)
    ap.add_argument("--adjoint-steps", type=int, default=2000)
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def workload(atoms: int, source: str = "engine"):
    """Run and cloud parameters of the 1e7-atom trapped workload.  source="oracle" takes them from
    the CPU restatement's copy of the preset table, so that the reference arm never loads the
    engine library."""
    if source == "oracle":
        import oracle
        run, c = oracle.preset(2)
    else:
        from cudadsmc_b200 import preset
        run, c = preset(2)
    c.n_atoms = atoms
    c.capacity = atoms
    return run, c


def config_of(args, ws: int) -> dict:
    """The workload's config dict, printed identically by both arms."""
    return {"workload": WORKLOAD, "atoms_per_gpu": args.atoms, "cells": 128 ** 3,
            "trap": "quadrupole B'=2.5 T/m", "T_uK": 50, "dt": 1e-6,
            "physics": "NTC collide + Larmor + Verlet + Majorana + knife 6->4 kT",
            "l2": "inputs larger than L2 (48 B/atom x 1e7 = 480 MB per state buffer)",
            "parallelism": f"replicas{ws}" if ws > 1 else "single-gpu"}


def cpu_baseline(run, cloud, steps: int, threads: int | None = None, warmup: int = 2) -> dict:
    """The CPU restatement (OpenMP, float) timed on the host cores for a bounded sample."""
    import oracle
    if threads:
        oracle.set_threads(threads)
    nthreads = oracle.max_threads()
    o = oracle.Oracle(run, cloud, fast=True)
    o.init_cloud(run.seed)
    o.step(warmup)
    d0 = o.diagnostics()
    t0 = time.perf_counter()
    o.step(steps)
    t1 = time.perf_counter()
    d1 = o.diagnostics()
    atom_steps = d1["atom_steps"] - d0["atom_steps"]
    # the same restatement on one host thread, one more step of the same cloud
    oracle.set_threads(1)
    t2 = time.perf_counter()
    o.step(1)
    t3 = time.perf_counter()
    one = o.diagnostics()["atom_steps"] - d1["atom_steps"]
    oracle.set_threads(nthreads)
    return {"value": atom_steps / (t1 - t0), "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{cloud.n_atoms:.0e} atoms, {steps} timed steps after init + {warmup} warm-up steps "
                      f"({t1 - t0:.1f} s), OpenMP float build of oracle/dsmc_oracle.cpp",
            "single_thread": {"value": one / (t3 - t2), "unit": UNIT, "cores": 1,
                              "sample": f"1 further step of the same cloud on one thread ({t3 - t2:.1f} s)"}}


def adjoint_vs_plain(stream, steps: int, checkpoint_every: int) -> dict:
    """The adjoint workload (1e6 atoms, 0.1 mT bias, 30 uK, 8-segment knife ramp): device time of a
    plain forward run of `steps` steps against the pathwise-adjoint call on the same cloud (the
    recorded physical run + the smoothed forward + the checkpointed recomputation and adjoint), in
    FP32; the FP64 adjoint's gradient gives the FP32 drift."""
    import numpy as np
    import torch
    from cudadsmc_b200 import FP32, FP64, Simulation, preset
    run, c = preset(4)
    plain = Simulation(run, c)
    plain.set_stream(stream.cuda_stream)
    plain.init_cloud(4321)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    plain.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms_plain = e0.elapsed_time(e1)
    plain.close()
    grads = {}
    for prec, name in ((FP32, "fp32"), (FP64, "fp64")):
        s = Simulation(run, c)
        s.set_stream(stream.cuda_stream)
        s.init_cloud(4321)
        grads[name] = s.adjoint_run(steps, checkpoint_every=checkpoint_every, precision=prec, sigmoid_width_kT=0.2)
        s.close()
    g = grads["fp32"]
    vec = lambda d: np.array([d["dL_dBp"], d["dL_dB0"]] + list(d["dL_deta"]))
    g32, g64 = vec(grads["fp32"]), vec(grads["fp64"])
    scale = np.max(np.abs(g64))
    return {"atoms": c.n_atoms, "steps": steps, "checkpoint_every": checkpoint_every, "precision": "fp32",
            "ms_plain_forward": ms_plain, "ms_record": g["ms_record"], "ms_smoothed_forward": g["ms_forward"],
            "ms_adjoint": g["ms_backward"],
            "fwd_adjoint_over_plain": (g["ms_record"] + g["ms_forward"] + g["ms_backward"]) / ms_plain,
            "collisions_recorded": g["collisions"], "loss": g["loss"],
            "grad_fp32_vs_fp64_max_abs_over_max": float(np.max(np.abs(g32 - g64)) / scale) if scale > 0 else 0.0}


def fp32_drift(stream, atoms: int, steps: int) -> dict:
    """The measured workload in FP32 against an FP64 run of the same cloud: the FP64 initial state,
    rounded to FP32, advanced `steps` steps in both precisions (same seeds, same random numbers);
    the relative difference of every diagnostic."""
    import numpy as np
    from cudadsmc_b200 import FP64, Simulation
    run, c = workload(atoms)
    run64 = run.copy()
    run64.precision = FP64
    s64 = Simulation(run64, c)
    s64.set_stream(stream.cuda_stream)
    s64.init_cloud(run.seed)
    st = s64.get_state()

    def lanes32(a):
        out = a.astype(np.float32)
        out[:, 3] = a[:, 3].view(np.uint64).astype(np.uint32).view(np.float32)  # id / flag bits
        return out

    s32 = Simulation(run, c)
    s32.set_stream(stream.cuda_stream)
    s32.set_state(lanes32(st["pos"]), lanes32(st["vel"]), st["psi"].astype(np.float32), st["cloud_counts"])
    del st
    s64.step(steps)
    s32.step(steps)
    a, b = s32.diagnostics(), s64.diagnostics()
    keys = ("n_alive", "temperature", "e_kin", "e_pot", "e_evaporated", "n_evaporated", "n_majorana",
            "n_knife", "collisions", "candidates", "sum_v2", "sum_absB")
    rel = {k: (abs(a[k] - b[k]) / abs(b[k]) if b[k] else float(abs(a[k]))) for k in keys}
    s32.close()
    s64.close()
    return {"atoms": atoms, "steps": steps, "relative_drift": rel,
            "definition": "|FP32 - FP64| / |FP64| per diagnostic after the same steps from the same state"}


def fp64_throughput(stream, atoms: int, steps: int, warmup: int) -> dict:
    """The same workload with FP64 state and arithmetic (the reference's precision): device-timed
    atom-steps/s over `steps` steps after `warmup`, for a like-precision point beside the FP32 line."""
    import torch
    from cudadsmc_b200 import FP64, Simulation
    run, c = workload(atoms)
    run.precision = FP64
    s = Simulation(run, c)
    s.set_stream(stream.cuda_stream)
    s.init_cloud(run.seed)
    s.step(warmup)
    s.synchronize()
    d0 = s.diagnostics()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    d1 = s.diagnostics()
    s.set_profiling(True)
    s.step(3)
    kt = s.kernel_times()
    s.close()
    return {"value": (d1["atom_steps"] - d0["atom_steps"]) / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "warmup": warmup, "dtype": "f64",
            "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in kt.items()}}


def batched_vs_sequential(stream, steps: int) -> dict:
    """256 clouds stepped together in one handle vs the same clouds as 256 single-cloud handles
    run one after another on the same stream; per-cloud results are identical (checked)."""
    import torch
    from cudadsmc_b200 import Simulation
    from cudadsmc_b200.workloads import batched_ensemble
    run, clouds = batched_ensemble()
    batch = Simulation(run, clouds)
    batch.set_stream(stream.cuda_stream)
    batch.init_cloud(run.seed)
    tile, _ = batch.autotune(3)
    table = batch.autotune_table()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d0 = batch.diagnostics()
    e0.record(stream)
    batch.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms_batch = e0.elapsed_time(e1)
    d1 = batch.diagnostics()
    singles = []
    for c in clouds:
        s = Simulation(run, c)
        s.set_stream(stream.cuda_stream)
        s.init_cloud(run.seed)
        singles.append(s)
    # bring the single runs to the batch's step count before timing
    pre = d0["step"]
    for s in singles:
        s.step(pre)
    torch.cuda.synchronize()
    e0.record(stream)
    for s in singles:
        s.step(steps)
    e1.record(stream)
    e1.synchronize()
    ms_seq = e0.elapsed_time(e1)
    same = all(singles[k].diagnostics()["sum_v2"] == batch.diagnostics(k)["sum_v2"] and
               singles[k].diagnostics()["n_alive"] == batch.diagnostics(k)["n_alive"] for k in range(len(clouds)))
    for s in singles:
        s.close()
    atoms = d1["atom_steps"] - d0["atom_steps"]
    batch.close()
    return {"clouds": len(clouds), "atoms": int(sum(c.n_atoms for c in clouds)), "steps": steps,
            "tile_atoms": tile, "blocks_per_sm": table["chosen_blocks_per_sm"],
            "autotune": [{"tile_atoms": t, "blocks_per_sm": b, "ms_per_step": round(m, 5)}
                         for t, b, m in zip(table["tile_atoms"], table["blocks_per_sm"], table["ms_per_step"])],
            "batched_atom_steps_per_s": atoms / (ms_batch * 1e-3),
            "sequential_atom_steps_per_s": atoms / (ms_seq * 1e-3), "speedup": ms_seq / ms_batch,
            "ms_per_step_batched": ms_batch / steps, "ms_per_step_sequential": ms_seq / steps,
            "identical_per_cloud_results": bool(same)}


def run_batched_sharded(args):
    """`--batched`: the 256-cloud batched ensemble, its clouds sharded over the ranks (each rank one
    batched handle holding its shard), per-cloud diagnostics gathered with one NCCL all-reduce after
    the timed steps; rank 0 checks them against the whole batch run on its own GPU."""
    import torch
    import torch.distributed as dist
    from cudadsmc_b200 import Simulation
    from cudadsmc_b200.replicas import GATHERED_FIELDS, run_sharded_batch
    from cudadsmc_b200.workloads import batched_ensemble
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    run, clouds = batched_ensemble()

    def make_sim(r, cl):
        s = Simulation(r, cl)
        s.set_stream(stream.cuda_stream)
        return s

    def timer(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    if ws > 1:
        dist.barrier()
    ms, atom_steps, table = run_sharded_batch(make_sim, run, clouds, args.batched_steps, run.seed, timer)
    same = None
    if rank == 0:
        if ws > 1:
            s = make_sim(run, clouds)
            s.init_cloud(run.seed)
            s.step(args.batched_steps)
            s.synchronize()
            same = all(float(s.diagnostics(k)[f]) == table[k][f] for k in range(len(clouds)) for f in GATHERED_FIELDS)
            s.close()
        line = {"metric": "atom-steps/s, 256-cloud batched ensemble", "value": atom_steps / (ms * 1e-3), "unit": UNIT,
                "n_gpus": ws, "steps": args.batched_steps, "warmup": 0, "ms_per_step": ms / args.batched_steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded Philox clouds, no dataset)",
                "config": {"workload": "batched-256-clouds", "clouds": len(clouds),
                           "atoms": int(sum(c.n_atoms for c in clouds)),
                           "parallelism": f"clouds sharded over {ws} ranks" if ws > 1 else "single-gpu"},
                "identical_to_single_gpu_batch": same}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    run, c = workload(args.atoms, source="oracle")
    # the whole --steps K --warmup W run on the host cores (about 0.4 s per step at 1e7 atoms on 16
    # threads), each step the full workload
    res = cpu_baseline(run, c, steps=max(1, args.steps), warmup=args.warmup)
    line = {"impl": "reference", "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": max(1, args.steps), "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Philox thermal cloud, no dataset)",
            "config": config_of(args, ws),
            "cpu_baseline": res,
            "e2e": {"value": res["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.batched:
        return run_batched_sharded(args)
    import numpy as np
    import torch
    import torch.distributed as dist
    from cudadsmc_b200 import Simulation

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    run, c = workload(args.atoms)
    sim = Simulation(run, c)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    sim.init_cloud(run.seed + 7919 * rank)

    # ------------------------------------------------------------------ device-resident timing
    sim.step(args.warmup)
    sim.synchronize()
    d0 = sim.diagnostics()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(args.steps)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    d1 = sim.diagnostics()
    atom_steps = d1["atom_steps"] - d0["atom_steps"]
    if ws > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        a = torch.tensor([atom_steps], device="cuda", dtype=torch.float64)
        dist.all_reduce(a)
        atom_steps = int(a.item())
    value = atom_steps / (ms * 1e-3)

    # ------------------------------------------------------------------ per-kernel times (events)
    sim.set_profiling(True)
    sim.step(5)
    kt = sim.kernel_times()
    sim.set_profiling(False)
    n_now = sim.diagnostics()["n_alive"]
    step_ms = kt["step_pass"][0] / kt["step_pass"][1]
    perm_ms = kt["permute_pass"][0] / kt["permute_pass"][1]
    # step_pass: gather pos, vel, psi (48 B) through src (4 B), write them back (48 B) with an
    # 8-byte sort key; permute_pass: read the key (8 B), write the next permutation (4 B)
    bytes_atom_step = 48 + 4 + 48 + 8
    bytes_atom_perm = 8 + 4
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak = float(json.load(f)["hbm_gbs"])
        peak_src = "measured"
    achieved = bytes_atom_step * n_now / (step_ms * 1e-3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "step_pass_traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            traffic = float(json.load(f)["dram_bytes_per_atom"]) * n_now
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "step_pass", "peak_source": peak_src,
                "algorithmic_bytes_per_atom": bytes_atom_step,
                "kernels_ms": {k: v[0] / max(v[1], 1) for k, v in kt.items()},
                "permute_pass_frac": bytes_atom_perm * n_now / (perm_ms * 1e-3) / 1e9 / peak}

    # ------------------------------------------------------------------ end to end, host buffers
    e2e = None
    if not args.no_e2e:
        st = sim.get_state()
        pin = {k: torch.from_numpy(np.ascontiguousarray(st[k])).pin_memory() for k in ("pos", "vel", "psi")}
        counts = st["cloud_counts"]
        sim2 = Simulation(run, c)
        sim2.set_stream(stream.cuda_stream)
        sim2.set_state(pin["pos"].numpy(), pin["vel"].numpy(), pin["psi"].numpy(), counts)
        sim2.step(args.warmup)
        sim2.synchronize()
        out = {k: torch.empty((c.capacity, 4), dtype=v.dtype).pin_memory() for k, v in pin.items()}
        out_np = {k: v.numpy() for k, v in out.items()}
        sim2.reserve_diagnostics(args.steps)  # pinned slots: one diagnostics read-back per step
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ee0 = torch.cuda.Event(enable_timing=True)
        ee0.record(stream)
        sim2.set_state(pin["pos"].numpy(), pin["vel"].numpy(), pin["psi"].numpy(), counts)
        a0 = sim2.diagnostics()["atom_steps"]
        for k in range(args.steps):
            sim2.step(1)
            sim2.diagnostics_enqueue(k)  # the step's totals copied to the host, without a wait
        st2 = sim2.get_state(out=out_np)
        per_step = [sim2.diagnostics_collect(k) for k in range(args.steps)]
        dd = per_step[-1]
        diag_bytes = sim2.diagnostics_copy_bytes()
        ee1 = torch.cuda.Event(enable_timing=True)
        ee1.record(stream)
        ee1.synchronize()
        wall = time.perf_counter() - t0
        e_ms = ee0.elapsed_time(ee1)
        a_steps = dd["atom_steps"] - a0
        if ws > 1:
            t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
            a = torch.tensor([a_steps], device="cuda", dtype=torch.float64)
            dist.all_reduce(a)
            a_steps = int(a.item())
        state_bytes = sum(v.numel() * v.element_size() for v in pin.values())
        out_bytes = sum(st2[k].nbytes for k in ("pos", "vel", "psi"))
        e2e = {"value": a_steps / (e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": state_bytes / args.steps,
               "d2h_bytes_per_step": out_bytes / args.steps + diag_bytes,
               "K": args.steps,
               "definition": "dsmc_set_state from pinned host buffers, K x (dsmc_step(1) + the step's "
                             "diagnostics copied to pinned host memory with dsmc_diagnostics_enqueue), "
                             "dsmc_get_state to host, the K diagnostics collected; all inside the timed "
                             "region (K = --steps)",
               "wall_s": wall}
        sim2.close()

    # ------------------------------------------------------------------ batched vs sequential
    batched = None
    if rank == 0 and ws == 1 and not args.no_batched:
        batched = batched_vs_sequential(stream, steps=args.batched_steps)

    # ------------------------------------------------------------------ FP32 against FP64
    drift = None
    if rank == 0 and ws == 1 and not args.no_drift:
        drift = fp32_drift(stream, args.atoms, args.drift_steps)

    # ------------------------------------------------------------------ FP64 throughput
    fp64 = None
    if rank == 0 and ws == 1 and not args.no_fp64:
        fp64 = fp64_throughput(stream, args.atoms, args.fp64_steps, args.warmup)

    # ------------------------------------------------------------------ forward + adjoint vs plain
    adjoint = None
    if rank == 0 and ws == 1 and not args.no_adjoint:
        adjoint = adjoint_vs_plain(stream, steps=args.adjoint_steps, checkpoint_every=100)

    # ------------------------------------------------------------------ CPU baseline
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(run, c, steps=args.cpu_steps, warmup=args.cpu_warmup)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded Philox thermal cloud, no dataset)",
                "config": config_of(args, ws),
                "clocks": clk, "gpu_launches": args.steps * sim.launches_per_step(),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "batched": batched, "adjoint": adjoint, "fp32_drift": drift, "fp64": fp64,
                "n_alive_end": d1["n_alive"]}
        print(json.dumps(line), flush=True)
    sim.close()
    if ws > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
