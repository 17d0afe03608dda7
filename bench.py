#!/usr/bin/env python
"""Benchmark of the SAP contact step on one node.

Workload (BASELINE metric, config "batched uniform"): 4096 worlds of a 35-DOF
floating-base humanoid (6 + 29 revolute, serial-chain tree), 8-32 contacts per
world, phi0 ~ U[-2e-3, 0], mu ~ U[0.3, 1], v* ~ N(0, 0.5); seeded synthetic
inputs (no dataset exists for this path).  A step is one SAP stage-2 solve of
all worlds (prepare + Newton + armijo_decay line search to the reference's
tolerances) from the cold start v0, so every step does the full work.

`value` is world-steps/s of the fast path (FP32 Hessian/factorization, FP64
gradient/cost/line search/convergence) with inputs resident in HBM; the plain
FP64 solve is reported beside it.  `e2e` is the same metric through the
public API with host inputs: pinned host -> device copy of the step's inputs
and a device -> host read of the solved velocities inside the timed region.

Multi-GPU (torchrun): worlds are independent, so each rank solves its own
4096 worlds (weak scaling, no data-path collective); the barrier and the
max-over-ranks reduction of the timings are the only collectives.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one solve
# launch on this workload, measured once with ncu.
NCU_TRAFFIC_BYTES = 117.821440e6 + 5.310464e6

METRIC = "world-steps/s, 4096 humanoids: learned+FP32 vs plain FP64, same B200, same tol"
WORLDS = 4096
SEED = 2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--worlds", type=int, default=WORLDS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def algorithmic_bytes(prob) -> int:
    """Compulsory FP64 I/O of the contact solve, world by world with the actual
    contact count: 8*[3*C*n + n^2 + 2n + 5C] (A, J, v*, v0, contact params)
    plus 8*[n + 3C] (v and gamma written)."""
    n = prob.dof_per_env
    C = np.clip(prob.contact_count.astype(np.int64), 0, prob.max_contacts)
    per_world = 8 * (3 * C * n + n * n + 2 * n + 5 * C) + 8 * (n + 3 * C)
    return int(per_world.sum())


class ClockSampler:
    """nvidia-smi clock / throttle sampling around the timed region.

    Samples stream to a file every 50 ms from before the warm-up until the
    timed region has ended; samples stamped inside the region are used (the
    nearest ones if the region is shorter than the sampling period)."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        import tempfile

        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(prefix="sapb_clocks_", suffix=".csv")
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        deadline = time.time() + 5.0  # wait for the first sample
        while time.time() < deadline:
            if os.path.exists(self.path) and os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def mark_begin(self):
        self.t0 = time.time()

    def mark_end(self):
        self.t1 = time.time()
        time.sleep(0.12)  # let a sample land after the region

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        try:
            lines = open(self.path).read().splitlines()
            os.unlink(self.path)
        except OSError:
            lines = []
        from datetime import datetime

        for line in lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                ts = datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[1]), float(parts[2]), parts[4:8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        inside = [r for r in rows if self.t0 is not None and self.t0 <= r[0] <= self.t1]
        if not inside and self.t0 is not None:
            mid = 0.5 * (self.t0 + self.t1)
            inside = sorted(rows, key=lambda r: abs(r[0] - mid))[:2]
        reasons = sorted({n for r in inside for n, v in zip(self.NAMES, r[3]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[1] for r in inside])), "sm_max_mhz": max(r[2] for r in inside),
                "reasons": reasons, "samples": len(inside)}


def oracle_time(prob, steps: int, threads: int, min_seconds: float = 0.0):
    """Seconds per full-batch oracle solve (armijo_decay, FP64)."""
    from oracle import oracle

    oracle.solve(prob.subset(np.arange(min(prob.num_envs, 64))), "armijo_decay", threads=threads)  # warm
    times = []
    t_start = time.perf_counter()
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        oracle.solve(prob, "armijo_decay", threads=threads)
        times.append(time.perf_counter() - t0)
        if min_seconds and time.perf_counter() - t_start > min_seconds:
            break
    return float(np.mean(times)), len(times)


def run_reference(args, rank: int, world_size: int):
    """Reference arm: the reference's own implementation is Python + NVIDIA
    Warp, which cannot be installed here, so the CPU restatement of its
    algorithm (oracle/, FP64, OpenMP over worlds) is timed on all host cores."""
    if rank != 0:
        return
    from sap_warp_b200 import scenes

    prob = scenes.humanoid_contact_problem(args.worlds, seed=SEED)
    cores = os.cpu_count() or 1
    for _ in range(max(0, args.warmup)):
        oracle_time(prob.subset(np.arange(min(256, prob.num_envs))), 1, cores)
    sec, k = oracle_time(prob, args.steps, cores, min_seconds=60.0)
    value = prob.num_envs / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "world-steps/s", "n_gpus": args.gpus,
        "steps": k, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, shapes of the batched-uniform config)",
        "config": {"workload": f"{prob.num_envs} humanoid worlds x 35 DOF, 8-32 contacts, armijo_decay, FP64",
                   "worlds": prob.num_envs, "dof_per_env": prob.dof_per_env, "max_contacts": prob.max_contacts},
        "cpu_baseline": {"value": value, "unit": "world-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{k} full {prob.num_envs}-world solves"},
        "e2e": {"value": value, "unit": "world-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference (Python + NVIDIA Warp) is not installable offline; the FP64 CPU restatement of its "
                "algorithm is timed instead",
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world_size)
        return

    import torch

    from sap_warp_b200 import scenes
    from sap_warp_b200._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world_size > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    prob = scenes.humanoid_contact_problem(args.worlds, seed=SEED + 1000 * rank)
    t = problem_to_device(prob, dev)
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
    opt_fast = make_options("armijo_decay", hessian_precision="fp32", linear_solve_precision="fp32")
    opt_fp64 = make_options("armijo_decay")
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        tt = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    def timed(opts, steps, warmup, sampler=None):
        for _ in range(warmup):
            contact_solve(**t, buffers=buf, options=opts)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.mark_begin()
        ev0.record(stream)
        for _ in range(steps):
            contact_solve(**t, buffers=buf, options=opts)
        ev1.record(stream)
        barrier()
        if sampler:
            sampler.mark_end()
        return max_over_ranks(ev0.elapsed_time(ev1) / steps)

    # plain FP64 solve
    ms_fp64 = timed(opt_fp64, args.steps, args.warmup)
    it_fp64 = float(buf.newton_iterations.double().mean())
    conv_fp64 = bool(buf.converged.all())
    v_fp64 = buf.v.clone()
    # fast path (the headline)
    sampler = ClockSampler(local_rank)
    sampler.start()
    ms_fast = timed(opt_fast, args.steps, args.warmup, sampler)
    clocks = sampler.stop()
    it_fast = float(buf.newton_iterations.double().mean())
    conv_fast = bool(buf.converged.all())
    rel = float(((buf.v - v_fp64).abs().view(-1, prob.dof_per_env).amax(1) /
                 v_fp64.abs().view(-1, prob.dof_per_env).amax(1)).max())

    # end to end through the public API with host buffers
    host = {k: v.cpu().pin_memory() for k, v in t.items()}
    dev_in = {k: torch.empty_like(v) for k, v in t.items()}
    v_host = torch.empty(buf.v.shape, dtype=buf.v.dtype).pin_memory()
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    d2h = v_host.numel() * v_host.element_size()

    def e2e_step():
        for k, v in host.items():
            dev_in[k].copy_(v, non_blocking=True)
        contact_solve(**dev_in, buffers=buf, options=opt_fast)
        v_host.copy_(buf.v, non_blocking=True)

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / args.steps)

    alg = algorithmic_bytes(prob)
    total_worlds = prob.num_envs * world_size
    value = total_worlds / (ms_fast * 1e-3)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved = alg / (ms_fast * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "world-steps/s", "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_fast, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (FP32 Hessian/factor)", "data": "synthetic (seeded)",
        "config": {"workload": f"{prob.num_envs} humanoid worlds x 35 DOF (6+29 revolute), 8-32 contacts, "
                               "armijo_decay to reference tolerances, cold start v0",
                   "worlds_per_gpu": prob.num_envs, "dof_per_env": prob.dof_per_env,
                   "max_contacts": prob.max_contacts, "parallelism": f"world shards x{world_size}",
                   "l2": "inputs (A+J = %.0f MB) larger than L2" % (alg / 1e6)},
        "plain_fp64": {"value": total_worlds / (ms_fp64 * 1e-3), "ms_per_step": ms_fp64,
                       "mean_newton_iterations": it_fp64, "all_converged": conv_fp64},
        "fast": {"mean_newton_iterations": it_fast, "all_converged": conv_fast,
                 "max_rel_v_diff_vs_fp64": rel, "speedup_vs_fp64": ms_fp64 / ms_fast},
        "e2e": {"value": total_worlds / (ms_e2e * 1e-3), "unit": "world-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak,
                     "traffic": NCU_TRAFFIC_BYTES if args.worlds == WORLDS else None,
                     "note": "kernel is FP64/FP32-pipe bound, not HBM bound; achieved = algorithmic bytes / "
                             "kernel time (of measured peak)"},
        "gpu_launches": args.steps,
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        sample = prob.subset(np.arange(min(1024, prob.num_envs)))
        sec, k = oracle_time(sample, 200, cores, min_seconds=10.0)
        line["cpu_baseline"] = {"value": sample.num_envs / sec, "unit": "world-steps/s", "cores": cores,
                                "kind": "port", "sample": f"{k} solves of {sample.num_envs} worlds"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
