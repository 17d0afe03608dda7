#!/usr/bin/env python
"""Benchmark of the SAP contact step on one node.

Workload (batched uniform humanoids): 4096 worlds of a 35-DOF floating-base
humanoid (6 + 29 revolute, serial-chain tree), 8-32 body-vs-ground point
contacts per world on the distal links, phi0 ~ U[-2e-3, 0] m at the start,
mu ~ U[0.3, 1], pair stiffness 1e5 N/m, dissipation time 0.01 s, joint
velocities ~ N(0, 0.5), dt = 2 ms; seeded synthetic inputs (no dataset exists
for this path).  A step is one full SolverSAP.step of all worlds -- free
motion, contact Jacobian, the stage-2 Newton solve with armijo_decay to the
reference's tolerances (optimality 1e-14 abs / 1e-6 rel), position
integration -- and the timed steps continue one rollout.

The timed window starts after a fixed settling prefix of SETTLE_STEPS steps
(plain FP64 solver, untimed), so a short run measures the steady rollout
rather than its easy first steps; every arm starts from the same settled
state.

Arms (same scene, same trajectory up to the solve tolerance):
  value        learned + FP32: FP32 Hessian / factorization with FP64
               gradient, cost, line search and convergence test, and the
               learned warm start (each contact's start impulse: the
               quadratic extrapolation of its last three solves' impulses
               where it has that history, the network's prediction where it
               is new; tried against the previous velocity);
  plain_fp64   the reference's method: FP64 throughout, warm start from the
               previous step's velocity;
  previous_impulses_fp32   the ablation without the network;
  carried_impulses_fp32    the ablation without the network and without
               extrapolation (the last solve's impulses as they were).
`e2e` is the headline arm through the public API with host buffers: the
step's inputs (state and contacts) copied from pinned host memory and the new
state read back inside the timed region.  `stage2_solve_only` is the contact
solve alone on the stage-2 snapshot of the same configuration (A, J given).

Multi-GPU (torchrun): worlds are independent, so each rank steps its own 4096
worlds (weak scaling, no data-path collective); the barrier and the
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

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one contact
# solve launch of the headline arm on this workload (4096 humanoids, learned
# start, FP32 Hessian; the fifth step after the 100-step settling prefix),
# from one ncu capture: 159.75 MB read + 6.61 MB written.
NCU_SOLVE_TRAFFIC_BYTES = 166_363_136

METRIC = "world-steps/s, 4096 humanoids: learned+FP32 vs plain FP64, same B200, same tol"
WORLDS = 4096
SEED = 2
DT = 2.0e-3
MAX_CONTACTS = 32
SETTLE_STEPS = 100


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--worlds", type=int, default=WORLDS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--weights", default=None, help="warm-start network weights (default: packaged)")
    return ap.parse_args()


def solve_bytes_per_world(n: int, counts: np.ndarray, velocities: int = 0, impulse_sets: int = 0,
                          factor: bool = False) -> np.ndarray:
    """Compulsory FP64 I/O of the contact solve per world with the actual
    contact count C: reads A (n^2), J (3Cn), v*, v0, v_guess (3n), 5 contact
    parameters (5C); writes v, v_guess (2n), gamma (3C), mode (C/2 words);
    plus for candidate starts the start or base velocities (n each), the
    impulse sets (3C each) and the factor (n^2) where it is read."""
    C = counts.astype(np.int64)
    b = 8 * (n * n + 3 * C * n + 3 * n + 5 * C) + 8 * (2 * n + 3 * C) + 4 * C
    return b + 8 * (velocities * n + impulse_sets * 3 * C + (n * n if factor else 0))


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


# ---- CPU pipeline of the step (oracle restatement), for the baselines ---------
def cpu_scene(worlds: int, seed: int):
    """The rollout scene built on the host: same distributions as
    models.rollout_scene, body poses from the C restatement."""
    from oracle import oracle
    from sap_warp_b200 import models

    rng = np.random.default_rng(seed)
    tpl = models.world_template("humanoid", rng)
    g = models.replicate(tpl, worlds, rng, mu_range=(0.3, 1.0), stiffness=1.0e5, tau_d=0.005)
    q = models.random_joint_q(tpl, rng, worlds)
    n, B = tpl["dofs_per_world"], tpl["bodies_per_world"]
    qd = rng.normal(scale=0.5, size=(worlds, n))
    hm = oracle.HostModel(tpl, g)
    empty = dict(count=np.zeros(1, np.int32), shape0=np.zeros(1, np.int32), shape1=np.zeros(1, np.int32),
                 point0=np.zeros((1, 3)), point1=np.zeros((1, 3)), normal=np.zeros((1, 3)), margin0=np.zeros(1),
                 margin1=np.zeros(1))
    bq = oracle.free_motion_contacts(hm, q, qd, empty, np.full(worlds, DT), 1)["body_q"].reshape(worlds, B, 7)
    counts = rng.integers(8, 33, size=worlds)
    con = models.ground_contacts(rng, bq[..., :3], bq[..., 3:], counts, bodies_from=B // 2,
                                 capacity=int(counts.sum()))
    return dict(tpl=tpl, hm=hm, q=q, qd=qd, con=con)


def cpu_steps(scene: dict, steps: int, threads: int, min_seconds: float = 0.0):
    """Seconds per world-step of the CPU pipeline -- the C restatements of
    the free motion and contact rows and of the solve (OpenMP over worlds) and
    of the integration -- drake preset, FP64, previous-velocity warm start."""
    from oracle import oracle
    from sap_warp_b200 import scenes

    hm, tpl = scene["hm"], scene["tpl"]
    q, qd = scene["q"].copy(), scene["qd"].copy()
    W, n, B = q.shape[0], tpl["dofs_per_world"], tpl["bodies_per_world"]
    dt = np.full(W, DT)
    done, t0 = 0, time.perf_counter()
    for k in range(max(1, steps)):
        r = oracle.free_motion_contacts(hm, q, qd, scene["con"], dt, MAX_CONTACTS, point_mode="contact_midpoint",
                                        weight_mode="diag_delassus", threads=threads)
        prob = scenes.ContactProblemArrays(
            num_envs=W, dof_per_env=n, max_contacts=MAX_CONTACTS, bodies_per_env=B,
            contact_count=np.minimum(r["count"], MAX_CONTACTS).astype(np.int32), dynamics_matrix=r["A"],
            jacobian=r["jac"], phi0=r["phi0"], w_eff=r["w"], mu=r["mu"], stiffness=r["k"], tau_d=r["tau"],
            body0=r["body0"], body1=r["body1"], body_dof_start=np.zeros(W * B, np.int32),
            body_dof_count=np.full(W * B, n, np.int32), v_star=r["v_star"].reshape(-1), v0=qd.reshape(-1), dt=dt)
        sol = oracle.solve(prob, "armijo_decay", threads=threads, v_guess=qd.reshape(-1), v_guess_active=k > 0)
        v = sol["v"].reshape(W, n)
        q = oracle.integrate_positions(hm, q.reshape(-1), qd.reshape(-1), v.reshape(-1), dt,
                                       "sap_euler").reshape(W, -1)
        qd = v
        done += 1
        if min_seconds and time.perf_counter() - t0 > min_seconds:
            break
    return (time.perf_counter() - t0) / done, done


def oracle_errors(dev) -> dict:
    """Error of the GPU solve against the FP64 oracle per configuration, on
    samples the oracle finishes in seconds: the stage-2 solve (armijo_decay,
    the reference's tolerances) of the same seeded problem on the GPU in FP64
    and with the FP32 Hessian / factorization, and in the oracle (FP64).
    Per world: max |v - v_oracle| / max |v_oracle|; reported as the max and
    the 99th percentile over the sample.  Part of the CPU-baseline leg (the
    oracle runs on the host)."""
    import torch

    from oracle import oracle
    from sap_warp_b200 import scenes
    from sap_warp_b200._solve import (ContactSolveBuffers, blocked_contact_solve, blocked_problem_to_device,
                                      contact_solve, make_options, problem_to_device)

    def rel(vg, vo, n):
        vg, vo = vg.reshape(-1, n), vo.reshape(-1, n)
        e = np.abs(vg - vo).max(1) / np.maximum(np.abs(vo).max(1), 1e-300)
        return {"max": float(e.max()), "p99": float(np.quantile(e, 0.99)), "worlds": int(e.size)}

    out = {}
    cases = (("humanoid_35dof", scenes.humanoid_contact_problem(256, seed=SEED + 17), None),
             ("quadruped_18dof", scenes.quadruped_contact_problem(256, seed=SEED + 18), None))
    mix, _ = scenes.mixed_contact_problem(384, seed=SEED + 19)
    cases = cases + (("uneven_13_18_35dof", mix, scenes.work_order(mix)),)
    for name, prob, order in cases:
        ref = oracle.solve(prob, "armijo_decay")
        t = problem_to_device(prob, dev)
        wo = None if order is None else torch.as_tensor(order, dtype=torch.int32, device=dev)
        row = {}
        for prec in ("fp64", "fp32"):
            buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
            contact_solve(**t, buffers=buf, options=make_options("armijo_decay", hessian_precision=prec,
                                                                 linear_solve_precision=prec), world_order=wo)
            torch.cuda.synchronize()
            row[prec] = rel(buf.v.cpu().numpy(), ref["v"], prob.dof_per_env)
        out[name] = row
    boxes = scenes.box_stack_problem(2, seed=SEED + 20)
    ref = oracle.solve(boxes.to_dense(), "armijo_decay")
    tb = blocked_problem_to_device(boxes, dev)
    row = {}
    for prec in ("fp64", "fp32"):
        buf = ContactSolveBuffers(boxes.num_envs, boxes.dof_per_env, boxes.max_contacts, dev)
        blocked_contact_solve(buffers=buf, options=make_options("armijo_decay", hessian_precision=prec,
                                                                linear_solve_precision=prec), trees_per_env=64, **tb)
        torch.cuda.synchronize()
        row[prec] = rel(buf.v.cpu().numpy(), ref["v"], boxes.dof_per_env)
    out["boxes_384dof"] = row
    # worlds of an arm gripping one of 8 boxes, whole-step free motion and
    # rows on the GPU in the tree-blocked layout (trees of 7 and 6 DOFs) ->
    # the blocked solve, against the oracle's free motion, rows and dense
    # solve of the same step
    from sap_warp_b200 import models
    from sap_warp_b200.runtime import SapState
    from sap_warp_b200.solver import SolverSAP

    W, C = 64, 112
    model, state, control, con, host, hv = models.box_scene(W, SEED + 21, dev, boxes=8, sites=(3, 5), arm=True)
    hm = oracle.HostModel(hv["tpl"], hv["g"])
    dt = np.full(W, DT)
    r = oracle.free_motion_contacts(hm, hv["q"], hv["qd"], host, dt, C, point_mode="contact_midpoint",
                                    weight_mode="diag_delassus")
    tds = np.concatenate([[0], 7 + 6 * np.arange(9)]).astype(np.int32)
    bstart = np.concatenate([np.zeros(7, np.int32), tds[1:-1]])
    bcount = np.concatenate([np.full(7, 7, np.int32), np.full(8, 6, np.int32)])
    prob = scenes.ContactProblemArrays(
        num_envs=W, dof_per_env=55, max_contacts=C, bodies_per_env=15,
        contact_count=np.minimum(r["count"], C).astype(np.int32), dynamics_matrix=r["A"], jacobian=r["jac"],
        phi0=r["phi0"], w_eff=r["w"], mu=r["mu"], stiffness=r["k"], tau_d=r["tau"], body0=r["body0"],
        body1=r["body1"], body_dof_start=np.tile(bstart, W), body_dof_count=np.tile(bcount, W),
        v_star=r["v_star"].reshape(-1), v0=hv["qd"].reshape(-1), dt=dt)
    ref = oracle.solve(prob, "armijo_decay")
    row = {}
    for prec in ("fp64", "fp32"):
        solver = SolverSAP(model, max_rigid_contact=C, contact_preset_variant="drake", contact_tau_d=0.0,
                           tree_blocked=True, hessian_precision=prec)
        out_state = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(),
                             body_q=state.body_q.clone(), body_f=state.body_f.clone())
        solver.step(state, out_state, control, con, DT)
        torch.cuda.synchronize()
        row[prec] = rel(solver.last_contact_solve_result.v_flat.cpu().numpy(), ref["v"], 55)
    out["arm_8_boxes_55dof_tree_blocked"] = row
    return out


def run_reference(args, rank: int, world_size: int):
    """Reference arm: the reference's own implementation is Python + NVIDIA
    Warp, which cannot be installed here, so the CPU restatement of its step
    (oracle/, FP64, OpenMP over worlds in the solve) is timed on the host."""
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    sample_worlds = 1024
    scene = cpu_scene(sample_worlds, SEED)
    cpu_steps(scene, max(1, min(args.warmup, 2)), cores)
    sec, k = cpu_steps(scene, max(args.steps, 1), cores, min_seconds=60.0)
    value = sample_worlds / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "world-steps/s", "n_gpus": args.gpus,
        "steps": k, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, shapes of the batched-uniform config)",
        "config": {"workload": f"humanoid rollout, 35 DOF, 8-32 contacts, full SAP step, armijo_decay, FP64, "
                               f"sampled on {sample_worlds} worlds", "worlds": sample_worlds},
        "cpu_baseline": {"value": value, "unit": "world-steps/s", "cores": cores, "kind": "port",
                         "sample": f"{k} steps of a {sample_worlds}-world rollout"},
        "e2e": {"value": value, "unit": "world-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference (Python + NVIDIA Warp) is not installable offline; the FP64 C restatement of its "
                "step (OpenMP over worlds) is timed instead",
    }
    print(json.dumps(line), flush=True)


def main():
    from sap_warp_b200.shards import RankGroup, env_ranks, shard_of

    args = parse()
    rank, world_size, local_rank = env_ranks()
    if args.impl == "reference":
        run_reference(args, rank, world_size)
        return

    import torch

    from sap_warp_b200 import models, scenes
    from sap_warp_b200._solve import (ContactSolveBuffers, blocked_contact_solve, blocked_problem_to_device,
                                      contact_solve, make_options, problem_to_device)
    from sap_warp_b200.runtime import SapState
    from sap_warp_b200.solver import SolverSAP
    from sap_warp_b200.warmstart import DEFAULT_WEIGHTS, LearnedWarmStart

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world_size > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    stream = torch.cuda.current_stream(dev)
    group = RankGroup(dist, dev)
    barrier, max_over_ranks = group.barrier, group.max_over_ranks
    shard = shard_of(rank, world_size, args.worlds, SEED)

    model, state_init, control, contacts, _ = models.rollout_scene("humanoid", shard.worlds, shard.seed, dev)
    W = args.worlds
    ws = LearnedWarmStart.load(args.weights or DEFAULT_WEIGHTS, dev)
    # settle: SETTLE_STEPS untimed steps of the plain FP64 solver; every arm
    # starts its warm-up and timed window from the settled state
    settler = SolverSAP(model, max_rigid_contact=MAX_CONTACTS, contact_preset_variant="drake", hessian_precision="fp64")
    s_a = SapState(joint_q=state_init.joint_q.clone(), joint_qd=state_init.joint_qd.clone(),
                   body_q=state_init.body_q.clone(), body_f=state_init.body_f.clone())
    s_b = SapState(joint_q=state_init.joint_q.clone(), joint_qd=state_init.joint_qd.clone(),
                   body_q=state_init.body_q.clone(), body_f=state_init.body_f.clone())
    for _ in range(SETTLE_STEPS):
        settler.step(s_a, s_b, control, contacts, DT)
        s_a, s_b = s_b, s_a
    state0 = s_a
    del settler, s_b

    def fresh_states():
        a = SapState(joint_q=state0.joint_q.clone(), joint_qd=state0.joint_qd.clone(), body_q=state0.body_q.clone(),
                     body_f=state0.body_f.clone())
        b = SapState(joint_q=state0.joint_q.clone(), joint_qd=state0.joint_qd.clone(), body_q=state0.body_q.clone(),
                     body_f=state0.body_f.clone())
        return a, b

    def make_solver(prec, warm, history=3):
        return SolverSAP(model, max_rigid_contact=MAX_CONTACTS, contact_preset_variant="drake",
                         hessian_precision=prec, warm_start=warm, learned_warm_start=ws if warm == "learned" else None,
                         impulse_history=history, autotune=True)

    def run_arm(prec, warm, sampler=None, history=3):
        """Two passes over the same stretch of the rollout (steps warmup ..
        warmup + steps of the same trajectory): eager steps with per-stage
        events and per-step statistics (iterations, chosen starts), then,
        from the initial state again, the timed steps as replays of a CUDA
        graph of two whole steps."""
        pairs = max(args.steps // 2, 1)
        warm_pairs = max((args.warmup + 1) // 2, 1)
        solver = make_solver(prec, warm, history)
        s_in, s_out = fresh_states()
        for _ in range(2 * warm_pairs):
            solver.step(s_in, s_out, control, contacts, DT)
            s_in, s_out = s_out, s_in
        barrier()
        solver.stage_events = []
        iters, chosen, flops = [], [], []
        nd = 35.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(2 * pairs):
            solver.step(s_in, s_out, control, contacts, DT)
            cs = solver.contact_solve
            k = cs.newton_iterations_env.double()
            iters.append(k.sum())
            chosen.append(torch.bincount(cs.warm_start_accepted_env.long(), minlength=3))
            # algorithmic FP64-equivalent arithmetic of this step's solve (see roofline.fp64)
            Cw = solver.contact_jacobian.contact_env_count.clamp(0, MAX_CONTACTS).double()
            t = cs.ls_iterations_total.double()
            flops.append((k * (6 * Cw * nd * nd + nd ** 3 / 3 + 2 * nd * nd + 6 * Cw * nd)
                          + (k + 1) * (4 * nd * nd + 12 * Cw * nd) + 80 * Cw * t).sum())
            s_in, s_out = s_out, s_in
        e1.record(stream)
        barrier()
        ms_eager = max_over_ranks(e0.elapsed_time(e1) / (2 * pairs))
        stages = {k: v / (2 * pairs) for k, v in solver.stage_times().items()}
        solver.stage_events = None
        it = float(torch.stack(iters).double().sum().item()) / (2 * pairs * W)
        solve_flops = float(torch.stack(flops).sum().item()) / (2 * pairs)
        ch = torch.stack(chosen).sum(0).cpu().numpy()
        conv = bool(solver.contact_solve.converged_env.all())
        counts = solver.contact_jacobian.contact_env_count.clamp(max=MAX_CONTACTS).cpu().numpy()
        final_eager = s_in.joint_qd.clone()
        # timed: graph replays from the initial state
        solver = make_solver(prec, warm, history)
        g_in, g_out = fresh_states()
        graph = solver.capture_steps(g_in, g_out, control, contacts, DT, warmup=warm_pairs)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler:
            sampler.mark_begin()
        ev0.record(stream)
        for _ in range(pairs):
            graph.replay()
        ev1.record(stream)
        barrier()
        if sampler:
            sampler.mark_end()
        ms = max_over_ranks(ev0.elapsed_time(ev1) / (2 * pairs))
        del graph
        same = bool(torch.equal(g_in.joint_qd, final_eager))
        return dict(ms=ms, ms_eager=ms_eager, stages=stages, iters=it, chosen=ch, converged=conv, counts=counts,
                    solver=solver, final=g_in, graph_matches_eager=same, solve_flops_fp64=solve_flops)

    plain = run_arm("fp64", "previous_velocity")
    prev = run_arm("fp32", "previous_impulses")
    carried = run_arm("fp32", "previous_impulses", history=1)
    sampler = ClockSampler(local_rank)
    sampler.start()
    fast = run_arm("fp32", "learned", sampler)
    clocks = sampler.stop()
    # final states of the arms agree to the solve tolerance
    dq = float((fast["final"].joint_qd - plain["final"].joint_qd).abs().max() /
               plain["final"].joint_qd.abs().max().clamp(min=1e-30))

    # ---- end to end through the public API with host buffers -----------------
    # Every step copies its state (joint_q, joint_qd) and its contacts from
    # pinned host memory and its new state back to the host.  Headline: two
    # whole steps and their copies in one graph (capture_host_steps), each
    # step's contacts copied while the step before it computes.  Beside it:
    # the same copies and eager steps serialised on one stream.
    from sap_warp_b200.runtime import SapContacts

    c_names = [k for k in vars(contacts) if isinstance(getattr(contacts, k), torch.Tensor)]
    host_state = {"joint_q": state0.joint_q.cpu().pin_memory(), "joint_qd": state0.joint_qd.cpu().pin_memory()}
    host_cs = tuple(SapContacts(**{k: getattr(contacts, k).cpu().pin_memory() for k in c_names}) for _ in range(2))
    h2d = (host_state["joint_q"].numel() * 8 + host_state["joint_qd"].numel() * 8
           + sum(getattr(host_cs[0], k).numel() * getattr(host_cs[0], k).element_size() for k in c_names))
    d2h = host_state["joint_q"].numel() * 8 + host_state["joint_qd"].numel() * 8
    solver = make_solver("fp32", "learned")
    s_in, s_out = fresh_states()
    pairs = max(args.steps // 2, 1)
    hg = solver.capture_host_steps(host_state, host_cs, s_in, s_out, control, DT,
                                   warmup=max((args.warmup + 1) // 2, 1))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(pairs):
        hg.replay()
    e1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1) / (2 * pairs))
    e2e_final_q = host_state["joint_q"].clone()
    del hg

    solver = make_solver("fp32", "learned")
    s_in, s_out = fresh_states()
    host_q = state0.joint_q.cpu().pin_memory()
    host_qd = state0.joint_qd.cpu().pin_memory()
    host_c = {k: getattr(host_cs[0], k) for k in c_names}

    def e2e_step(a, b):
        a.joint_q.copy_(host_q, non_blocking=True)
        a.joint_qd.copy_(host_qd, non_blocking=True)
        for k, v in host_c.items():
            getattr(contacts, k).copy_(v, non_blocking=True)
        solver.step(a, b, control, contacts, DT)
        host_q.copy_(b.joint_q, non_blocking=True)
        host_qd.copy_(b.joint_qd, non_blocking=True)

    for _ in range(2 * max((args.warmup + 1) // 2, 1)):
        e2e_step(s_in, s_out)
        s_in, s_out = s_out, s_in
    barrier()
    e0.record(stream)
    for _ in range(2 * pairs):
        e2e_step(s_in, s_out)
        s_in, s_out = s_out, s_in
    e1.record(stream)
    barrier()
    ms_e2e_serial = max_over_ranks(e0.elapsed_time(e1) / (2 * pairs))
    torch.cuda.synchronize()
    e2e_same = bool(torch.equal(host_q, e2e_final_q))

    # ---- contacts regenerated from the pose every step (models.site_scene):
    # contact generation + the step, the three arms, eager steps timed by
    # events after a settling prefix ----
    from sap_warp_b200.collision import ContactGenerator

    smodel, sstate0, scontrol, sshapes, _ = models.site_scene("humanoid", shard.worlds, shard.seed + 7, dev)
    site = {"worlds": W, "contacts": "32 sphere sites per world over per-site ground patches, 8-32 touching at "
                                     "the start; contacts regenerated from the pose every step (they appear and "
                                     "vanish)"}
    for label, prec, warm in (("plain_fp64", "fp64", "previous_velocity"),
                              ("previous_impulses_fp32", "fp32", "previous_impulses"),
                              ("learned_fp32", "fp32", "learned")):
        ssolver = SolverSAP(smodel, max_rigid_contact=MAX_CONTACTS, contact_preset_variant="drake",
                            hessian_precision=prec, warm_start=warm, learned_warm_start=ws if warm == "learned" else None)
        sgen = ContactGenerator(sshapes, ssolver.view, capacity=shard.worlds * MAX_CONTACTS, gap=1.0e-3)
        sa = SapState(joint_q=sstate0.joint_q.clone(), joint_qd=sstate0.joint_qd.clone(),
                      body_q=sstate0.body_q.clone(), body_f=sstate0.body_f.clone())
        sb = SapState(joint_q=sstate0.joint_q.clone(), joint_qd=sstate0.joint_qd.clone(),
                      body_q=sstate0.body_q.clone(), body_f=sstate0.body_f.clone())
        for _ in range(20 + args.warmup):
            ssolver.step(sa, sb, scontrol, sgen.generate(sa.joint_q), DT)
            sa, sb = sb, sa
        barrier()
        k_site = max(1, min(args.steps, 40))
        its, cnt = [], []
        ssolver.stage_events = []
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(k_site):
            c = sgen.generate(sa.joint_q)
            ssolver.step(sa, sb, scontrol, c, DT)
            its.append(ssolver.contact_solve.newton_iterations_env.double().mean())
            cnt.append(c.rigid_contact_count.double())
            sa, sb = sb, sa
        a1.record(stream)
        barrier()
        ms = max_over_ranks(a0.elapsed_time(a1) / k_site)
        site[label] = {"value": W * world_size / (ms * 1e-3), "ms_per_step_with_generation": ms,
                       "stages_ms": {k: v / k_site for k, v in ssolver.stage_times().items()},
                       "mean_newton_iterations": float(torch.stack(its).mean()),
                       "mean_contacts_per_world": float(torch.stack(cnt).mean()) / shard.worlds,
                       "all_converged": bool(ssolver.contact_solve.converged_env.all())}
        del ssolver, sgen
    site["speedup_vs_plain_fp64"] = (site["plain_fp64"]["ms_per_step_with_generation"]
                                     / site["learned_fp32"]["ms_per_step_with_generation"])

    # ---- stage-2 solve alone on the snapshot of the configuration -------------
    prob = scenes.humanoid_contact_problem(args.worlds, seed=SEED + 1000 * rank)
    t = problem_to_device(prob, dev)
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
    snap = {}
    for label, opts in (("fp64", make_options("armijo_decay")),
                        ("fp32", make_options("armijo_decay", hessian_precision="fp32"))):
        for _ in range(args.warmup):
            contact_solve(**t, buffers=buf, options=opts)
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k_snap = max(1, min(args.steps, 50))
        a0.record(stream)
        for _ in range(k_snap):
            contact_solve(**t, buffers=buf, options=opts)
        a1.record(stream)
        barrier()
        ms = max_over_ranks(a0.elapsed_time(a1) / k_snap)
        snap[label] = {"value": prob.num_envs * world_size / (ms * 1e-3), "ms_per_solve": ms,
                       "mean_newton_iterations": float(buf.newton_iterations.double().mean())}

    # ---- uneven batch: 8192 worlds, a third each 13 / 18 / 35 DOF, one launch ----
    mix, _ = scenes.mixed_contact_problem(2 * args.worlds, seed=3 + 1000 * rank)
    tm = problem_to_device(mix, dev)
    mbuf = ContactSolveBuffers(mix.num_envs, mix.dof_per_env, mix.max_contacts, dev)
    order = torch.as_tensor(scenes.work_order(mix), dtype=torch.int32).to(dev)
    uneven = {"worlds": mix.num_envs, "dofs": "13 (arm+box, 2 trees) / 18 / 35: padded to 35 (identity blocks), "
                                              "or each world's own count (per_world_dofs: dof_count, compact storage)",
              "contacts": "2-8 gripper / min(Poisson(12), 64)"}
    tc = problem_to_device(scenes.compact_problem(mix), dev)
    dcount = torch.as_tensor(mix.dofs_active, dtype=torch.int32).to(dev)
    for label, opts, wo, tt, dc in (
            ("fp64_sorted", make_options("armijo_decay"), order, tm, None),
            ("fp32_sorted", make_options("armijo_decay", hessian_precision="fp32"), order, tm, None),
            ("fp32_index_order", make_options("armijo_decay", hessian_precision="fp32"), None, tm, None),
            ("fp64_per_world_dofs", make_options("armijo_decay"), order, tc, dcount),
            ("fp32_per_world_dofs", make_options("armijo_decay", hessian_precision="fp32"), order, tc, dcount)):
        for _ in range(max(args.warmup, 1)):
            contact_solve(**tt, buffers=mbuf, options=opts, world_order=wo, dof_count=dc)
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k_mix = max(1, min(args.steps, 20))
        a0.record(stream)
        for _ in range(k_mix):
            contact_solve(**tt, buffers=mbuf, options=opts, world_order=wo, dof_count=dc)
        a1.record(stream)
        barrier()
        ms = max_over_ranks(a0.elapsed_time(a1) / k_mix)
        uneven[label] = {"value": mix.num_envs * world_size / (ms * 1e-3), "ms_per_solve": ms,
                         "all_converged": bool(mbuf.converged.all())}

    # ---- the uneven batch as whole steps: one model of arm + box (13 DOF),
    # quadruped (18) and humanoid (35) worlds, a third each (models.concat_models),
    # stepped as one batch (CUDA graph of two steps, replayed) ----
    per_kind = max(1, (2 * args.worlds) // 3)
    umodel, ustate, ucontrol, ucon, _ = models.mixed_rollout_scene(per_kind, 3 + 1000 * rank, dev)
    UW = int(umodel.world_count)
    uneven_step = {"worlds": UW, "dofs": "13 (arm+box) / 18 / 35, each world its own count (no padding)",
                   "contacts": "8-32 ground contacts per world", "timing": "graph of two steps, replayed"}
    for label, prec, warm in (("plain_fp64", "fp64", "previous_velocity"),
                              ("previous_impulses_fp32", "fp32", "previous_impulses"),
                              ("learned_fp32", "fp32", "learned")):
        usolver = SolverSAP(umodel, max_rigid_contact=MAX_CONTACTS, contact_preset_variant="drake",
                            hessian_precision=prec, warm_start=warm)
        ua = SapState(joint_q=ustate.joint_q.clone(), joint_qd=ustate.joint_qd.clone(), body_q=ustate.body_q.clone(),
                      body_f=ustate.body_f.clone())
        ub = SapState(joint_q=ustate.joint_q.clone(), joint_qd=ustate.joint_qd.clone(), body_q=ustate.body_q.clone(),
                      body_f=ustate.body_f.clone())
        ugraph = usolver.capture_steps(ua, ub, ucontrol, ucon, DT, warmup=max((args.warmup + 1) // 2, 1))
        barrier()
        k_u = max(1, min(args.steps, 20) // 2)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(k_u):
            ugraph.replay()
        a1.record(stream)
        barrier()
        ms = max_over_ranks(a0.elapsed_time(a1) / (2 * k_u))
        del ugraph
        uneven_step[label] = {"value": UW * world_size / (ms * 1e-3), "ms_per_step": ms,
                              "mean_newton_iterations": float(usolver.contact_solve.newton_iterations_env.double().mean()),
                              "all_converged": bool(usolver.contact_solve.converged_env.all())}

    # ---- the launch-shape autotuner's view: each resident-CTA count per SM
    # timed on the snapshot and on the uneven batch (SolveAutotuner's rule) ----
    from sap_warp_b200 import _abi as _abi_mod
    from sap_warp_b200._lib import load as _load_lib
    from sap_warp_b200.autotune import SolveAutotuner

    tuned = {}
    for label, tt, bb, opts, wo in (
            ("humanoid_fp32", t, buf, make_options("armijo_decay", hessian_precision="fp32"), None),
            ("humanoid_fp64", t, buf, make_options("armijo_decay"), None),
            ("uneven_fp32", tm, mbuf, make_options("armijo_decay", hessian_precision="fp32"), order)):
        occ = int(_load_lib().sapb_contact_solve_occupancy(bb.dof_per_env, bb.max_contacts, opts.hessian_precision,
                                                            opts.line_search_variant))

        def time_ms(shape, tt=tt, bb=bb, opts=opts, wo=wo):
            opts.ctas_per_sm, opts.ldlt_block, opts.threads_per_cta = shape
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            contact_solve(**tt, buffers=bb, options=opts, world_order=wo)
            e1.record(stream)
            e1.synchronize()
            return e0.elapsed_time(e1)

        wl = (__import__("ctypes").c_int32 * 8)()
        nw = max(min(int(_load_lib().sapb_contact_solve_ldlt_blocks(bb.dof_per_env, wl, 8)), 8), 1)
        # the 256-thread runtime-size kernel at its own occupancy, its width
        occ_w = int(_load_lib().sapb_contact_solve_occupancy_threads(bb.dof_per_env, bb.max_contacts,
                                                                      opts.hessian_precision,
                                                                      opts.line_search_variant, 256))
        gw = (__import__("ctypes").c_int32 * 8)()
        _load_lib().sapb_contact_solve_ldlt_blocks(1, gw, 8)
        cands = [(k, int(wl[w]), 128) for w in range(nw) for k in range(1, occ + 1)]
        cands += [(k, int(gw[0]), 256) for k in range(1, occ_w + 1)]
        tuner = SolveAutotuner(repeats=5)
        chosen = tuner.tune(label, cands, time_ms, default=(occ, int(wl[0]), 128))
        opts.ctas_per_sm, opts.ldlt_block, opts.threads_per_cta = 0, 0, 0
        tuned[label] = {"occupancy": occ, "occupancy_256_threads": occ_w, "ldlt_blocks": [int(wl[w]) for w in range(nw)],
                        "chosen": list(chosen), "ms": tuner.table[label]["ms"]}

    # ---- worlds of 64 free boxes (384 DOFs, ~400 contacts): tree-blocked solve ----
    boxes = scenes.box_stack_problem(512, seed=4 + 1000 * rank)
    tb = blocked_problem_to_device(boxes, dev)
    bbuf = ContactSolveBuffers(boxes.num_envs, boxes.dof_per_env, boxes.max_contacts, dev)
    box_line = {"worlds": boxes.num_envs, "trees": "64 free boxes (6 DOF each, n = 384)",
                "contacts": f"mean {float(boxes.contact_count.mean()):.0f} per world (stacks + side contacts)"}
    for label, prec in (("fp64", "fp64"), ("fp32", "fp32")):
        opts = make_options("armijo_decay", hessian_precision=prec, linear_solve_precision=prec)
        for _ in range(max(args.warmup, 1)):
            blocked_contact_solve(buffers=bbuf, options=opts, trees_per_env=64, **tb)
        barrier()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k_box = max(1, min(args.steps, 5))
        a0.record(stream)
        for _ in range(k_box):
            blocked_contact_solve(buffers=bbuf, options=opts, trees_per_env=64, **tb)
        a1.record(stream)
        barrier()
        ms = max_over_ranks(a0.elapsed_time(a1) / k_box)
        box_line[label] = {"value": boxes.num_envs * world_size / (ms * 1e-3), "ms_per_solve": ms,
                           "mean_newton_iterations": float(bbuf.newton_iterations.double().mean()),
                           "all_converged": bool(bbuf.converged.all())}

    # ---- the whole step on 512 worlds of 64 free boxes (tree-blocked free
    # motion and solve, FP32 Hessian), previous-velocity vs previous-impulses start
    bmodel, bstate, bcontrol, bcon, _, bhost = models.box_scene(512, 75 + 1000 * rank, dev)
    box_step = {"worlds": 512, "trees": "64 free boxes per world (n = 384)",
                "contacts": f"{int(bcon.rigid_contact_count.item())} in all"}
    for warm in ("previous_velocity", "previous_impulses", "learned"):
        bsolver = SolverSAP(bmodel, max_rigid_contact=512, contact_preset_variant="drake", hessian_precision="fp32",
                            warm_start=warm)
        ba = SapState(joint_q=bstate.joint_q.clone(), joint_qd=bstate.joint_qd.clone(), body_q=bstate.body_q.clone(),
                      body_f=bstate.body_f.clone())
        bb = SapState(joint_q=bstate.joint_q.clone(), joint_qd=bstate.joint_qd.clone(), body_q=bstate.body_q.clone(),
                      body_f=bstate.body_f.clone())
        for _ in range(2):
            bsolver.step(ba, bb, bcontrol, bcon, DT)
            ba, bb = bb, ba
        barrier()
        k_bs = max(1, min(args.steps, 10))
        its, acc = [], []
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(k_bs):
            bsolver.step(ba, bb, bcontrol, bcon, DT)
            its.append(bsolver.contact_solve.newton_iterations_env.sum())
            acc.append(bsolver.contact_solve.warm_start_accepted_env.sum())
            ba, bb = bb, ba
        a1.record(stream)
        barrier()
        ms = max_over_ranks(a0.elapsed_time(a1) / k_bs)
        box_step[warm] = {"value": 512 * world_size / (ms * 1e-3), "ms_per_step": ms,
                          "mean_newton_iterations": float(torch.stack(its).double().sum()) / (512 * k_bs),
                          "candidate_taken": float(torch.stack(acc).double().sum()) / (512 * k_bs),
                          "all_converged": bool(bsolver.contact_solve.converged_env.all())}
    # ---- worlds of a 7-revolute arm gripping one of its free boxes (trees of
    # 7 and 6 DOFs, tree-blocked in blocks of 7): the dense and the
    # tree-blocked step on 2048 worlds of the arm and 8 boxes (55 DOFs: both
    # layouts apply), and the tree-blocked step on 512 worlds of the arm and
    # 32 boxes (199 DOFs: beyond the dense kernel)
    def time_steps(solver, st0, ctl, con, worlds, k):
        sa = SapState(joint_q=st0.joint_q.clone(), joint_qd=st0.joint_qd.clone(), body_q=st0.body_q.clone(),
                      body_f=st0.body_f.clone())
        sb = SapState(joint_q=st0.joint_q.clone(), joint_qd=st0.joint_qd.clone(), body_q=st0.body_q.clone(),
                      body_f=st0.body_f.clone())
        for _ in range(2):
            solver.step(sa, sb, ctl, con, DT)
            sa, sb = sb, sa
        barrier()
        its = []
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(k):
            solver.step(sa, sb, ctl, con, DT)
            its.append(solver.contact_solve.newton_iterations_env.sum())
            sa, sb = sb, sa
        a1.record(stream)
        barrier()
        ms = max_over_ranks(a0.elapsed_time(a1) / k)
        return {"value": worlds * world_size / (ms * 1e-3), "ms_per_step": ms,
                "mean_newton_iterations": float(torch.stack(its).double().sum()) / (worlds * k),
                "all_converged": bool(solver.contact_solve.converged_env.all())}

    k_arm = max(1, min(args.steps, 10))
    arm_step = {"trees": "a 7-revolute fixed-base arm (7 DOFs) and free boxes (6 DOFs each), tree-blocked in "
                         "blocks of 7; the arm's last link grips one box (2-8 contacts coupling the two trees)"}
    amodel, astate, acontrol, acon, _, _ = models.box_scene(2048, 77 + 1000 * rank, dev, boxes=8, sites=(3, 5),
                                                            arm=True)
    arm_step["arm_8_boxes"] = {"worlds": 2048, "dofs": 55,
                               "contacts": f"{int(acon.rigid_contact_count.item())} in all"}
    for label, blocked, prec, warm in (("dense_fp64_previous_velocity", False, "fp64", "previous_velocity"),
                                       ("blocked_fp64_previous_velocity", True, "fp64", "previous_velocity"),
                                       ("dense_fp32_previous_impulses", False, "fp32", "previous_impulses"),
                                       ("blocked_fp32_previous_impulses", True, "fp32", "previous_impulses")):
        # the dense arms autotuned (CTAs per SM, LDL^T width, 128 or 256
        # threads per world: these worlds leave one CTA per SM)
        asolver = SolverSAP(amodel, max_rigid_contact=112, contact_preset_variant="drake", hessian_precision=prec,
                            warm_start=warm, tree_blocked=blocked, autotune=not blocked)
        arm_step["arm_8_boxes"][label] = time_steps(asolver, astate, acontrol, acon, 2048, k_arm)
        if not blocked:
            arm_step["arm_8_boxes"][label]["autotune"] = {
                k.split("-NVIDIA")[0]: {"chosen": v["choice"], "ms": v["ms"]}
                for k, v in asolver.contact_solve.autotuner.table.items()}
        del asolver
    amodel, astate, acontrol, acon, _, _ = models.box_scene(512, 78 + 1000 * rank, dev, boxes=32, sites=(8, 12),
                                                            arm=True)
    arm_step["arm_32_boxes"] = {"worlds": 512, "dofs": 199,
                                "contacts": f"{int(acon.rigid_contact_count.item())} in all"}
    for label, prec, warm in (("blocked_fp64_previous_velocity", "fp64", "previous_velocity"),
                              ("blocked_fp32_previous_impulses", "fp32", "previous_impulses")):
        asolver = SolverSAP(amodel, max_rigid_contact=384, contact_preset_variant="drake", hessian_precision=prec,
                            warm_start=warm)
        arm_step["arm_32_boxes"][label] = time_steps(asolver, astate, acontrol, acon, 512, k_arm)
        del asolver
    del amodel, astate, acontrol, acon

    # ---- contact generation for the same worlds' shapes (64 boxes each + a
    # ground plane): forward kinematics, count, scan, write ----
    from sap_warp_b200.collision import ContactGenerator
    from sap_warp_b200.solver import _ModelView

    bshapes = models.box_shapes(bhost)
    gen = ContactGenerator(bshapes, _ModelView(bmodel), capacity=512 * 1024, gap=2.0e-3)
    for _ in range(3):
        gen.generate(bstate.joint_q)
    barrier()
    k_gen = max(1, min(args.steps, 20))
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(k_gen):
        gen.generate(bstate.joint_q)
    a1.record(stream)
    barrier()
    ms = max_over_ranks(a0.elapsed_time(a1) / k_gen)
    pairs = 512 * (64 * 1 + 64 * 63 // 2)
    contact_gen = {"worlds": 512, "shapes": "64 boxes per world + a shared ground plane",
                   "candidate_pairs": pairs, "contacts": int(gen.count.item()), "ms_per_call": ms,
                   "value": 512 * world_size / (ms * 1e-3), "unit": "world-generations/s",
                   "pairs_per_s": pairs * world_size / (ms * 1e-3)}
    del gen, bsolver, bmodel, bstate, bcon

    total = W * world_size
    value = total / (fast["ms"] * 1e-3)
    # measured FMA rates of this GPU (the FP64 pipe's roofline denominator)
    fma = {}
    for label, prec in (("fp64", _abi_mod.SAPB_FP64), ("fp32", _abi_mod.SAPB_FP32)):
        rate = __import__("ctypes").c_double(0.0)
        st = _load_lib().sapb_measure_fma_rate(prec, 1 << 14, __import__("ctypes").byref(rate),
                                               __import__("ctypes").c_void_p(stream.cuda_stream))
        fma[label] = rate.value if st == 0 else float("nan")
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    n = 35
    solve_ms = fast["stages"].get("contact_solve", float("nan"))
    # learned arm on a fixed contact set: the base velocity (the history's
    # start) and the network's impulse set, all zero, so no factor is read
    alg = float(solve_bytes_per_world(n, fast["counts"], velocities=1, impulse_sets=1).sum())
    achieved = alg / (solve_ms * 1e-3) / 1e9
    # FP64 arithmetic of the plain arm's solve (algorithmic count from its
    # measured Newton iterations and line-search trials) against the measured
    # FP64 FMA rate
    pf = plain["solve_flops_fp64"]
    plain_solve_ms = plain["stages"].get("contact_solve", float("nan"))
    fp64_achieved = pf / (plain_solve_ms * 1e-3) / 1e12
    fp64_peak = fma["fp64"] / 1e12
    # this library's kernels per step of the learned arm: contact scatter, contact history, free motion,
    # features, active tiles, MLP forward, impulses, solve, work order, tail
    launches_per_step = 10
    line = {
        "metric": METRIC, "value": value, "unit": "world-steps/s", "n_gpus": world_size, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": fast["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": plain["ms"] / fast["ms"],
        "vs_baseline_basis": "the metric's own baseline: the plain FP64 arm (the reference's method: FP64 "
                             "throughout, previous-velocity warm start) on the same B200, same scene, window and "
                             "tolerance -- its ms_per_step over this arm's (no published number exists)",
        "plain_fp64_value": total / (plain["ms"] * 1e-3), "plain_fp64_ms_per_step": plain["ms"],
        "speedup_vs_plain_fp64": plain["ms"] / fast["ms"],
        "solve_stage_speedup_vs_plain_fp64": plain["stages"].get("contact_solve", float("nan")) / max(
            fast["stages"].get("contact_solve", float("nan")) + fast["stages"].get("warm_start", 0.0), 1e-9),
        "newton_iterations_per_world_step": {"learned_fp32": fast["iters"], "plain_fp64": plain["iters"],
                                             "previous_impulses_fp32": prev["iters"],
                                             "carried_impulses_fp32": carried["iters"]},
        "dtype": "f64 (FP32 Hessian/factor)", "data": "synthetic (seeded rollout scene)",
        "config": {"workload": f"{W} humanoid worlds x 35 DOF (6+29 revolute), 8-32 ground contacts, full "
                               "SolverSAP step (drake preset), armijo_decay to reference tolerances, rollout",
                   "worlds_per_gpu": W, "dof_per_env": n, "max_contacts": MAX_CONTACTS, "dt": DT,
                   "parallelism": f"world shards x{world_size}",
                   "l2": "per-step working set (A, J, factor, rows) larger than L2",
                   "window": f"steps {SETTLE_STEPS}+ of the rollout (after an untimed settling prefix)"},
        "timing": "CUDA graph of two whole steps replayed steps/2 times after the warm-up; stages and "
                  "statistics from an eager pass over the same steps of the same trajectory",
        "plain_fp64": {"value": total / (plain["ms"] * 1e-3), "ms_per_step": plain["ms"],
                       "ms_per_step_eager": plain["ms_eager"],
                       "mean_newton_iterations": plain["iters"], "all_converged": plain["converged"],
                       "stages_ms": plain["stages"]},
        "learned_fp32": {"mean_newton_iterations": fast["iters"], "all_converged": fast["converged"],
                         "ms_per_step_eager": fast["ms_eager"],
                         "graph_replay_matches_eager": fast["graph_matches_eager"],
                         "chosen_start": {"previous_velocity": int(fast["chosen"][0]),
                                          "history_impulses_and_network": int(fast["chosen"][1])},
                         "stages_ms": fast["stages"], "speedup_vs_plain_fp64": plain["ms"] / fast["ms"],
                         "max_rel_qd_diff_vs_plain_fp64_after_rollout": dq},
        "previous_impulses_fp32": {"value": total / (prev["ms"] * 1e-3), "ms_per_step": prev["ms"],
                                   "mean_newton_iterations": prev["iters"], "stages_ms": prev["stages"],
                                   "impulse_history": 3},
        "carried_impulses_fp32": {"value": total / (carried["ms"] * 1e-3), "ms_per_step": carried["ms"],
                                  "mean_newton_iterations": carried["iters"], "stages_ms": carried["stages"],
                                  "impulse_history": 1},
        "stage2_solve_only": snap,
        "uneven_batch_solve_only": uneven,
        "uneven_batch_step": uneven_step,
        "box_worlds_solve_only": box_line,
        "box_worlds_step": box_step,
        "arm_box_worlds_step": arm_step,
        "regenerated_contacts_rollout": site,
        "contact_generation": contact_gen,
        "autotune_launch_shape": tuned,
        "e2e": {"value": total / (ms_e2e * 1e-3), "unit": "world-steps/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": ms_e2e,
                "path": "SolverSAP.capture_host_steps: two steps and their host copies per graph replay, "
                        "contacts copied on a second stream during the previous step",
                "serial_eager": {"value": total / (ms_e2e_serial * 1e-3), "ms_per_step": ms_e2e_serial},
                "matches_serial_eager": e2e_same},
        "roofline": {"bound": "hbm", "kernel": "contact_solve_kernel", "achieved": achieved, "peak": hbm_peak,
                     "unit": "GB/s", "frac": achieved / hbm_peak, "traffic": NCU_SOLVE_TRAFFIC_BYTES,
                     "note": "achieved = algorithmic bytes of the solve launch / its mean duration inside the "
                             "timed steps (of measured peak); the kernel is latency bound, not HBM bound",
                     "fp64": {"kernel": "contact_solve_kernel (plain FP64 arm)", "achieved": fp64_achieved,
                              "peak": fp64_peak, "unit": "TFLOP/s", "frac": fp64_achieved / fp64_peak,
                              "peak_source": "sapb_measure_fma_rate on this GPU (FP64 FMA chains), this run",
                              "flops": "algorithmic: per world k (6 C n^2 + n^3/3 + 2 n^2 + 6 C n) + "
                                       "(k + 1)(4 n^2 + 12 C n) + 80 C t, k Newton iterations, t trials"}},
        "fma_rate_tflops": {k: v / 1e12 for k, v in fma.items()},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        scene = cpu_scene(1024, SEED)
        sec, k = cpu_steps(scene, 1000, cores, min_seconds=10.0)
        line["cpu_baseline"] = {"value": 1024 / sec, "unit": "world-steps/s", "cores": cores, "kind": "port",
                                "sample": f"{k} steps of a 1024-world rollout (C restatement: free motion, rows, "
                                          f"solve, integration; OpenMP over worlds)"}
        line["error_vs_fp64_oracle"] = oracle_errors(dev)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
