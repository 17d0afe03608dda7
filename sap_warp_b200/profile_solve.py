"""Run a fixed workload of the contact step for profiling.

    python -m sap_warp_b200.profile_solve --mode snapshot --worlds 4096 --precision fp64 --launches 5
    python -m sap_warp_b200.profile_solve --mode rollout --worlds 4096 --steps 8 --warm-start learned \\
        --precision fp32
    python -m sap_warp_b200.profile_solve --mode boxes --worlds 512 --precision fp32 --launches 3
    python -m sap_warp_b200.profile_solve --mode arm_boxes --worlds 4096 --boxes 8 --steps 6 --precision fp64 \
        --warm-start previous_velocity --layout blocked

snapshot: the stage-2 solve alone on the batched humanoid problem (A, J
given): warm-up launches, then `--launches` timed launches.
rollout: SolverSAP steps (drake preset) of the humanoid rollout scene with
the given warm start and Hessian precision: `--steps` steps, the last half
timed, after `--settle` steps of a plain FP64 solver (the bench's settling
prefix).  boxes: the tree-blocked solve alone on worlds of 64 free boxes
(scenes.box_stack_problem).  arm_boxes: SolverSAP steps on worlds of a
7-revolute arm gripping one of `--boxes` free boxes (models.box_scene with
the arm), in the tree-blocked or the dense layout, `--steps` steps, the last
half timed.  Each prints the mean time per launch / step.  Used as the target
command of ncu captures (select a kernel with `-k regex:...` and skip the
warm-up launches with `-s`).
"""

from __future__ import annotations

import argparse

import torch

from . import models, scenes
from ._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device


def snapshot(args, dev) -> None:
    prob = scenes.humanoid_contact_problem(args.worlds, seed=args.seed)
    t = problem_to_device(prob, dev)
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
    opt = make_options(args.variant, hessian_precision=args.precision, linear_solve_precision=args.precision)
    for _ in range(args.warmup):
        contact_solve(**t, buffers=buf, options=opt)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.launches):
        contact_solve(**t, buffers=buf, options=opt)
    e1.record()
    torch.cuda.synchronize()
    print(f"{args.precision} {args.worlds} worlds: {e0.elapsed_time(e1) / max(args.launches, 1):.4f} ms/launch, "
          f"mean Newton iterations {buf.newton_iterations.double().mean().item():.3f}")


def boxes(args, dev) -> None:
    from ._solve import blocked_contact_solve, blocked_problem_to_device

    prob = scenes.box_stack_problem(args.worlds, seed=args.seed)
    t = blocked_problem_to_device(prob, dev)
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
    opt = make_options(args.variant, hessian_precision=args.precision, linear_solve_precision=args.precision)
    for _ in range(args.warmup):
        blocked_contact_solve(**t, buffers=buf, options=opt, trees_per_env=prob.trees_per_env)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.launches):
        blocked_contact_solve(**t, buffers=buf, options=opt, trees_per_env=prob.trees_per_env)
    e1.record()
    torch.cuda.synchronize()
    print(f"boxes {args.precision} {args.worlds} worlds: {e0.elapsed_time(e1) / max(args.launches, 1):.4f} "
          f"ms/launch, mean Newton iterations {buf.newton_iterations.double().mean().item():.3f}")


def rollout(args, dev) -> None:
    from .runtime import SapState
    from .solver import SolverSAP

    model, state, control, contacts, _ = models.rollout_scene("humanoid", args.worlds, args.seed, dev)
    solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision=args.precision,
                       warm_start=args.warm_start)
    other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
    if args.settle > 0:
        settler = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp64")
        for _ in range(args.settle):
            settler.step(state, other, control, contacts, 2.0e-3)
            state, other = other, state
        del settler
    half = max(args.steps // 2, 1)
    for _ in range(args.steps - half):
        solver.step(state, other, control, contacts, 2.0e-3)
        state, other = other, state
    torch.cuda.synchronize()
    solver.stage_events = []
    for _ in range(half):
        solver.step(state, other, control, contacts, 2.0e-3)
        state, other = other, state
    stages = {k: round(v / half, 4) for k, v in solver.stage_times().items()}
    print(f"rollout {args.worlds} worlds, {args.warm_start}, {args.precision}: stages ms/step {stages}, "
          f"mean Newton iterations {solver.contact_solve.newton_iterations_env.double().mean().item():.3f}")


def arm_boxes(args, dev) -> None:
    from .runtime import SapState
    from .solver import SolverSAP

    model, state, control, contacts, _, _ = models.box_scene(args.worlds, args.seed, dev, boxes=args.boxes,
                                                             sites=(3, 5), arm=True)
    solver = SolverSAP(model, max_rigid_contact=112, contact_preset_variant="drake", hessian_precision=args.precision,
                       warm_start=args.warm_start, tree_blocked=args.layout == "blocked")
    other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
    half = max(args.steps // 2, 1)
    for _ in range(args.steps - half):
        solver.step(state, other, control, contacts, 2.0e-3)
        state, other = other, state
    torch.cuda.synchronize()
    solver.stage_events = []
    for _ in range(half):
        solver.step(state, other, control, contacts, 2.0e-3)
        state, other = other, state
    stages = {k: round(v / half, 4) for k, v in solver.stage_times().items()}
    print(f"arm and {args.boxes} boxes, {args.worlds} worlds, {args.layout}, {args.warm_start}, {args.precision}: "
          f"stages ms/step {stages}, mean Newton iterations "
          f"{solver.contact_solve.newton_iterations_env.double().mean().item():.3f}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", choices=["snapshot", "rollout", "boxes", "arm_boxes"], default="snapshot")
    ap.add_argument("--boxes", type=int, default=8, help="arm_boxes: free boxes per world")
    ap.add_argument("--layout", choices=["blocked", "dense"], default="blocked", help="arm_boxes: the layout")
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--variant", default="armijo_decay")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--launches", type=int, default=5)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--settle", type=int, default=0,
                    help="rollout: untimed steps of a plain FP64 solver first (its solve launches come first)")
    ap.add_argument("--warm-start", default="learned",
                    choices=["previous_velocity", "previous_impulses", "learned"])
    ap.add_argument("--seed", type=int, default=2)
    args = ap.parse_args()
    dev = torch.device("cuda:0")
    {"snapshot": snapshot, "rollout": rollout, "boxes": boxes, "arm_boxes": arm_boxes}[args.mode](args, dev)


if __name__ == "__main__":
    main()
