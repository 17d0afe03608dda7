"""Run the batched contact solve on a fixed workload for profiling.

    python -m sap_warp_b200.profile_solve --worlds 4096 --precision fp64 --launches 5

Builds the bench's humanoid workload, issues warm-up launches, then times
`--launches` launches with CUDA events and prints the mean.  Used as the
target command of ncu captures (select the solve kernel with
`-k regex:contact_solve` and skip the warm-up launches with `-s`).
"""

from __future__ import annotations

import argparse

import torch

from . import scenes
from ._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--worlds", type=int, default=4096)
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--variant", default="armijo_decay")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--launches", type=int, default=5)
    ap.add_argument("--seed", type=int, default=2)
    args = ap.parse_args()
    dev = torch.device("cuda:0")
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


if __name__ == "__main__":
    main()
