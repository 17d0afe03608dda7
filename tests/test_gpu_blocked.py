"""Tree-blocked solve (sapb_blocked_contact_solve) of worlds of free boxes:
parity with the CPU oracle run on the same problem in the dense layout, with
the dense GPU kernel where both apply, the dense -> blocked gather, the
full-size (64 boxes, 384 DOFs) case and the fill-capacity status."""

import numpy as np
import pytest
import torch

from sap_warp_b200 import _abi, scenes
from sap_warp_b200._solve import (ContactSolveBuffers, blocked_contact_solve, blocked_fill_capacity,
                                  blocked_problem_to_device, contact_solve, dense_to_blocked, make_options,
                                  problem_to_device)
from tests import sap_numpy as sn
from tests.test_gpu_contact_solve import assert_parity

pytestmark = pytest.mark.gpu

KEYS = ("v", "contact_gamma", "contact_mode", "cost", "newton_iterations", "line_search_iterations", "converged",
        "status", "grad_norm")


def run_blocked(bp, device, variant="armijo_decay", **kw):
    t = blocked_problem_to_device(bp, device)
    buf = ContactSolveBuffers(bp.num_envs, bp.dof_per_env, bp.max_contacts, device)
    blocked_contact_solve(buffers=buf, options=make_options(variant, **kw), trees_per_env=bp.trees_per_env,
                          tree_dofs=bp.tree_dofs, **t)
    torch.cuda.synchronize()
    return {k: getattr(buf, k).cpu().numpy() for k in KEYS}


@pytest.mark.parametrize("variant", ["armijo_decay", "exact_root", "monotone_decay"])
def test_box_stacks_parity_fp64(cuda_device, oracle, variant):
    bp = scenes.box_stack_problem(16, seed=41, boxes=16, max_contacts=128, sites=(4, 6))
    d = bp.to_dense()
    ref = oracle.solve(d, variant)
    gpu = run_blocked(bp, cuda_device, variant)
    assert np.all(ref["converged"] == 1)
    if variant == "monotone_decay":
        same = gpu["newton_iterations"] == ref["newton_iterations"]
        assert same.mean() > 0.9
        np.testing.assert_array_equal(gpu["converged"], ref["converged"])
        return
    assert_parity(d, gpu, ref)
    assert np.all(gpu["status"] == 0)
    assert np.abs(gpu["newton_iterations"] - ref["newton_iterations"]).max() <= 3


def test_box_stacks_mixed_precision(cuda_device, oracle):
    bp = scenes.box_stack_problem(16, seed=42, boxes=16, max_contacts=128, sites=(4, 6))
    d = bp.to_dense()
    ref = oracle.solve(d, "armijo_decay")
    gpu = run_blocked(bp, cuda_device, "armijo_decay", hessian_precision="fp32", linear_solve_precision="fp32")
    # FP32 Newton directions, FP64 gradient and test: the same optimum
    np.testing.assert_array_equal(gpu["converged"], 1)
    assert_parity(d, gpu, ref, tight=1e-5, loose=1e-4, max_loose_frac=0.1)


def test_blocked_matches_dense_kernel(cuda_device):
    # 8 boxes = 48 DOFs: within the dense kernel's range, so both GPU paths apply
    bp = scenes.box_stack_problem(64, seed=43, boxes=8, max_contacts=64, sites=(2, 4))
    d = bp.to_dense()
    t = problem_to_device(d, cuda_device)
    buf = ContactSolveBuffers(d.num_envs, d.dof_per_env, d.max_contacts, cuda_device)
    contact_solve(**t, buffers=buf, options=make_options("armijo_decay"))
    torch.cuda.synchronize()
    dense = {k: getattr(buf, k).cpu().numpy() for k in KEYS}
    blocked = run_blocked(bp, cuda_device)
    assert_parity(d, blocked, dense, tight=1e-8, loose=1e-4)
    np.testing.assert_array_equal(blocked["converged"], dense["converged"])


def test_dense_to_blocked_gather(cuda_device):
    bp = scenes.box_stack_problem(4, seed=44, boxes=12, max_contacts=96, sites=(3, 5))
    d = bp.to_dense()
    t = problem_to_device(d, cuda_device)
    g = dense_to_blocked(t, d.num_envs, d.dof_per_env, d.max_contacts, bp.trees_per_env)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(g["tree_mass"].cpu().numpy(), bp.tree_mass)
    live = np.arange(d.max_contacts)[None, :] < bp.contact_count[:, None]
    np.testing.assert_array_equal(g["contact_tree"].cpu().numpy()[live], bp.contact_tree[live])
    np.testing.assert_array_equal(g["jacobian"].cpu().numpy()[live], bp.jacobian[live])


def test_full_size_box_worlds(cuda_device, oracle):
    """64 boxes (384 DOFs), ~400 contacts per world: every world converges to a
    stationary point (checked in numpy), and two worlds match the oracle."""
    bp = scenes.box_stack_problem(48, seed=4)
    assert bp.dof_per_env == 384 and bp.contact_count.min() > 300
    for prec in ("fp64", "fp32"):
        gpu = run_blocked(bp, cuda_device, "armijo_decay", hessian_precision=prec, linear_solve_precision=prec)
        assert np.all(gpu["converged"] == 1) and np.all(gpu["status"] == 0), prec
        d = bp.subset([0, 1]).to_dense()
        n = d.dof_per_env
        V = gpu["v"].reshape(-1, n)
        for e in range(2):
            c = d.contact_count[e]
            _, grad, _, _ = sn.objective(V[e], d.dynamics_matrix[e], d.v_star.reshape(-1, n)[e], d.jacobian[e],
                                         d.phi0[e], d.w_eff[e], d.mu[e], d.stiffness[e], d.tau_d[e], c)
            dsc = 1.0 / np.sqrt(np.diag(d.dynamics_matrix[e]))
            s = max(np.linalg.norm(dsc * (d.dynamics_matrix[e] @ V[e])), 1.0)
            assert np.linalg.norm(dsc * grad) <= 1e-6 * s * 1.01 + 1e-12
    ref = oracle.solve(bp.subset([0, 1]).to_dense(), "armijo_decay")
    gpu = run_blocked(bp.subset([0, 1]), cuda_device, "armijo_decay")
    assert_parity(bp.subset([0, 1]).to_dense(), gpu, ref, max_loose_frac=0.5)


def test_fill_capacity_status(cuda_device):
    """A world whose contacts couple most pairs of its 64 trees needs more
    off-diagonal factor blocks than fit on chip: it reports
    SAPB_WORLD_FACTOR_CAPACITY and returns v = v*; its neighbours solve."""
    bp = scenes.box_stack_problem(3, seed=45)
    cap = blocked_fill_capacity(64, 6, bp.max_contacts, "fp64")
    assert 0 < cap < 64 * 63 // 2
    rng = np.random.default_rng(0)
    live = int(bp.contact_count[1])
    for c in range(live):  # world 1: contacts between random pairs of trees
        a, b = rng.choice(64, size=2, replace=False)
        bp.contact_tree[1, c] = (a, b)
    gpu = run_blocked(bp, cuda_device)
    assert gpu["status"][1] == _abi.SAPB_WORLD_FACTOR_CAPACITY and gpu["converged"][1] == 0
    n = bp.dof_per_env
    np.testing.assert_array_equal(gpu["v"].reshape(-1, n)[1], bp.v_star.reshape(-1, n)[1])
    assert gpu["converged"][0] == 1 and gpu["converged"][2] == 1


def test_blocked_candidate_start_matches_dense_kernel(cuda_device):
    """One set of candidate impulses (the plain solution, scaled near 1 in
    half the worlds and by 4 in the others): the blocked solve takes the
    same starts as the dense kernel (both FP64) and reaches the same answer."""
    bp = scenes.box_stack_problem(64, seed=45, boxes=8, max_contacts=64, sites=(2, 4))
    d = bp.to_dense()
    t = problem_to_device(d, cuda_device)
    buf = ContactSolveBuffers(d.num_envs, d.dof_per_env, d.max_contacts, cuda_device)
    contact_solve(**t, buffers=buf, options=make_options("armijo_decay"))
    torch.cuda.synchronize()
    scale = torch.where(torch.arange(d.num_envs, device=cuda_device) % 2 == 0, 1.02, 4.0).double()
    gamma0 = (buf.contact_gamma.reshape(d.num_envs, d.max_contacts, 3) * scale[:, None, None]).contiguous()
    buf_d = ContactSolveBuffers(d.num_envs, d.dof_per_env, d.max_contacts, cuda_device)
    contact_solve(**t, buffers=buf_d, options=make_options("armijo_decay"), gamma0=gamma0)
    torch.cuda.synchronize()
    dense = {k: getattr(buf_d, k).cpu().numpy() for k in KEYS + ("warm_start_accepted",)}
    tb = blocked_problem_to_device(bp, cuda_device)
    buf_b = ContactSolveBuffers(bp.num_envs, bp.dof_per_env, bp.max_contacts, cuda_device)
    blocked_contact_solve(buffers=buf_b, options=make_options("armijo_decay"), trees_per_env=bp.trees_per_env,
                          tree_dofs=bp.tree_dofs, gamma0=gamma0, **tb)
    torch.cuda.synchronize()
    blocked = {k: getattr(buf_b, k).cpu().numpy() for k in KEYS + ("warm_start_accepted",)}
    acc = blocked["warm_start_accepted"]
    np.testing.assert_array_equal(acc, dense["warm_start_accepted"])
    assert acc[0::2].mean() > 0.9 and acc[1::2].mean() < acc[0::2].mean()  # near-solution sets taken
    assert_parity(d, blocked, dense, tight=1e-8, loose=1e-4)
    np.testing.assert_array_equal(blocked["converged"], 1)
    # near the solution a world needs fewer iterations than from the plain start
    assert blocked["newton_iterations"][0::2].mean() < dense_plain_iterations(buf)


def dense_plain_iterations(buf):
    return float(buf.newton_iterations.double().mean())


def test_box_rollout_previous_impulses(cuda_device):
    """64-box worlds stepped by SolverSAP with the previous step's impulses
    as a candidate start: every step converges, the candidate is taken in
    most worlds after the first step, Newton iterations drop against the
    previous-velocity start (by about an eighth on these stacks: stiction
    keeps Newton long even near the solution), and both runs end at the same
    state to the solve tolerance."""
    from sap_warp_b200 import models
    from sap_warp_b200.runtime import SapState
    from sap_warp_b200.solver import SolverSAP

    model, state, control, con, _, _ = models.box_scene(16, 74, cuda_device)
    runs = {}
    for warm in ("previous_velocity", "previous_impulses"):
        solver = SolverSAP(model, max_rigid_contact=512, contact_preset_variant="drake", hessian_precision="fp32",
                           warm_start=warm)
        assert solver.contact_solve.tree_blocked
        a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        iters, taken = [], []
        for k in range(12):
            solver.step(a, b, control, con, 2e-3)
            assert bool(solver.contact_solve.converged_env.all())
            if k >= 2:
                iters.append(float(solver.contact_solve.newton_iterations_env.double().mean()))
                taken.append(float(solver.contact_solve.warm_start_accepted_env.double().mean()))
            a, b = b, a
        runs[warm] = (np.mean(iters), np.mean(taken), a.joint_qd.clone())
    it_v, _, qd_v = runs["previous_velocity"]
    it_i, taken_i, qd_i = runs["previous_impulses"]
    assert taken_i > 0.5
    assert it_i < it_v
    rel = float((qd_i - qd_v).abs().max() / qd_v.abs().max().clamp(min=1e-30))
    assert rel < 1e-3
