"""The whole SolverSAP step on worlds of free boxes in the tree-blocked
layout: the blocked free motion and contact rows against the dense ones on
the GPU, one step against the C oracle pipeline (free motion, rows, dense
solve, integration), and a full-size (64 boxes, 384 DOFs) rollout, eager and
replayed from a CUDA graph."""

import numpy as np
import pytest
import torch

from sap_warp_b200 import models, scenes
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SapContactJacobian, SolverSAP
from tests.test_gpu_contact_solve import assert_parity

pytestmark = pytest.mark.gpu


def _clone(state):
    return SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                    body_f=state.body_f.clone())


@pytest.mark.parametrize("weight_mode,point_mode", [("body_inertia", "witness_point"),
                                                    ("diag_delassus", "contact_midpoint")])
def test_blocked_rows_match_dense_rows(cuda_device, weight_mode, point_mode):
    model, state, control, con, _, _ = models.box_scene(16, 61, cuda_device, boxes=8, sites=(2, 4))
    C = 96
    kw = dict(max_rigid_contact=C, contact_weight_mode=weight_mode, contact_point_mode=point_mode,
              fallback_tau_d=0.0)
    dense = SapContactJacobian(model, tree_blocked=False, **kw)
    blk = SapContactJacobian(model, tree_blocked=True, **kw)
    rd = dense.compute(state, con, control=control, dt=2e-3)
    rb = blk.compute(state, con, control=control, dt=2e-3)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(rb.contact_env_count.cpu(), rd.contact_env_count.cpu())
    np.testing.assert_allclose(blk.v_star.cpu(), dense.v_star.cpu(), rtol=1e-12, atol=1e-12)
    A = rd.dynamics_matrix_env.cpu().numpy().reshape(16, 8, 6, 8, 6)
    Tm = rb.tree_mass_env.cpu().numpy()
    for t in range(8):
        np.testing.assert_allclose(Tm[:, t], A[:, t, :, t, :], rtol=0, atol=1e-15 * np.abs(A).max())
    for name in ("contact_env_phi0", "contact_env_w_eff", "contact_env_mu", "contact_env_stiffness",
                 "contact_env_tau_d"):
        np.testing.assert_allclose(getattr(rb, name).cpu(), getattr(rd, name).cpu(), rtol=1e-13, atol=1e-15)
    # blocked rows scattered to dense columns == the dense rows
    Jd = rd.contact_env_jacobian.cpu().numpy()
    Jb = rb.contact_env_jacobian.cpu().numpy()
    ct = rb.contact_env_tree.cpu().numpy()
    cnt = np.minimum(rd.contact_env_count.cpu().numpy(), C)
    for e in range(16):
        for c in range(cnt[e]):
            row = np.zeros((3, 48))
            for s in range(2):
                if ct[e, c, s] >= 0:
                    row[:, 6 * ct[e, c, s]:6 * ct[e, c, s] + 6] += Jb[e, c, :, 6 * s:6 * s + 6]
            np.testing.assert_allclose(row, Jd[e, c], rtol=0, atol=1e-14)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_box_step_matches_oracle_pipeline(cuda_device, oracle, precision):
    """SolverSAP.step (tree-blocked) == C free motion and rows -> C oracle
    dense solve -> C integration, on worlds of 8 free boxes."""
    W, B = 24, 8
    model, state, control, con, host, hv = models.box_scene(W, 62, cuda_device, boxes=B, sites=(2, 4))
    C = 96
    solver = SolverSAP(model, max_rigid_contact=C, contact_preset_variant="drake", contact_tau_d=0.0,
                       tree_blocked=True, hessian_precision=precision)
    out = _clone(state)
    solver.step(state, out, control, con, 2e-3)
    torch.cuda.synchronize()
    hm = oracle.HostModel(hv["tpl"], hv["g"])
    dt = np.full(W, 2e-3)
    r = oracle.free_motion_contacts(hm, hv["q"], hv["qd"], host, dt, C, point_mode="contact_midpoint",
                                    weight_mode="diag_delassus")
    n = 6 * B
    prob = scenes.ContactProblemArrays(
        num_envs=W, dof_per_env=n, max_contacts=C, bodies_per_env=B,
        contact_count=np.minimum(r["count"], C).astype(np.int32), dynamics_matrix=r["A"], jacobian=r["jac"],
        phi0=r["phi0"], w_eff=r["w"], mu=r["mu"], stiffness=r["k"], tau_d=r["tau"], body0=r["body0"],
        body1=r["body1"], body_dof_start=np.tile(np.arange(B, dtype=np.int32) * 6, W),
        body_dof_count=np.full(W * B, 6, np.int32), v_star=r["v_star"].reshape(-1), v0=hv["qd"].reshape(-1), dt=dt)
    sol = oracle.solve(prob, "armijo_decay")
    assert np.all(sol["converged"] == 1)
    sr = solver.last_contact_solve_result
    gpu = {k: v.cpu().numpy() for k, v in dict(
        v=sr.v_flat, contact_gamma=sr.contact_gamma, contact_mode=sr.contact_mode, cost=sr.cost,
        converged=sr.converged_env).items()}
    if precision == "fp64":
        assert_parity(prob, gpu, sol)
    else:
        assert_parity(prob, gpu, sol, tight=1e-5, loose=1e-4, max_loose_frac=0.1)
    q_ref = oracle.integrate_positions(hm, hv["q"].reshape(-1), hv["qd"].reshape(-1), gpu["v"], dt, "sap_euler")
    np.testing.assert_allclose(out.joint_q.cpu().numpy(), q_ref, rtol=0, atol=1e-12)


def test_full_size_box_rollout_and_graph(cuda_device):
    """64 boxes per world (384 DOFs; the solver picks the tree-blocked layout
    by itself): 10 steps converge with finite states, and a CUDA graph of two
    steps replays the eager trajectory bit for bit."""
    model, state, control, con, _, _ = models.box_scene(32, 63, cuda_device)
    kw = dict(max_rigid_contact=512, contact_preset_variant="drake", hessian_precision="fp32")
    solver = SolverSAP(model, **kw)
    assert solver.contact_solve.tree_blocked
    a, b = _clone(state), _clone(state)
    for _ in range(5):
        solver.step(a, b, control, con, 2e-3)
        assert bool(solver.contact_solve.converged_env.all())
        solver.step(b, a, control, con, 2e-3)
        assert bool(solver.contact_solve.converged_env.all())
    assert torch.isfinite(a.joint_q).all() and torch.isfinite(a.joint_qd).all()
    eager_q = a.joint_q.clone()
    g_solver = SolverSAP(model, **kw)
    ga, gb = _clone(state), _clone(state)
    graph = g_solver.capture_steps(ga, gb, control, con, 2e-3, warmup=1)  # the warm-up advances two steps
    for _ in range(4):
        graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(ga.joint_q, eager_q)
    del graph
