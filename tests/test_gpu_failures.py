"""Failure detection on the GPU without a GPU fault.

- A bounded mbarrier wait of the MLP kernels runs out (the test hook drops
  each CTA's first commit, so nothing can complete the wait): the kernel sets
  the timeout flag and exits, sapb_mlp_error reports SAPB_ERR_TIMEOUT, and the
  next launch on the same context computes the right answer.
- Host-made bad inputs to the contact solve: a NaN / Inf in A, J, phi0 or v*
  gives the world SAPB_WORLD_NOT_FINITE (not solved, v = its start velocity,
  no iterations), a Hessian that is not SPD gives SAPB_WORLD_NOT_SPD (the
  Newton loop stops at once); every other world's answer is the one a clean
  run gives, bit for bit, and nothing waits or hangs.
- A zero-mass body in a stepped model: that world's free motion has a
  singular mass matrix, its solve reports SAPB_WORLD_NOT_FINITE, the other
  worlds step exactly as in a clean model.
"""

import ctypes

import numpy as np
import pytest
import torch

from sap_warp_b200 import _abi, models, scenes
from sap_warp_b200._lib import load
from sap_warp_b200._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SolverSAP
from sap_warp_b200.warmstart import WarmStartMLP

pytestmark = pytest.mark.gpu


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_mlp_wait_runs_out_and_the_context_stays_usable(cuda_device):
    lib = load()
    mlp = WarmStartMLP(cuda_device, seed=3)
    rows = 1000
    g = torch.Generator(device="cpu").manual_seed(5)
    x = torch.randn(rows, 16, generator=g).to(torch.bfloat16).view(torch.int16).to(cuda_device)
    y_ref = torch.zeros(rows, 3, dtype=torch.float32, device=cuda_device)
    mlp.forward(x, y_ref)
    assert lib.sapb_mlp_error(_stream()) == _abi.SAPB_OK
    y = torch.full((rows, 3), 7.0, dtype=torch.float32, device=cuda_device)
    try:
        assert lib.sapb_mlp_test_hooks(64, 1) == _abi.SAPB_OK
        mlp.forward(x, y)
        assert lib.sapb_mlp_error(_stream()) == _abi.SAPB_ERR_TIMEOUT
    finally:
        assert lib.sapb_mlp_test_hooks(0, 0) == _abi.SAPB_OK
    # the flag was cleared by the read; the context still runs the network
    assert lib.sapb_mlp_error(_stream()) == _abi.SAPB_OK
    mlp.forward(x, y)
    torch.cuda.synchronize()
    assert torch.equal(y, y_ref)
    assert lib.sapb_mlp_error(_stream()) == _abi.SAPB_OK
    assert lib.sapb_mlp_test_hooks(-1, 0) == _abi.SAPB_ERR_INVALID_ARGUMENT


def _solve(prob, dev, prec="fp64"):
    t = problem_to_device(prob, dev)
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
    contact_solve(**t, buffers=buf, options=make_options("armijo_decay", hessian_precision=prec,
                                                         linear_solve_precision=prec))
    torch.cuda.synchronize()
    return {k: getattr(buf, k).cpu().numpy() for k in
            ("v", "contact_gamma", "newton_iterations", "converged", "status")}


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_bad_inputs_give_per_world_statuses(cuda_device, prec):
    prob = scenes.humanoid_contact_problem(64, seed=91)
    n = prob.dof_per_env
    clean = _solve(prob, cuda_device, prec)
    bad = scenes.humanoid_contact_problem(64, seed=91)
    assert np.all(bad.contact_count[[3, 5, 7, 9, 11]] > 0)
    bad.dynamics_matrix[3, 0, 0] = np.nan
    bad.jacobian[5, 0, 2, 4] = np.inf
    bad.phi0[7, 0] = np.nan
    bad.v_star.reshape(-1, n)[9, 2] = -np.inf
    bad.dynamics_matrix[11, 0, 0] = -1.0e6  # H = A + J^T G J + ... is not SPD
    out = _solve(bad, cuda_device, prec)
    for e in (3, 5, 7, 9):
        assert out["status"][e] == _abi.SAPB_WORLD_NOT_FINITE, (e, out["status"][e])
        assert out["converged"][e] == 0 and out["newton_iterations"][e] == 0
        np.testing.assert_array_equal(out["v"].reshape(-1, n)[e], bad.v0.reshape(-1, n)[e])
        assert np.all(out["contact_gamma"][e] == 0.0)
    assert out["status"][11] == _abi.SAPB_WORLD_NOT_SPD
    assert out["converged"][11] == 0 and out["newton_iterations"][11] <= 1
    others = np.setdiff1d(np.arange(prob.num_envs), [3, 5, 7, 9, 11])
    np.testing.assert_array_equal(out["v"].reshape(-1, n)[others], clean["v"].reshape(-1, n)[others])
    np.testing.assert_array_equal(out["status"][others], clean["status"][others])
    assert np.all(clean["status"] == 0) and np.all(clean["converged"] == 1)


def test_zero_mass_body_is_reported_not_propagated(cuda_device):
    W = 8
    model, state, control, contacts, _ = models.rollout_scene("humanoid", W, 92, cuda_device)
    B = model.body_count // W

    def run(m):
        solver = SolverSAP(m, max_rigid_contact=32, contact_preset_variant="drake")
        a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        solver.step(a, b, control, contacts, 2.0e-3)
        torch.cuda.synchronize()
        return b, solver.contact_solve.ls_status.cpu().numpy(), solver.contact_solve.converged_env.cpu().numpy()

    clean_state, clean_status, _ = run(model)
    leaf = 2 * B + B - 1  # the last body of world 2 (a leaf of its serial chain)
    n = model.joint_dof_count // W
    mass, inertia, arm = model.body_mass.clone(), model.body_inertia.clone(), model.joint_armature.clone()
    model.body_mass[leaf] = 0.0
    model.body_inertia[leaf] = 0.0
    model.joint_armature[2 * n:3 * n] = 0.0  # no armature either: the leaf's DOF has a zero mass-matrix row
    try:
        out_state, status, conv = run(model)
    finally:
        model.body_mass.copy_(mass)
        model.body_inertia.copy_(inertia)
        model.joint_armature.copy_(arm)
    assert status[2] == _abi.SAPB_WORLD_NOT_FINITE and conv[2] == 0
    nq = model.joint_coord_count // W
    keep = [e for e in range(W) if e != 2]
    qd, qd0 = out_state.joint_qd.reshape(W, n), clean_state.joint_qd.reshape(W, n)
    q, q0 = out_state.joint_q.reshape(W, nq), clean_state.joint_q.reshape(W, nq)
    assert torch.equal(qd[keep], qd0[keep]) and torch.equal(q[keep], q0[keep])
    assert bool(torch.isfinite(qd[2]).all() and torch.isfinite(q[2]).all())
