"""The dense solve's launch shape (resident CTAs per SM) on the GPU: the
occupancy bound, results independent of the shape, and SolverSAP's
autotuner timing the candidates on its first solve."""

import json

import numpy as np
import pytest
import torch

from sap_warp_b200 import _abi, models, scenes
from sap_warp_b200._lib import load
from sap_warp_b200._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SolverSAP

pytestmark = pytest.mark.gpu


def test_occupancy_bound(cuda_device):
    lib = load()
    fp32 = lib.sapb_contact_solve_occupancy(35, 32, _abi.SAPB_FP32, _abi.LINE_SEARCH_VARIANTS["armijo_decay"])
    fp64 = lib.sapb_contact_solve_occupancy(35, 32, _abi.SAPB_FP64, _abi.LINE_SEARCH_VARIANTS["armijo_decay"])
    assert 1 <= fp64 <= fp32 <= 8
    assert lib.sapb_contact_solve_occupancy(35, 32, _abi.SAPB_FP64, 99) == _abi.SAPB_ERR_INVALID_ARGUMENT


def test_results_do_not_depend_on_the_launch_shape(cuda_device):
    prob = scenes.humanoid_contact_problem(512, seed=81)
    t = problem_to_device(prob, cuda_device)
    out = []
    for k in (0, 1, 2):
        buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, cuda_device)
        contact_solve(**t, buffers=buf, options=make_options("armijo_decay", hessian_precision="fp32",
                                                             ctas_per_sm=k))
        torch.cuda.synchronize()
        out.append((buf.v.clone(), buf.newton_iterations.clone()))
    for v, it in out[1:]:
        assert torch.equal(v, out[0][0]) and torch.equal(it, out[0][1])


def test_solver_autotune_writes_its_choice(cuda_device, tmp_path):
    path = tmp_path / "tune.json"
    model, state, control, contacts, _ = models.rollout_scene("humanoid", 1024, 82, cuda_device)
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
              warm_start="previous_impulses")

    def run(**extra):
        solver = SolverSAP(model, **kw, **extra)
        a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        for _ in range(3):
            solver.step(a, b, control, contacts, 2e-3)
            a, b = b, a
        torch.cuda.synchronize()
        return a.joint_q.clone(), a.joint_qd.clone()

    q0, qd0 = run()
    q1, qd1 = run(autotune=str(path))
    assert torch.equal(q0, q1) and torch.equal(qd0, qd1)
    table = json.loads(path.read_text())
    assert len(table) == 1
    (key, entry), = table.items()
    assert key.startswith("n35-c32-fp32-armijo_decay-")
    occ = load().sapb_contact_solve_occupancy(35, 32, _abi.SAPB_FP32, _abi.LINE_SEARCH_VARIANTS["armijo_decay"])
    assert set(entry["ms"]) == {str(k) for k in range(1, occ + 1)}
    assert 1 <= entry["ctas_per_sm"] <= occ
    assert all(np.isfinite(float(v)) and float(v) > 0 for v in entry["ms"].values())


def test_tuning_after_the_first_step_keeps_the_answer(cuda_device, tmp_path):
    """Tuning on a later step (warm-start guess active, the guess being the
    output velocity): every timed solve starts from the same guess, and the
    step's answer equals an untuned run's bit for bit."""
    from sap_warp_b200.autotune import SolveAutotuner

    model, state, control, contacts, _ = models.rollout_scene("humanoid", 512, 83, cuda_device)
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32")

    def run(tune_at):
        solver = SolverSAP(model, **kw)
        a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        for k in range(4):
            if k == tune_at:
                solver.contact_solve.autotuner = SolveAutotuner(str(tmp_path / "late.json"))
            solver.step(a, b, control, contacts, 2e-3)
            a, b = b, a
        torch.cuda.synchronize()
        return a.joint_qd.clone(), solver.contact_solve.newton_iterations_env.clone()

    qd0, it0 = run(None)
    qd1, it1 = run(2)
    assert torch.equal(qd0, qd1) and torch.equal(it0, it1)
