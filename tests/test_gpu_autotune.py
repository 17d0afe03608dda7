"""The dense solve's launch shape (resident CTAs per SM), LDL^T block width
and threads per world on the GPU: the occupancy bound, results independent
of the CTA count (bit for bit), of the block width and of the 256-thread
kernel (to the solve's tolerance), and SolverSAP's autotuner timing the
candidates on its first solve."""

import ctypes
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
    armijo = _abi.LINE_SEARCH_VARIANTS["armijo_decay"]
    assert lib.sapb_contact_solve_occupancy_threads(35, 32, _abi.SAPB_FP32, armijo, 128) == fp32
    wide = lib.sapb_contact_solve_occupancy_threads(35, 32, _abi.SAPB_FP32, armijo, 256)
    assert 1 <= wide <= fp32
    assert lib.sapb_contact_solve_occupancy_threads(35, 32, _abi.SAPB_FP32, armijo, 64) == \
        _abi.SAPB_ERR_INVALID_ARGUMENT


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
    q2, qd2 = run(autotune=str(path))  # the saved choice, no timing
    assert torch.equal(q1, q2) and torch.equal(qd1, qd2)
    scale = float(qd0.abs().max())
    assert float((qd1 - qd0).abs().max()) <= 1e-6 * scale  # a different block width: same tolerance
    table = json.loads(path.read_text())
    assert len(table) == 1
    (key, entry), = table.items()
    assert key.startswith("n35-c32-fp32-armijo_decay-")
    occ = load().sapb_contact_solve_occupancy(35, 32, _abi.SAPB_FP32, _abi.LINE_SEARCH_VARIANTS["armijo_decay"])
    widths = (ctypes.c_int32 * 8)()
    nw = load().sapb_contact_solve_ldlt_blocks(35, widths, 8)
    assert nw >= 2 and widths[0] == 5
    armijo = _abi.LINE_SEARCH_VARIANTS["armijo_decay"]
    occ_wide = load().sapb_contact_solve_occupancy_threads(35, 32, _abi.SAPB_FP32, armijo, 256)
    gw = (ctypes.c_int32 * 8)()
    load().sapb_contact_solve_ldlt_blocks(1, gw, 8)
    assert set(entry["ms"]) == ({f"{k},{widths[b]},128" for b in range(nw) for k in range(1, occ + 1)}
                                | {f"{k},{gw[0]},256" for k in range(1, occ_wide + 1)})
    k, b, nt = entry["choice"]
    assert entry["ctas_per_sm"] == k and ((nt == 128 and 1 <= k <= occ and b in list(widths)[:nw])
                                          or (nt == 256 and 1 <= k <= occ_wide and b == gw[0]))
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

    qd1, it1 = run(2)  # tunes on step 2 (and saves its choice)
    qd0, it0 = run(2)  # step 2 takes the saved choice without timing
    assert torch.equal(qd0, qd1) and torch.equal(it0, it1)


def test_every_ldlt_block_width_reaches_the_tolerance(cuda_device, oracle):
    """Each LDL^T block width the kernel is built with solves the humanoid
    batch to the same tolerance: the answers agree with the FP64 oracle
    like the default width's."""
    prob = scenes.humanoid_contact_problem(256, seed=84)
    ref = oracle.solve(prob, "armijo_decay")
    t = problem_to_device(prob, cuda_device)
    widths = (ctypes.c_int32 * 8)()
    nw = load().sapb_contact_solve_ldlt_blocks(35, widths, 8)
    assert load().sapb_contact_solve_ldlt_blocks(36, widths, 8) >= 1 and widths[0] >= 1
    nw = load().sapb_contact_solve_ldlt_blocks(35, widths, 8)
    for prec in ("fp64", "fp32"):
        for b in list(widths)[:nw]:
            buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, cuda_device)
            contact_solve(**t, buffers=buf, options=make_options("armijo_decay", hessian_precision=prec,
                                                                 linear_solve_precision=prec, ldlt_block=b))
            torch.cuda.synchronize()
            assert bool(buf.converged.all()), (prec, b)
            n = prob.dof_per_env
            err = np.abs(buf.v.cpu().numpy() - ref["v"]).reshape(-1, n).max(1) / np.abs(ref["v"]).reshape(-1, n).max(1)
            assert np.quantile(err, 0.98) <= 1e-6 and err.max() <= 1e-4, (prec, b, err.max())


@pytest.mark.parametrize("kind", ["humanoid", "mixed"])
def test_wide_kernel_matches_the_oracle(cuda_device, oracle, kind):
    """The 256-thread runtime-size kernel (threads_per_cta = 256) solves to
    the same tolerance as the default kernel: against the FP64 oracle on the
    humanoid batch and on the uneven batch with per-world DOF counts, in both
    precisions; CTA counts do not change a bit."""
    if kind == "humanoid":
        prob = scenes.humanoid_contact_problem(256, seed=85)
        gpu_prob, extra = prob, {}
    else:
        prob, _ = scenes.mixed_contact_problem(384, seed=86)  # padded: the oracle's input
        gpu_prob = scenes.compact_problem(prob)
        extra = {"dof_count": torch.as_tensor(gpu_prob.dofs_active, dtype=torch.int32, device=cuda_device)}
    ref = oracle.solve(prob, "armijo_decay")
    t = problem_to_device(gpu_prob, cuda_device)
    n = prob.dof_per_env
    for prec in ("fp64", "fp32"):
        outs = []
        for k in (0, 1):
            buf = ContactSolveBuffers(prob.num_envs, n, prob.max_contacts, cuda_device)
            contact_solve(**t, **extra, buffers=buf, options=make_options(
                "armijo_decay", hessian_precision=prec, linear_solve_precision=prec, threads_per_cta=256,
                ctas_per_sm=k))
            torch.cuda.synchronize()
            outs.append(buf.v.clone())
            assert bool(buf.converged.all()), (kind, prec)
        assert torch.equal(outs[0], outs[1])
        got = outs[0].cpu().numpy().reshape(-1, n)
        want = ref["v"].reshape(-1, n)
        err = np.abs(got - want).max(1) / np.maximum(np.abs(want).max(1), 1e-30)
        assert np.quantile(err, 0.98) <= 1e-6 and err.max() <= 1e-4, (kind, prec, err.max())
