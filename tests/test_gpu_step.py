"""Free motion, contact Jacobian, integration and the whole SolverSAP step on
the GPU against the numpy restatement (oracle/free_motion.py) feeding the C
oracle's contact solve."""

import numpy as np
import pytest
import torch

from oracle import free_motion as ofm
from sap_warp_b200 import models, scenes
from sap_warp_b200.runtime import SapControl, SapState
from sap_warp_b200.solver import SapContactJacobian, SolverSAP

pytestmark = pytest.mark.gpu

KINDS = ["humanoid", "quadruped", "slider", "arm_box", "joints"]


def build(kind, worlds, seed, per_world=(8, 24), random_child_frames=False, max_contacts=32):
    rng = np.random.default_rng(seed)
    tpl = models.world_template(kind, rng, random_child_frames=random_child_frames)
    g = models.replicate(tpl, worlds, rng)
    q = models.random_joint_q(tpl, rng, worlds)
    n = tpl["dofs_per_world"]
    qd = rng.normal(scale=0.5, size=(worlds, n))
    om = ofm.Model(dict(tpl, gravity=g["gravity"][0], shape_body_global=g["shape_body"],
                        shape_mu=g["shape_material_mu"], shape_ke=g["shape_material_ke"],
                        shape_tau=g["shape_material_tau"]))
    B = tpl["bodies_per_world"]
    dt = np.full(worlds, 2e-3)
    fm = ofm.free_motion(om, q, qd, np.zeros_like(qd), np.zeros((worlds, B, 6)), dt)
    counts = rng.integers(per_world[0], per_world[1] + 1, size=worlds)
    con = models.ground_contacts(rng, fm["pos"], fm["quat"], counts, bodies_from=B // 2, capacity=int(counts.sum()) + 7)
    return dict(tpl=tpl, g=g, q=q, qd=qd, om=om, fm=fm, con=con, dt=dt, max_contacts=max_contacts)


def gpu_state(case, dev):
    model = models.to_model(case["tpl"], case["g"], case["q"], dev)
    state = SapState(joint_q=torch.as_tensor(case["q"].reshape(-1), device=dev),
                     joint_qd=torch.as_tensor(case["qd"].reshape(-1), device=dev), body_q=model.body_q.clone(),
                     body_f=torch.zeros(model.body_count, 6, dtype=torch.float64, device=dev))
    control = SapControl(joint_f=torch.zeros(model.joint_dof_count, dtype=torch.float64, device=dev))
    return model, state, control


def _sorted_slots(phi0, count, *arrays):
    """Per-world slot permutation sorting live contacts by phi0 (the GPU
    scatter is atomic, so slot order is arrival order)."""
    out = []
    for e in range(phi0.shape[0]):
        c = min(int(count[e]), phi0.shape[1])
        order = np.argsort(phi0[e, :c], kind="stable")
        out.append(order)
    return out


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("weight_mode,point_mode", [("body_inertia", "witness_point"),
                                                    ("diag_delassus", "contact_midpoint")])
def test_free_motion_and_contact_rows(cuda_device, kind, weight_mode, point_mode):
    case = build(kind, 24, seed=hash(kind) % 1000, random_child_frames=(kind in ("slider", "arm_box")))
    model, state, control = gpu_state(case, cuda_device)
    cj = SapContactJacobian(model, max_rigid_contact=case["max_contacts"], contact_weight_mode=weight_mode,
                            contact_point_mode=point_mode, fallback_tau_d=0.0)
    contacts = models.contacts_to_torch(case["con"], cuda_device)
    res = cj.compute(state, contacts, control=control, dt=2e-3)
    torch.cuda.synchronize()
    fm = case["fm"]
    n = case["tpl"]["dofs_per_world"]
    A = res.dynamics_matrix_env.cpu().numpy()
    np.testing.assert_allclose(A, fm["A"], rtol=1e-10, atol=1e-12 * np.abs(fm["A"]).max())
    np.testing.assert_allclose(cj.v_star.cpu().numpy().reshape(-1, n), fm["v_star"], rtol=1e-9, atol=1e-10)
    ref = ofm.contact_jacobian(case["om"], fm, case["con"], case["max_contacts"], point_mode=point_mode,
                               weight_mode=weight_mode, fallback_tau=0.0)
    cnt = res.contact_env_count.cpu().numpy()
    np.testing.assert_array_equal(cnt, ref["count"])
    phi = res.contact_env_phi0.cpu().numpy()
    J = res.contact_env_jacobian.cpu().numpy()
    got = dict(jac=J, phi0=phi, mu=res.contact_env_mu.cpu().numpy(), k=res.contact_env_stiffness.cpu().numpy(),
               tau=res.contact_env_tau_d.cpu().numpy(), w=res.contact_env_w_eff.cpu().numpy(),
               body1=res.contact_env_body1.cpu().numpy())
    g_order = _sorted_slots(phi, cnt)
    r_order = _sorted_slots(ref["phi0"], ref["count"])
    for e in range(len(cnt)):
        a, b = g_order[e], r_order[e]
        for key in ("phi0", "mu", "k", "tau", "w"):
            np.testing.assert_allclose(got[key][e, a], ref[key][e, b], rtol=1e-9, atol=1e-14, err_msg=key)
        np.testing.assert_array_equal(got["body1"][e, a], ref["body1"][e, b])
        np.testing.assert_allclose(got["jac"][e, a], ref["jac"][e, b], rtol=1e-9, atol=1e-11)


def test_factor_and_free_motion_contact_velocities(cuda_device):
    """The optional outputs for candidate starts: the LDL^T factor of A
    (L D L^T reconstructs A) and vc* = J_c v* per live slot."""
    case = build("humanoid", 16, seed=12)
    model, state, control = gpu_state(case, cuda_device)
    cj = SapContactJacobian(model, max_rigid_contact=case["max_contacts"])
    cj.keep_dynamics_factor()
    res = cj.compute(state, models.contacts_to_torch(case["con"], cuda_device), control=control, dt=2e-3)
    torch.cuda.synchronize()
    A = res.dynamics_matrix_env.cpu().numpy()
    F = res.dynamics_factor_env.cpu().numpy()
    n = A.shape[1]
    for e in range(A.shape[0]):
        d = np.diag(F[e]).copy()
        L = np.tril(F[e], -1) / d[None, :] + np.eye(n)
        np.testing.assert_allclose(L @ np.diag(d) @ L.T, A[e], rtol=1e-10, atol=1e-10 * np.abs(A[e]).max())
    J = res.contact_env_jacobian.cpu().numpy()
    vs = cj.v_star.cpu().numpy().reshape(-1, n)
    vc = cj.contact_env_vc_star.cpu().numpy()
    cnt = np.minimum(res.contact_env_count.cpu().numpy(), case["max_contacts"])
    want = np.einsum("ecrj,ej->ecr", J, vs)
    for e in range(len(cnt)):
        np.testing.assert_allclose(vc[e, :cnt[e]], want[e, :cnt[e]], rtol=1e-12, atol=1e-12)


def test_truncation_counts(cuda_device):
    case = build("quadruped", 8, seed=5, per_world=(20, 40), max_contacts=16)
    model, state, control = gpu_state(case, cuda_device)
    cj = SapContactJacobian(model, max_rigid_contact=16)
    cj.compute(state, models.contacts_to_torch(case["con"], cuda_device), control=control, dt=2e-3)
    torch.cuda.synchronize()
    ref = ofm.contact_jacobian(case["om"], case["fm"], case["con"], 16)
    np.testing.assert_array_equal(cj.contact_env_count.cpu().numpy(), ref["count"])
    assert int(cj.truncated.item()) == ref["truncated"] > 0


@pytest.mark.parametrize("mode", ["sap_euler", "midpoint"])
@pytest.mark.parametrize("kind", ["humanoid", "joints"])
def test_full_step_matches_oracle_pipeline(cuda_device, oracle, mode, kind):
    """SolverSAP.step == numpy free motion + contact rows -> C oracle solve ->
    numpy integration, for a humanoid batch and a batch of chains through
    every mobilizer kind (ball, distance, D6 with 1-3 rotation / translation
    axes; drake-like preset, FP64)."""
    case = build(kind, 32, seed=41, random_child_frames=True)
    model, state, control = gpu_state(case, cuda_device)
    solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", position_integration=mode,
                       contact_tau_d=0.0)
    out = SapState(joint_q=torch.zeros_like(state.joint_q), joint_qd=torch.zeros_like(state.joint_qd),
                   body_q=state.body_q.clone(), body_f=torch.zeros_like(state.body_f))
    solver.step(state, out, control, models.contacts_to_torch(case["con"], cuda_device), 2e-3)
    torch.cuda.synchronize()
    fm = case["fm"]
    n = case["tpl"]["dofs_per_world"]
    W = 32
    ref = ofm.contact_jacobian(case["om"], fm, case["con"], 32, point_mode="contact_midpoint",
                               weight_mode="diag_delassus", fallback_tau=0.0)
    prob = scenes.ContactProblemArrays(
        num_envs=W, dof_per_env=n, max_contacts=32, bodies_per_env=case["tpl"]["bodies_per_world"],
        contact_count=ref["count"].astype(np.int32), dynamics_matrix=fm["A"], jacobian=ref["jac"], phi0=ref["phi0"],
        w_eff=ref["w"], mu=ref["mu"], stiffness=ref["k"], tau_d=ref["tau"], body0=ref["body0"], body1=ref["body1"],
        body_dof_start=np.zeros(W * case["tpl"]["bodies_per_world"], np.int32),
        body_dof_count=np.full(W * case["tpl"]["bodies_per_world"], n, np.int32),
        v_star=fm["v_star"].reshape(-1), v0=case["qd"].reshape(-1), dt=case["dt"])
    sol = oracle.solve(prob, "armijo_decay")
    v_ref = sol["v"].reshape(W, n)
    v_gpu = out.joint_qd.cpu().numpy().reshape(W, n)
    err = np.abs(v_gpu - v_ref).max(1) / np.abs(v_ref).max(1)
    assert np.quantile(err, 0.95) <= 1e-6 and err.max() <= 1e-4, err.max()
    q_ref = ofm.integrate(case["om"], case["q"], case["qd"], v_ref, case["dt"], mode)
    q_gpu = out.joint_q.cpu().numpy().reshape(W, -1)
    np.testing.assert_allclose(q_gpu, q_ref, rtol=0, atol=1e-9)


def test_multi_step_rollout_is_stable(cuda_device):
    """100 steps of a quadruped batch standing on the ground: finite states,
    every world converges every step within a few Newton iterations (the warm
    start is the previous solution, which is also the next step's v0)."""
    case = build("quadruped", 64, seed=9)
    model, state, control = gpu_state(case, cuda_device)
    solver = SolverSAP(model, max_rigid_contact=16, contact_tau_d=0.005)
    other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
    con = models.contacts_to_torch(case["con"], cuda_device)
    iters = []
    for k in range(100):
        solver.step(state, other, control, con, 2e-3)
        iters.append(solver.contact_solve.newton_iterations_env.max().item())
        assert bool(solver.contact_solve.converged_env.all())
        state, other = other, state
    torch.cuda.synchronize()
    assert torch.isfinite(state.joint_q).all() and torch.isfinite(state.joint_qd).all()
    assert max(iters) <= 20, iters
