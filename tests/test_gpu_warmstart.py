"""The learned warm start on the GPU: per-contact features and the impulse map
against numpy, the gamma0 start of the solve against the C oracle's (same
accept decisions, same answer), and the ablation that shows what the trained
network gains over the plain start at equal tolerance."""

import numpy as np
import pytest
import torch

from sap_warp_b200 import scenes
from sap_warp_b200._solve import ContactSolveBuffers, build_problem, contact_solve, make_options, problem_to_device
from sap_warp_b200.warmstart import (FeatureNorm, LearnedWarmStart, WarmStartMLP, raw_features, residual_targets,
                                     rollout_dataset, solver_dataset, train, unprojected_targets)

pytestmark = pytest.mark.gpu


def numpy_features(prob, gamma_prev=None, normal_up=None, tau_fallback=0.0):
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    vs = prob.v_star.reshape(E, n)
    vc = np.einsum("ecrj,ej->ecr", prob.jacobian, vs)
    live = np.arange(C)[None, :] < prob.contact_count[:, None]
    w = np.maximum(prob.w_eff, 1e-12)
    f = np.zeros((E, C, 12))
    f[..., 0] = prob.phi0
    f[..., 1:4] = vc
    f[..., 4] = 1.0 if normal_up is None else normal_up
    f[..., 5] = prob.mu
    f[..., 6] = np.log10(np.maximum(prob.stiffness, 1e-30))
    f[..., 7] = prob.tau_d if prob.tau_d is not None else tau_fallback
    f[..., 8] = prob.dt[:, None]
    if gamma_prev is not None:
        f[..., 9:12] = w[..., None] * gamma_prev
    f[~live] = 0.0
    return f.reshape(E * C, 12).astype(np.float32)


def run(prob, dev, variant="armijo_decay", gamma0=None, **kw):
    t = problem_to_device(prob, dev)
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
    contact_solve(**t, buffers=buf, options=make_options(variant, **kw), gamma0=gamma0)
    torch.cuda.synchronize()
    return {k: getattr(buf, k).cpu().numpy() for k in
            ("v", "contact_gamma", "newton_iterations", "converged", "warm_start_accepted", "cost")}


def test_features_match_numpy(cuda_device):
    prob = scenes.humanoid_contact_problem(48, seed=31)
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    rng = np.random.default_rng(0)
    gp = rng.normal(size=(E, C, 3))
    t = problem_to_device(prob, cuda_device)
    nu = torch.as_tensor(prob.normal_up).to(cuda_device)
    raw = raw_features(t, E, n, C, normal_up=nu, gamma_prev=torch.as_tensor(gp).to(cuda_device)).cpu().numpy()
    ref = numpy_features(prob, gp, prob.normal_up)
    np.testing.assert_allclose(raw, ref, rtol=2e-6, atol=1e-9)
    # normalised BF16 rows: the kernel and FeatureNorm.encode agree bit for bit
    norm = FeatureNorm.from_data(ref[ref[:, 5] > 0], np.ones((1, 3)))
    ws = LearnedWarmStart(WarmStartMLP(cuda_device, seed=0), norm)
    ws.predict(num_envs=E, dof_per_env=n, max_contacts=C, normal_up=nu, gamma_prev=torch.as_tensor(gp).to(cuda_device),
               **t)
    x = ws.buffers(E, C)["x"]
    enc = norm.encode(torch.from_numpy(raw).to(cuda_device))
    live = torch.from_numpy((np.arange(C)[None, :] < prob.contact_count[:, None]).reshape(-1)).to(cuda_device)
    torch.testing.assert_close(x[live], enc[live], rtol=0, atol=0)
    assert int((x[~live] != 0).sum()) == 0


def test_impulses_are_scaled_and_projected(cuda_device, oracle):
    """gamma0 = SAP's regularized projection of y0 = gamma_prev + u / w, u the
    de-standardised network output, checked against the oracle's projection
    of the equivalent contact velocity vc = vhat - R y0."""
    prob = scenes.humanoid_contact_problem(16, seed=32)
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    norm = FeatureNorm.identity()
    norm.out_scale = np.array([0.5, 2.0, 3.0], np.float32)
    norm.out_shift = np.array([0.1, -0.2, 0.3], np.float32)
    ws = LearnedWarmStart(WarmStartMLP(cuda_device, seed=2), norm)
    t = problem_to_device(prob, cuda_device)
    gp = np.random.default_rng(1).normal(scale=0.01, size=(E, C, 3))
    g0 = ws.predict(num_envs=E, dof_per_env=n, max_contacts=C, gamma_prev=torch.as_tensor(gp).to(cuda_device),
                    **t).cpu().numpy()
    yout = ws.buffers(E, C)["y"].cpu().numpy().astype(np.float64).reshape(E, C, 3)
    u = yout * norm.out_scale.astype(np.float64) + norm.out_shift.astype(np.float64)
    live = np.arange(C)[None, :] < prob.contact_count[:, None]
    for e in range(E):
        for c in range(C):
            if not live[e, c]:
                assert np.all(g0[e, c] == 0.0)
                continue
            w = max(prob.w_eff[e, c], 1e-12)
            y0 = gp[e, c] + u[e, c] / w
            tau = prob.tau_d[e, c]
            ref = oracle.project([0.0, 0.0, 0.0], prob.phi0[e, c], prob.w_eff[e, c], prob.mu[e, c],
                                 prob.stiffness[e, c], tau, dt=prob.dt[e])
            vhat = -prob.phi0[e, c] / (prob.dt[e] + tau)
            vc = [-ref["rt"] * y0[0], -ref["rt"] * y0[1], vhat - ref["rn"] * y0[2]]
            want = oracle.project(vc, prob.phi0[e, c], prob.w_eff[e, c], prob.mu[e, c], prob.stiffness[e, c], tau,
                                  dt=prob.dt[e])["gamma"]
            np.testing.assert_allclose(g0[e, c], want, rtol=1e-9, atol=1e-12 * max(1.0, np.abs(want).max()))


def test_unprojected_targets_project_to_the_solution(cuda_device):
    """Projecting the training targets y* (at the converged velocity) gives
    back the solve's impulses: the targets and the impulse map agree."""
    prob = scenes.humanoid_contact_problem(64, seed=35)
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    t = problem_to_device(prob, cuda_device)
    sol = run(prob, cuda_device, "armijo_decay")
    u = unprojected_targets(t, torch.as_tensor(sol["v"]).to(cuda_device), E, n, C)
    ws = LearnedWarmStart(WarmStartMLP(cuda_device, seed=0), FeatureNorm.identity())
    b = ws.buffers(E, C)
    P = build_problem(num_envs=E, dof_per_env=n, max_contacts=C, **t)
    from sap_warp_b200._lib import load
    import ctypes
    y = u.to(torch.float32).contiguous()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert load().sapb_warmstart_impulses(ctypes.byref(P), y.data_ptr(), None, None, ctypes.byref(ws.norm_struct),
                                          ctypes.byref(ws.solve_options), b["gamma0"].data_ptr(), s) == 0
    g = b["gamma0"].cpu().numpy()
    want = sol["contact_gamma"][:, :C]
    scale = np.abs(want).max()
    assert np.abs(g - want).max() <= 1e-5 * scale, np.abs(g - want).max() / scale


@pytest.mark.parametrize("variant,sets", [("armijo_decay", 1), ("monotone_decay", 1), ("exact_root", 1),
                                          ("armijo_decay", 2)])
def test_gamma0_start_matches_oracle(cuda_device, oracle, variant, sets):
    """FP64 GPU and oracle choose the same start among the plain one and the
    candidate impulse sets (good in some worlds, bad in others) and reach the
    same answer."""
    prob = scenes.humanoid_contact_problem(64, seed=33)
    plain = oracle.solve(prob, variant)
    rng = np.random.default_rng(5)
    cands = []
    for k in range(sets):
        # every third world: all sets bad; otherwise set k is the better one in alternate worlds
        e = np.arange(64)[:, None, None]
        noise = np.where(e % 3 == 0, 5.0, np.where((e + k) % 2 == 0, 0.02, 0.2))
        cands.append(plain["contact_gamma"][:, :prob.max_contacts] *
                     (1.0 + noise * rng.normal(size=(64, prob.max_contacts, 3))))
    gamma0 = np.stack(cands) if sets > 1 else cands[0]
    ref = oracle.solve(prob, variant, gamma0=gamma0)
    got = run(prob, cuda_device, variant, gamma0=torch.as_tensor(gamma0).to(cuda_device).contiguous())
    acc = ref["warm_start_accepted"]
    assert 0 < (acc > 0).sum() < 64
    if sets > 1:
        assert set(np.unique(acc)) >= {1, 2}
    np.testing.assert_array_equal(got["warm_start_accepted"], acc)
    v, vr = got["v"].reshape(64, -1), ref["v"].reshape(64, -1)
    err = np.abs(v - vr).max(1) / np.abs(vr).max(1)
    assert np.quantile(err, 0.95) <= 1e-6 and err.max() <= 1e-4, err.max()
    assert got["converged"].all()


def _start_velocity(prob, gamma):
    """v* + A^-1 J^T gamma per world (numpy, FP64), (E*n,)."""
    E, n = prob.num_envs, prob.dof_per_env
    vs = prob.v_star.reshape(E, n)
    out = np.empty((E, n))
    for e in range(E):
        c = int(min(prob.contact_count[e], prob.max_contacts))
        jt = prob.jacobian[e, :c].reshape(3 * c, n).T @ gamma[e, :c].reshape(-1) if c else np.zeros(n)
        out[e] = vs[e] + np.linalg.solve(prob.dynamics_matrix[e], jt)
    return out.reshape(-1)


@pytest.mark.parametrize("variant", ["armijo_decay", "monotone_decay"])
def test_velocity_candidates_match_the_impulse_candidates(cuda_device, oracle, variant):
    """A start velocity v* + A^-1 J^T gamma given as v_candidates, and the
    impulses split into a base velocity (gamma0_base) plus the rest (gamma0),
    choose the same starts as the oracle given gamma and reach the same
    answer; worlds whose remaining impulses are all zero start at the base
    without the factor (every third world here)."""
    prob = scenes.humanoid_contact_problem(64, seed=33)
    plain = oracle.solve(prob, variant)
    rng = np.random.default_rng(5)
    e = np.arange(64)[:, None, None]
    noise = np.where(e % 3 == 0, 5.0, np.where(e % 2 == 0, 0.02, 0.2))
    gamma = plain["contact_gamma"][:, :prob.max_contacts] * (1.0 + noise * rng.normal(size=(64, prob.max_contacts, 3)))
    ref = oracle.solve(prob, variant, gamma0=gamma)
    acc = ref["warm_start_accepted"]
    assert 0 < (acc > 0).sum() < 64
    dev = cuda_device
    vc = torch.as_tensor(_start_velocity(prob, gamma), device=dev).contiguous()
    split = np.where((e % 3 == 1), 0.0, 0.5) * gamma  # world e % 3 == 1: all in the base
    base = torch.as_tensor(_start_velocity(prob, gamma - split), device=dev).contiguous()
    for kw in ({"v_candidates": vc},
               {"gamma0": torch.as_tensor(split, device=dev).contiguous(), "gamma0_base": base}):
        t = problem_to_device(prob, dev)
        buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
        contact_solve(**t, buffers=buf, options=make_options(variant), **kw)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(buf.warm_start_accepted.cpu().numpy(), acc, err_msg=str(list(kw)))
        v, vr = buf.v.cpu().numpy().reshape(64, -1), ref["v"].reshape(64, -1)
        err = np.abs(v - vr).max(1) / np.abs(vr).max(1)
        assert np.quantile(err, 0.95) <= 1e-6 and err.max() <= 1e-4, err.max()
        assert bool(buf.converged.all())


def test_exact_impulses_start_at_the_solution(cuda_device, oracle):
    """gamma0 = gamma* gives v_L = v* + A^-1 J^T gamma* = the solution, so
    Newton stops at once."""
    prob = scenes.humanoid_contact_problem(64, seed=34)
    sol = oracle.solve(prob, "armijo_decay")
    g = torch.as_tensor(sol["contact_gamma"][:, :prob.max_contacts]).to(cuda_device).contiguous()
    for precision in ("fp64", "fp32"):
        got = run(prob, cuda_device, "armijo_decay", gamma0=g, hessian_precision=precision)
        assert got["warm_start_accepted"].all()
        assert got["newton_iterations"].max() <= (1 if precision == "fp64" else 2), precision
        assert got["converged"].all()


def test_learned_start_against_previous_impulses(cuda_device):
    """Ablation on rollouts whose contacts are regenerated from the pose every
    step (models.site_scene: contacts appear and vanish).  A network trained
    in-test on the new contacts of solver rollouts serves SolverSAP's learned
    start (carried impulses for contacts that existed last step, the
    network's prediction for new ones).  Against the same method without
    the network (previous impulses, new contacts starting at zero) it must
    not cost Newton iterations, and both cut the reference's
    previous-velocity start's iterations; every world converges at the same
    tolerance and the network predicts some contacts.  (Measured gain over
    previous impulses: under 1 %; the carried impulses give the reduction.)"""
    from sap_warp_b200 import models
    from sap_warp_b200.collision import ContactGenerator
    from sap_warp_b200.runtime import SapState
    from sap_warp_b200.solver import SolverSAP
    from sap_warp_b200.warmstart import site_rollout_dataset

    raw, u = site_rollout_dataset("humanoid", 1024, (400, 401), 30, cuda_device)
    assert raw.shape[0] > 500, raw.shape
    norm = FeatureNorm.from_data(raw.cpu().numpy(), residual_targets(raw, u).cpu().numpy())
    mlp = WarmStartMLP(cuda_device, seed=0)
    log = train(mlp, raw, u, norm, steps=1500, batch=4096, lr=2e-3, log_every=500)
    assert log[-1][1] < 0.8 * log[0][1], log
    ws = LearnedWarmStart(mlp, norm)
    stats = {}
    for mode in ("previous_velocity", "previous_impulses", "learned"):
        model, state, control, shapes, _ = models.site_scene("humanoid", 1024, 402, cuda_device)
        solver = SolverSAP(model, max_rigid_contact=32, hessian_precision="fp32", warm_start=mode,
                           learned_warm_start=ws if mode == "learned" else None)
        gen = ContactGenerator(shapes, solver.view, capacity=1024 * 32, gap=1.0e-3)
        other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                         body_f=state.body_f.clone())
        its, predicted = [], 0
        for k in range(30):
            solver.step(state, other, control, gen.generate(state.joint_q), 2.0e-3)
            cs = solver.contact_solve
            assert bool(cs.converged_env.all()), (mode, k)
            its.append(cs.newton_iterations_env.double().mean().item())
            if mode == "learned":
                cnt = solver.contact_jacobian.contact_env_count.clamp(max=32)
                live = torch.arange(32, device=cuda_device)[None, :] < cnt[:, None]
                predicted += int((live & (solver.has_history == 0)).sum())
            state, other = other, state
        stats[mode] = (float(np.mean(its[3:])), predicted)
        assert torch.isfinite(state.joint_q).all()
    print(stats)
    assert stats["learned"][1] > 0, stats  # the network served new contacts
    assert stats["previous_impulses"][0] < 0.8 * stats["previous_velocity"][0], stats
    assert stats["learned"][0] <= 1.02 * stats["previous_impulses"][0], stats


def test_skipping_the_plain_start_keeps_it_as_the_fallback(cuda_device, oracle):
    """skip_plain_start: the candidate start velocity is taken without
    evaluating the plain one; where the candidate's cost is not finite (NaN
    here, every fourth world) the plain start is the fallback and those
    worlds solve exactly as without candidates."""
    prob = scenes.humanoid_contact_problem(64, seed=35)
    sol = oracle.solve(prob, "armijo_decay")
    g = sol["contact_gamma"][:, :prob.max_contacts] * 1.01
    vc = _start_velocity(prob, g).reshape(64, -1)
    vc[::4] = np.nan
    t = problem_to_device(prob, cuda_device)
    plain = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, cuda_device)
    contact_solve(**t, buffers=plain, options=make_options("armijo_decay"))
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, cuda_device)
    opts = make_options("armijo_decay")
    opts.skip_plain_start = 1
    contact_solve(**t, buffers=buf, options=opts,
                  v_candidates=torch.as_tensor(vc.reshape(-1), device=cuda_device).contiguous())
    torch.cuda.synchronize()
    acc = buf.warm_start_accepted.cpu().numpy()
    assert np.all(acc[::4] == 0) and np.all(np.delete(acc, np.s_[::4]) == 1)
    v, vp = buf.v.cpu().numpy().reshape(64, -1), plain.v.cpu().numpy().reshape(64, -1)
    np.testing.assert_array_equal(v[::4], vp[::4])
    assert bool(buf.converged.all())
    # the candidate worlds start elsewhere than the oracle and stop at the
    # same tolerance: agreement to the conditioning times that tolerance
    err = np.abs(v - sol["v"].reshape(64, -1)).max(1) / np.abs(sol["v"].reshape(64, -1)).max(1)
    assert err.max() <= 1e-4, err.max()
