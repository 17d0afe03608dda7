"""The learned warm start on the GPU: per-contact features and the impulse map
against numpy, the gamma0 start of the solve against the C oracle's (same
accept decisions, same answer), and the ablation that shows what the trained
network gains over the plain start at equal tolerance."""

import numpy as np
import pytest
import torch

from sap_warp_b200 import scenes
from sap_warp_b200._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device
from sap_warp_b200.warmstart import (FeatureNorm, LearnedWarmStart, WarmStartMLP, raw_features, residual_targets,
                                     solver_dataset, train)

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


def test_impulses_are_scaled_and_projected(cuda_device):
    prob = scenes.humanoid_contact_problem(32, seed=32)
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    norm = FeatureNorm.identity()
    norm.out_scale = np.array([0.5, 2.0, 3.0], np.float32)
    norm.out_shift = np.array([0.1, -0.2, 0.3], np.float32)
    ws = LearnedWarmStart(WarmStartMLP(cuda_device, seed=2), norm)
    t = problem_to_device(prob, cuda_device)
    gp = np.random.default_rng(1).normal(scale=0.01, size=(E, C, 3))
    g0 = ws.predict(num_envs=E, dof_per_env=n, max_contacts=C, gamma_prev=torch.as_tensor(gp).to(cuda_device),
                    **t).cpu().numpy()
    y = ws.buffers(E, C)["y"].cpu().numpy().astype(np.float64).reshape(E, C, 3)
    u = y * norm.out_scale.astype(np.float64) + norm.out_shift.astype(np.float64)
    g = gp + u / np.maximum(prob.w_eff, 1e-12)[..., None]
    g[..., 2] = np.maximum(g[..., 2], 0.0)
    tm = np.linalg.norm(g[..., :2], axis=-1)
    lim = prob.mu * g[..., 2]
    sc = np.where(tm > lim, np.where(tm > 0, lim / np.where(tm > 0, tm, 1.0), 0.0), 1.0)
    g[..., :2] *= sc[..., None]
    g[~(np.arange(C)[None, :] < prob.contact_count[:, None])] = 0.0
    np.testing.assert_allclose(g0, g, rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("variant", ["armijo_decay", "monotone_decay", "exact_root"])
def test_gamma0_start_matches_oracle(cuda_device, oracle, variant):
    """FP64 GPU and oracle take the same accept decisions on a gamma0 that is
    good in some worlds and bad in others, and reach the same answer."""
    prob = scenes.humanoid_contact_problem(64, seed=33)
    plain = oracle.solve(prob, variant)
    rng = np.random.default_rng(5)
    noise = np.where(np.arange(64)[:, None, None] % 3 == 0, 5.0, 0.05)
    gamma0 = plain["contact_gamma"][:, :prob.max_contacts] * (1.0 + noise * rng.normal(size=(64, prob.max_contacts, 3)))
    ref = oracle.solve(prob, variant, gamma0=gamma0)
    got = run(prob, cuda_device, variant, gamma0=torch.as_tensor(gamma0).to(cuda_device).contiguous())
    acc = ref["warm_start_accepted"]
    assert 0 < acc.sum() < 64
    np.testing.assert_array_equal(got["warm_start_accepted"], acc)
    v, vr = got["v"].reshape(64, -1), ref["v"].reshape(64, -1)
    err = np.abs(v - vr).max(1) / np.abs(vr).max(1)
    assert np.quantile(err, 0.95) <= 1e-6 and err.max() <= 1e-4, err.max()
    assert got["converged"].all()


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


def test_learned_start_reduces_newton_iterations(cuda_device, oracle):
    """Ablation: a network trained in-test on solver-generated contacts cuts
    the mean Newton iterations of held-out worlds against both plain starts
    (v0 and v*) at the same tolerance.  Accuracy is measured against a tightly
    converged FP64 oracle solution (rel. tol 1e-12): any start that stops at
    the reference tolerance lands within tolerance x conditioning of it, and
    the learned start must be as accurate as the plain ones."""
    train_probs = [scenes.humanoid_contact_problem(2048, seed=s) for s in (300, 301, 302)]
    raw, u = solver_dataset(train_probs, cuda_device)
    norm = FeatureNorm.from_data(raw.cpu().numpy(), residual_targets(raw, u).cpu().numpy())
    mlp = WarmStartMLP(cuda_device, seed=0)
    log = train(mlp, raw, u, norm, steps=1500, batch=8192, lr=2e-3, log_every=500)
    assert log[-1][1] < 0.5 * log[0][1], log
    ws = LearnedWarmStart(mlp, norm)

    prob = scenes.humanoid_contact_problem(1024, seed=303)
    E, n, C = prob.num_envs, prob.dof_per_env, prob.max_contacts
    t = problem_to_device(prob, cuda_device)
    gamma0 = ws.predict(num_envs=E, dof_per_env=n, max_contacts=C,
                        normal_up=torch.as_tensor(prob.normal_up).to(cuda_device), **t)
    tight = oracle.solve(prob, "armijo_decay", optimality_rel_tol=1e-12, cost_rel_tol=0.0, cost_abs_tol=0.0)
    vr = tight["v"].reshape(E, n)
    stats = {}
    for label, g0, v0, prec in (("plain_v0_fp64", None, None, "fp64"), ("plain_v0", None, None, "fp32"),
                                ("plain_vstar", None, t["v_star"], "fp32"), ("learned", gamma0, None, "fp32"),
                                ("learned_fp64", gamma0, None, "fp64")):
        tt = dict(t)
        if v0 is not None:
            tt["v0"] = v0
        buf = ContactSolveBuffers(E, n, C, cuda_device)
        contact_solve(**tt, buffers=buf, options=make_options("armijo_decay", hessian_precision=prec), gamma0=g0)
        torch.cuda.synchronize()
        v = buf.v.cpu().numpy().reshape(E, n)
        err = np.abs(v - vr).max(1) / np.abs(vr).max(1)
        stats[label] = dict(iters=buf.newton_iterations.double().mean().item(),
                            accepted=buf.warm_start_accepted.double().mean().item(),
                            converged=bool(buf.converged.all()), err98=float(np.quantile(err, 0.98)),
                            errmax=float(err.max()))
    print(stats)
    for label, st in stats.items():
        assert st["converged"], label
        assert st["errmax"] <= 1e-4, (label, st)
    assert stats["learned"]["err98"] <= max(1e-6, 2.0 * stats["plain_v0"]["err98"]), stats
    assert stats["learned"]["accepted"] > 0.5, stats
    assert stats["learned"]["iters"] < min(stats["plain_v0"]["iters"], stats["plain_vstar"]["iters"]), stats
