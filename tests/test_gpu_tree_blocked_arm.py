"""The tree-blocked layout on worlds of articulated trees of different sizes:
a 7-revolute arm among free boxes (trees of 7 and 6 DOFs in blocks of 7),
its gripper contacts coupling the arm's tree with a box's.  The blocked free
motion and rows against the dense ones on the GPU, the blocked solve against
the dense kernel, one step against the C oracle pipeline (free motion, rows,
dense solve, integration), the dense -> blocked gather with a tree map, a
world beyond the dense kernel's size (rollout and graph replay), and a tree
larger than its block refused and a non-finite world reported."""

import ctypes

import numpy as np
import pytest
import torch

from sap_warp_b200 import _abi, models, scenes
from sap_warp_b200._lib import SapbError, load
from sap_warp_b200._solve import dense_to_blocked
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SapContactJacobian, SolverSAP
from tests.test_gpu_contact_solve import assert_parity

pytestmark = pytest.mark.gpu

DT = 2e-3


def _clone(state):
    return SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                    body_f=state.body_f.clone())


def _trees(boxes):
    return np.concatenate([[0], 7 + 6 * np.arange(boxes + 1)]).astype(np.int64)


@pytest.mark.parametrize("weight_mode,point_mode", [("body_inertia", "witness_point"),
                                                    ("diag_delassus", "contact_midpoint")])
def test_arm_blocked_rows_match_dense_rows(cuda_device, weight_mode, point_mode):
    W, Bx, C = 12, 6, 96
    model, state, control, con, _, _ = models.box_scene(W, 71, cuda_device, boxes=Bx, sites=(2, 4), arm=True)
    kw = dict(max_rigid_contact=C, contact_weight_mode=weight_mode, contact_point_mode=point_mode,
              fallback_tau_d=0.0)
    dense = SapContactJacobian(model, tree_blocked=False, **kw)
    blk = SapContactJacobian(model, tree_blocked=True, **kw)
    assert blk.view.tree_block == 7 and blk.view.Aw == Bx + 1
    rd = dense.compute(state, con, control=control, dt=DT)
    rb = blk.compute(state, con, control=control, dt=DT)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(rb.contact_env_count.cpu(), rd.contact_env_count.cpu())
    np.testing.assert_allclose(blk.v_star.cpu(), dense.v_star.cpu(), rtol=1e-12, atol=1e-12)
    tds = _trees(Bx)
    n = int(tds[-1])
    A = rd.dynamics_matrix_env.cpu().numpy()
    Tm = rb.tree_mass_env.cpu().numpy()
    assert Tm.shape == (W, Bx + 1, 7, 7)
    for t in range(Bx + 1):
        s0, nt = int(tds[t]), int(tds[t + 1] - tds[t])
        np.testing.assert_allclose(Tm[:, t, :nt, :nt], A[:, s0:s0 + nt, s0:s0 + nt], rtol=0,
                                   atol=1e-15 * np.abs(A).max())
        pad = Tm[:, t, nt:, :].copy()
        ident = np.zeros_like(pad)
        for a in range(nt, 7):
            ident[:, a - nt, a] = 1.0
        np.testing.assert_array_equal(pad, ident)  # the identity in the padding
        np.testing.assert_array_equal(Tm[:, t, :nt, nt:], 0.0)
    # the off-tree blocks of the dense A are zero: A is block diagonal by tree
    mask = np.zeros((n, n), bool)
    for t in range(Bx + 1):
        mask[tds[t]:tds[t + 1], tds[t]:tds[t + 1]] = True
    assert np.all(A[:, ~mask] == 0.0)
    for name in ("contact_env_phi0", "contact_env_w_eff", "contact_env_mu", "contact_env_stiffness",
                 "contact_env_tau_d"):
        np.testing.assert_allclose(getattr(rb, name).cpu(), getattr(rd, name).cpu(), rtol=1e-13, atol=1e-15)
    Jd = rd.contact_env_jacobian.cpu().numpy()
    Jb = rb.contact_env_jacobian.cpu().numpy()
    ct = rb.contact_env_tree.cpu().numpy()
    cnt = np.minimum(rd.contact_env_count.cpu().numpy(), C)
    gripped = 0
    for e in range(W):
        for c in range(cnt[e]):
            row = np.zeros((3, n))
            for s in range(2):
                t = ct[e, c, s]
                if t >= 0:
                    nt = int(tds[t + 1] - tds[t])
                    row[:, tds[t]:tds[t] + nt] += Jb[e, c, :, 7 * s:7 * s + nt]
                    np.testing.assert_array_equal(Jb[e, c, :, 7 * s + nt:7 * s + 7], 0.0)
            np.testing.assert_allclose(row, Jd[e, c], rtol=0, atol=1e-14)
            gripped += int(0 in ct[e, c])
    assert gripped >= 2 * W  # every world's gripper contacts touch the arm's tree


@pytest.mark.parametrize("precision,warm", [("fp64", "previous_velocity"), ("fp32", "previous_velocity"),
                                            ("fp64", "learned")])
def test_arm_box_step_matches_oracle_pipeline(cuda_device, oracle, precision, warm):
    """SolverSAP.step (tree-blocked, trees of 7 and 6 DOFs) == C free motion
    and rows -> C oracle dense solve -> C integration; the learned start
    (the network's impulses as the blocked solve's candidate) changes the
    start, not the answer."""
    W, Bx, C = 16, 6, 96
    model, state, control, con, host, hv = models.box_scene(W, 72, cuda_device, boxes=Bx, sites=(2, 4), arm=True)
    solver = SolverSAP(model, max_rigid_contact=C, contact_preset_variant="drake", contact_tau_d=0.0,
                       tree_blocked=True, hessian_precision=precision, warm_start=warm)
    out = _clone(state)
    solver.step(state, out, control, con, DT)
    torch.cuda.synchronize()
    hm = oracle.HostModel(hv["tpl"], hv["g"])
    dt = np.full(W, DT)
    r = oracle.free_motion_contacts(hm, hv["q"], hv["qd"], host, dt, C, point_mode="contact_midpoint",
                                    weight_mode="diag_delassus")
    tds = _trees(Bx)
    n = int(tds[-1])
    bstart = np.concatenate([np.zeros(7, np.int32), tds[1:-1].astype(np.int32)])
    bcount = np.concatenate([np.full(7, 7, np.int32), np.full(Bx, 6, np.int32)])
    prob = scenes.ContactProblemArrays(
        num_envs=W, dof_per_env=n, max_contacts=C, bodies_per_env=7 + Bx,
        contact_count=np.minimum(r["count"], C).astype(np.int32), dynamics_matrix=r["A"], jacobian=r["jac"],
        phi0=r["phi0"], w_eff=r["w"], mu=r["mu"], stiffness=r["k"], tau_d=r["tau"], body0=r["body0"],
        body1=r["body1"], body_dof_start=np.tile(bstart, W), body_dof_count=np.tile(bcount, W),
        v_star=r["v_star"].reshape(-1), v0=hv["qd"].reshape(-1), dt=dt)
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


def test_arm_blocked_step_matches_dense_step(cuda_device):
    """Three steps of the tree-blocked and the dense SolverSAP on the same
    worlds (43 DOFs: both apply) agree to the solve's tolerance,
    previous-impulse starts."""
    W, Bx = 24, 6
    model, state, control, con, _, _ = models.box_scene(W, 73, cuda_device, boxes=Bx, sites=(2, 4), arm=True)
    kw = dict(max_rigid_contact=96, contact_preset_variant="drake", warm_start="previous_impulses")
    runs = {}
    for blocked in (False, True):
        solver = SolverSAP(model, tree_blocked=blocked, **kw)
        a, b = _clone(state), _clone(state)
        for _ in range(3):
            solver.step(a, b, control, con, DT)
            a, b = b, a
        torch.cuda.synchronize()
        assert bool(solver.contact_solve.converged_env.all())
        runs[blocked] = (a.joint_qd.cpu().numpy(), a.joint_q.cpu().numpy())
    # both solves stop at the same optimality tolerance (relative 1e-6 of the
    # gradient's scale) along different factorizations, so the three steps'
    # velocities agree to that tolerance, not to rounding
    scale = np.abs(runs[False][0]).max()
    np.testing.assert_allclose(runs[True][0], runs[False][0], rtol=0, atol=2e-5 * scale)
    np.testing.assert_allclose(runs[True][1], runs[False][1], rtol=0, atol=1e-8)


def test_learned_start_rollout_in_tree_blocked_layout(cuda_device):
    """An arm among 24 boxes (tree-blocked), 8 steps from the previous
    velocity and with the learned start (history impulses where a contact
    has them, the network's on new contacts): both converge, the learned
    candidate is taken, and the trajectories agree to the solve's
    tolerance."""
    model, state, control, con, _, _ = models.box_scene(48, 77, cuda_device, boxes=24, sites=(6, 9), arm=True)
    kw = dict(max_rigid_contact=256, contact_preset_variant="drake", hessian_precision="fp32")
    runs = {}
    for warm in ("previous_velocity", "learned"):
        solver = SolverSAP(model, warm_start=warm, **kw)
        assert solver.contact_solve.tree_blocked
        a, b = _clone(state), _clone(state)
        taken = []
        for _ in range(8):
            solver.step(a, b, control, con, DT)
            assert bool(solver.contact_solve.converged_env.all())
            taken.append(float(solver.contact_solve.warm_start_accepted_env.double().mean()))
            a, b = b, a
        torch.cuda.synchronize()
        runs[warm] = (np.mean(taken[2:]), a.joint_qd.clone())
    assert runs["learned"][0] > 0.5
    qv, ql = runs["previous_velocity"][1], runs["learned"][1]
    assert float((ql - qv).abs().max() / qv.abs().max()) < 1e-3


def test_dense_to_blocked_gather_with_tree_map(cuda_device):
    """sapb_dense_to_blocked with tree_dof_start gives the free-motion
    kernel's blocked outputs from its dense ones."""
    W, Bx, C = 8, 5, 80
    model, state, control, con, _, _ = models.box_scene(W, 74, cuda_device, boxes=Bx, sites=(2, 3), arm=True)
    kw = dict(max_rigid_contact=C, fallback_tau_d=0.0)
    dense = SapContactJacobian(model, tree_blocked=False, **kw)
    blk = SapContactJacobian(model, tree_blocked=True, **kw)
    rd = dense.compute(state, con, control=control, dt=DT)
    rb = blk.compute(state, con, control=control, dt=DT)
    tds = torch.as_tensor(_trees(Bx).astype(np.int32), device=cuda_device)
    n = int(tds[-1])
    v = blk.view
    arrays = dict(contact_count=rd.contact_env_count, dynamics_matrix=rd.dynamics_matrix_env.reshape(-1),
                  jacobian=rd.contact_env_jacobian.reshape(-1), phi0=rd.contact_env_phi0, w_eff=rd.contact_env_w_eff,
                  mu=rd.contact_env_mu, stiffness=rd.contact_env_stiffness, tau_d=rd.contact_env_tau_d,
                  body0=rd.contact_env_body0, body1=rd.contact_env_body1,
                  body_dof_start=v.body_dof_start, body_dof_count=v.body_dof_count,
                  v_star=dense.v_star, v0=state.joint_qd, dt=torch.full((W,), DT, dtype=torch.float64,
                                                                           device=cuda_device))
    g = dense_to_blocked(arrays, W, n, C, Bx + 1, 7, tree_dof_start=tds)
    torch.cuda.synchronize()
    cnt = np.minimum(rd.contact_env_count.cpu().numpy(), C)
    live = np.arange(C)[None, :] < cnt[:, None]
    np.testing.assert_allclose(g["tree_mass"].cpu(), rb.tree_mass_env.cpu(), rtol=0, atol=1e-12)
    # the gather keeps each side where the dense problem has it (a static
    # shape0 leaves side 0 empty) and the free motion moves a lone side to
    # side 0: the same rows once scattered back to the world's DOFs
    tn = _trees(Bx)

    def dense_rows(jac, tree):
        out = np.zeros((W, C, 3, n))
        for e in range(W):
            for c in range(cnt[e]):
                for s in range(2):
                    t = tree[e, c, s]
                    if t >= 0:
                        nt = int(tn[t + 1] - tn[t])
                        out[e, c, :, tn[t]:tn[t] + nt] += jac[e, c, :, 7 * s:7 * s + nt]
        return out

    ctg, ctb = g["contact_tree"].cpu().numpy(), rb.contact_env_tree.cpu().numpy()
    np.testing.assert_array_equal(np.sort(ctg[live], axis=-1), np.sort(ctb[live], axis=-1))
    np.testing.assert_allclose(dense_rows(g["jacobian"].cpu().numpy(), ctg),
                               dense_rows(rb.contact_env_jacobian.cpu().numpy(), ctb), rtol=0, atol=1e-14)


def test_large_arm_world_rollout_and_graph(cuda_device):
    """An arm among 24 boxes (151 DOFs, beyond the dense kernel; the solver
    picks the tree-blocked layout by itself): 10 steps converge with finite
    states, and a CUDA graph of two steps replays the eager trajectory bit
    for bit."""
    model, state, control, con, _, _ = models.box_scene(64, 75, cuda_device, boxes=24, sites=(6, 9), arm=True)
    kw = dict(max_rigid_contact=256, contact_preset_variant="drake", hessian_precision="fp32",
              warm_start="previous_impulses")
    solver = SolverSAP(model, **kw)
    assert solver.contact_solve.tree_blocked and solver.contact_solve.view.tree_block == 7
    a, b = _clone(state), _clone(state)
    for _ in range(5):
        solver.step(a, b, control, con, DT)
        assert bool(solver.contact_solve.converged_env.all())
        solver.step(b, a, control, con, DT)
        assert bool(solver.contact_solve.converged_env.all())
    assert torch.isfinite(a.joint_q).all() and torch.isfinite(a.joint_qd).all()
    eager_q = a.joint_q.clone()
    g_solver = SolverSAP(model, **kw)
    ga, gb = _clone(state), _clone(state)
    graph = g_solver.capture_steps(ga, gb, control, con, DT, warmup=1)  # the warm-up advances two steps
    for _ in range(4):
        graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(ga.joint_q, eager_q)
    del graph


def test_tree_beyond_block_rejected_and_nonfinite_world_reported(cuda_device):
    """Blocked outputs in blocks of 6 for worlds whose arm has 7 DOFs are
    refused before any launch; a world with NaN in v* gets the per-world
    status SAPB_WORLD_NOT_FINITE from the blocked solve (v = its start
    velocity, no iterations) while the other worlds solve normally."""
    W, Bx, C = 4, 3, 64
    model, state, control, con, _, _ = models.box_scene(W, 76, cuda_device, boxes=Bx, sites=(2, 2), arm=True)
    cj = SapContactJacobian(model, max_rigid_contact=C, tree_blocked=True, fallback_tau_d=0.0)
    cj.opts.tree_dofs = 6  # too small for the arm
    with pytest.raises(SapbError) as err:
        cj.compute(state, con, control=control, dt=DT)
    assert err.value.status == _abi.SAPB_ERR_UNSUPPORTED
    cj.opts.tree_dofs = 7
    r = cj.compute(state, con, control=control, dt=DT)
    n = 7 + 6 * Bx
    v_star = cj.v_star.clone()
    v_star[n + 3] = float("nan")  # world 1
    lib = load()
    P = _abi.BlockedProblem()
    P.num_envs, P.trees_per_env, P.tree_dofs, P.max_contacts = W, Bx + 1, 7, C
    tds = torch.as_tensor(_trees(Bx).astype(np.int32), device=cuda_device)
    P.tree_dof_start, P.dofs_per_world = tds.data_ptr(), n
    P.contact_count, P.tree_mass = r.contact_env_count.data_ptr(), r.tree_mass_env.data_ptr()
    P.jacobian, P.contact_tree = r.contact_env_jacobian.data_ptr(), r.contact_env_tree.data_ptr()
    P.phi0, P.w_eff, P.mu = r.contact_env_phi0.data_ptr(), r.contact_env_w_eff.data_ptr(), r.contact_env_mu.data_ptr()
    P.stiffness, P.tau_d = r.contact_env_stiffness.data_ptr(), r.contact_env_tau_d.data_ptr()
    v0 = state.joint_qd.clone()
    dt = torch.full((W,), DT, dtype=torch.float64, device=cuda_device)
    P.v_star, P.v0, P.dt = v_star.data_ptr(), v0.data_ptr(), dt.data_ptr()
    opts = _abi.SolveOptions()
    lib.sapb_solve_options_default(ctypes.byref(opts), _abi.SAPB_LS_ARMIJO_DECAY)
    v = torch.zeros(W * n, dtype=torch.float64, device=cuda_device)
    st = torch.full((W,), 7, dtype=torch.int32, device=cuda_device)
    it = torch.full((W,), -1, dtype=torch.int32, device=cuda_device)
    conv = torch.zeros(W, dtype=torch.int32, device=cuda_device)
    out = _abi.SolveOutputs()
    out.v, out.status, out.newton_iterations = v.data_ptr(), st.data_ptr(), it.data_ptr()
    out.converged = conv.data_ptr()
    ws = torch.zeros(lib.sapb_blocked_solve_workspace_size(W, Bx + 1, C), dtype=torch.uint8, device=cuda_device)
    rc = lib.sapb_blocked_contact_solve(ctypes.byref(P), ctypes.byref(opts), ctypes.byref(out), ws.data_ptr(),
                                        ws.numel(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == _abi.SAPB_OK
    torch.cuda.synchronize()
    assert st.tolist() == [0, _abi.SAPB_WORLD_NOT_FINITE, 0, 0]
    assert it[1].item() == 0 and conv[1].item() == 0
    assert bool(conv[[0, 2, 3]].all())
    torch.testing.assert_close(v[n:2 * n], v0[n:2 * n], rtol=0, atol=0)  # v = the start velocity
    assert torch.isfinite(v).all()


def test_driven_arm_blocked_step_matches_dense_step(cuda_device):
    """A position-controlled arm among boxes (drives and limits on its
    joints, models.with_drives): three steps of the tree-blocked solve, its
    drive / limit terms read through the tree map, agree with the dense
    solve's to the solve's tolerance."""
    W, Bx = 24, 6
    model, state, control, con, _, _ = models.box_scene(W, 79, cuda_device, boxes=Bx, sites=(2, 4), arm=True)
    model, control = models.with_drives(model, state, control, np.random.default_rng(5))
    kw = dict(max_rigid_contact=96, contact_preset_variant="drake", warm_start="previous_impulses")
    runs = {}
    for blocked in (False, True):
        solver = SolverSAP(model, tree_blocked=blocked, **kw)
        assert solver.view.has_pd and solver.view.has_limits
        a, b = _clone(state), _clone(state)
        for _ in range(3):
            solver.step(a, b, control, con, DT)
            a, b = b, a
        torch.cuda.synchronize()
        assert bool(solver.contact_solve.converged_env.all())
        runs[blocked] = (a.joint_qd.cpu().numpy(), a.joint_q.cpu().numpy())
    scale = np.abs(runs[False][0]).max()
    np.testing.assert_allclose(runs[True][0], runs[False][0], rtol=0, atol=2e-5 * scale)
    np.testing.assert_allclose(runs[True][1], runs[False][1], rtol=0, atol=1e-8)
    # the drives act: the arm's velocities differ from an undriven run
    free = SolverSAP(models.box_scene(W, 79, cuda_device, boxes=Bx, sites=(2, 4), arm=True)[0], tree_blocked=True,
                     **kw)
    a, b = _clone(state), _clone(state)
    for _ in range(3):
        free.step(a, b, control, con, DT)
        a, b = b, a
    torch.cuda.synchronize()
    arm = np.arange(W)[:, None] * (7 + 6 * Bx) + np.arange(7)[None, :]
    assert np.abs(a.joint_qd.cpu().numpy()[arm] - runs[True][0][arm]).max() > 1e-3 * scale
