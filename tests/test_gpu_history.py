"""Contact history: impulses carried across steps by contact identity
(sapb_contact_history_update through the C ABI), the site scene's
regenerated contacts against the numpy restatement of contact generation,
and rollouts whose contacts appear and vanish."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import boundary as ob
from oracle import contacts as oc
from sap_warp_b200 import _abi, models
from sap_warp_b200._lib import check, load
from sap_warp_b200.collision import ContactGenerator
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SolverSAP, _ModelView

pytestmark = pytest.mark.gpu


class _Hist:
    def __init__(self, W, C, dev, order=1):
        z = lambda *s, dt=torch.float64: torch.zeros(*s, dtype=dt, device=dev)
        self.W, self.C, self.order = W, C, order
        self.key_shape, self.key_point, self.key_count = z(W, C, 2, dt=torch.int32), z(W, C, 3), z(W, dt=torch.int32)
        self.gamma_hist, self.has = z(W, C, 3), z(W, C, dt=torch.int32)
        self.gamma_older, self.gamma_start = z(W, C, 3), z(W, C, 3)

    def update(self, counts, source, s0, s1, p1, gamma_prev):
        H = _abi.ContactHistory()
        H.num_envs, H.max_contacts, H.num_flat = self.W, self.C, int(s0.numel())
        H.contact_count, H.contact_source = counts.data_ptr(), source.data_ptr()
        H.flat_shape0, H.flat_shape1, H.flat_point1 = s0.data_ptr(), s1.data_ptr(), p1.data_ptr()
        H.key_shape, H.key_point, H.key_count = (self.key_shape.data_ptr(), self.key_point.data_ptr(),
                                                 self.key_count.data_ptr())
        H.gamma_prev, H.gamma_hist, H.has_history = gamma_prev.data_ptr(), self.gamma_hist.data_ptr(), \
            self.has.data_ptr()
        H.order, H.gamma_older, H.gamma_start = self.order, self.gamma_older.data_ptr(), self.gamma_start.data_ptr()
        check(load().sapb_contact_history_update(ctypes.byref(H), None), "sapb_contact_history_update")
        torch.cuda.synchronize()


def _flat(dev, worlds):
    """Flat arrays of per-world contact lists [(shape0, shape1, point1)], and
    the slot -> flat index map."""
    C = 8
    s0, s1, p1, src, counts = [], [], [], np.full((len(worlds), C), -1, np.int32), []
    for w, lst in enumerate(worlds):
        for k, (a, b, p) in enumerate(lst):
            src[w, k] = len(s0)
            s0.append(a)
            s1.append(b)
            p1.append(p)
        counts.append(len(lst))
    t = lambda a, dt: torch.as_tensor(np.asarray(a), dtype=dt, device=dev)
    return (t(counts, torch.int32), t(src, torch.int32), t(s0, torch.int32), t(s1, torch.int32),
            t(np.asarray(p1, np.float64).reshape(-1, 3), torch.float64))


def test_history_follows_contacts_across_slot_shifts(cuda_device):
    h = _Hist(2, 8, cuda_device)
    g_none = torch.zeros(2, 8, 3, dtype=torch.float64, device=cuda_device)
    prev = [[(1, 10, (0, 0, 0)), (1, 11, (1, 0, 0)), (1, 12, (2, 0, 0)), (1, 13, (3, 0, 0))],
            [(2, 20, (0, 0, 0)), (2, 20, (1, 0, 0))]]
    h.update(*_flat(cuda_device, prev), g_none)
    assert int(h.has.sum()) == 0  # nothing before the first step
    gamma_prev = torch.arange(2 * 8 * 3, dtype=torch.float64, device=cuda_device).reshape(2, 8, 3) + 1.0
    # world 0: contact (1, 11) vanished, (1, 14) is new; world 1: the pair's two
    # contacts come in the other order and moved by a millimetre
    cur = [[(1, 10, (0, 0, 0)), (1, 12, (2, 0, 0)), (1, 13, (3, 0, 0)), (1, 14, (4, 0, 0))],
           [(2, 20, (1, 0, 1e-3)), (2, 20, (0, 0, 1e-3))]]
    h.update(*_flat(cuda_device, cur), gamma_prev)
    gh, has = h.gamma_hist.cpu().numpy(), h.has.cpu().numpy()
    gp = gamma_prev.cpu().numpy()
    np.testing.assert_array_equal(has[0, :5], [1, 1, 1, 0, 0])
    np.testing.assert_array_equal(gh[0, 0], gp[0, 0])
    np.testing.assert_array_equal(gh[0, 1], gp[0, 2])
    np.testing.assert_array_equal(gh[0, 2], gp[0, 3])
    assert np.all(gh[0, 3:] == 0.0)
    np.testing.assert_array_equal(has[1, :3], [1, 1, 0])
    np.testing.assert_array_equal(gh[1, 0], gp[1, 1])
    np.testing.assert_array_equal(gh[1, 1], gp[1, 0])
    np.testing.assert_array_equal(h.key_count.cpu().numpy(), [4, 2])


@pytest.mark.parametrize("order", [1, 2, 3])
def test_start_impulses_extrapolate_each_contacts_history(cuda_device, order):
    """Three solves' impulses along each contact's identity, through slot
    shifts: the start is the carried impulse (1 known), 2 g1 - g2 (2 known),
    3 g1 - 3 g2 + g3 (3 known), capped at the order; a contact that vanished
    for a step starts its history again; new contacts start at zero."""
    h = _Hist(1, 8, cuda_device, order=order)
    A, B, Cc, D = (1, 10, (0, 0, 0)), (1, 11, (1, 0, 0)), (1, 12, (2, 0, 0)), (1, 13, (3, 0, 0))
    # the contact sets of steps 0..3 (slots follow list order)
    steps = [[A, B, Cc], [D, A, B, Cc], [A, Cc, D], [B, A, Cc, D]]
    rng = np.random.default_rng(order)
    sol = {}  # contact -> list of its solves' impulses, most recent last
    gamma_prev = torch.zeros(1, 8, 3, dtype=torch.float64, device=cuda_device)
    prev_list = []
    for k, cur in enumerate(steps):
        h.update(*_flat(cuda_device, [cur]), gamma_prev)
        start, has = h.gamma_start.cpu().numpy()[0], h.has.cpu().numpy()[0]
        for slot, c in enumerate(cur):
            past = sol.get(c, []) if c in prev_list else []
            depth = min(len(past), order)
            assert has[slot] == depth, (k, slot, has[slot], depth)
            g = [np.asarray(x) for x in past[::-1]]  # g1, g2, g3
            want = np.zeros(3) if depth == 0 else g[0] if depth == 1 else \
                2.0 * g[0] - g[1] if depth == 2 else 3.0 * g[0] - 3.0 * g[1] + g[2]
            np.testing.assert_allclose(start[slot], want, rtol=0, atol=1e-12)
        assert np.all(start[len(cur):] == 0.0) and np.all(has[len(cur):] == 0)
        # this step's solve: a new impulse per live contact; a contact absent
        # at this step loses its history
        g = rng.normal(size=(8, 3))
        gamma_prev = torch.as_tensor(g[None], device=cuda_device).contiguous()
        sol = {c: (sol.get(c, []) if c in prev_list else []) + [g[slot]] for slot, c in enumerate(cur)}
        prev_list = list(cur)


def test_site_scene_contacts_match_the_restatement(cuda_device):
    model, state, control, shapes, host = models.site_scene("humanoid", 16, 41, cuda_device)
    gen = ContactGenerator(shapes, _ModelView(model), capacity=16 * 32, gap=1.0e-3)
    gen.generate(state.joint_q)
    torch.cuda.synchronize()
    bq, _ = ob.eval_fk(host["g"], host["q"].reshape(-1), np.zeros(model.joint_dof_count))
    ref = oc.generate(shapes, bq, gap=1.0e-3)
    n = len(ref["shape0"])
    assert int(gen.count.item()) == n == int(host["counts"].sum())
    np.testing.assert_array_equal(gen.shape0[:n].cpu().numpy(), ref["shape0"])
    np.testing.assert_array_equal(gen.shape1[:n].cpu().numpy(), ref["shape1"])
    np.testing.assert_allclose(gen.point1[:n].cpu().numpy(), ref["point1"], rtol=1e-12, atol=1e-12)
    groups = shapes.shape_collision_group
    assert np.all(groups[ref["shape0"]] == groups[ref["shape1"]])


def test_regenerated_contacts_rollout(cuda_device):
    """Contacts regenerated from the pose every step (they appear and
    vanish): the previous-impulse start, carried by contact identity, needs
    fewer Newton iterations than the previous-velocity start, every world
    converges, and new contacts get no carried impulse."""
    W, steps = 512, 40
    model, state, control, shapes, host = models.site_scene("humanoid", W, 42, cuda_device)
    iters, counts_seen, new_seen = {}, set(), 0
    for warm in ("previous_velocity", "previous_impulses"):
        solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
                           warm_start=warm)
        gen = ContactGenerator(shapes, solver.view, capacity=W * 32, gap=1.0e-3)
        a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        tot = 0.0
        for k in range(steps):
            contacts = gen.generate(a.joint_q, check_capacity=True)
            solver.step(a, b, control, contacts, 2.0e-3)
            a, b = b, a
            assert bool(solver.contact_solve.converged_env.all())
            tot += float(solver.contact_solve.newton_iterations_env.double().mean())
            if warm == "previous_impulses":
                counts_seen.add(int(contacts.rigid_contact_count.item()))
                if k > 0:
                    live = torch.arange(32, device=cuda_device)[None, :] < \
                        solver.contact_jacobian.contact_env_count.clamp(max=32)[:, None]
                    new_seen += int((live & (solver.has_history == 0)).sum())
        iters[warm] = tot / steps
        assert bool(torch.isfinite(a.joint_q).all())
    assert len(counts_seen) > 1, "the contact set never changed"
    assert new_seen > 0, "no contact appeared"
    assert iters["previous_impulses"] < iters["previous_velocity"]


def test_free_motion_forms_the_start_velocity(cuda_device):
    """With the history inside the free-motion launch, the start velocity it
    writes is v* + A^-1 J^T gamma_start of this step's slots (numpy on the
    launch's own A, J and start impulses), and the start impulses are the
    history's extrapolation of the last solves' impulses."""
    W, steps, n = 64, 5, 35
    model, state, control, contacts, _ = models.rollout_scene("humanoid", W, 63, cuda_device)
    solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
                       warm_start="previous_impulses")
    other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
    past = []
    for k in range(steps):
        solver.step(state, other, control, contacts, 2.0e-3)
        torch.cuda.synchronize()
        cj = solver.contact_jacobian
        A = cj.dynamics_matrix_env.cpu().numpy()
        J = cj.contact_env_jacobian.cpu().numpy()
        cnt = cj.contact_env_count.clamp(max=32).cpu().numpy()
        vs = cj.v_star.cpu().numpy().reshape(W, n)
        g = solver._gamma_prev.cpu().numpy()
        got = solver._v_start.cpu().numpy().reshape(W, n)
        for e in range(W):
            c = int(cnt[e])
            want = vs[e] + np.linalg.solve(A[e], J[e, :c].reshape(3 * c, n).T @ g[e, :c].reshape(-1))
            np.testing.assert_allclose(got[e], want, rtol=1e-9, atol=1e-9 * np.abs(want).max())
        # fixed contact set: every slot keeps its contact; start = extrapolation
        depth = min(k, 3)
        has = solver.has_history.cpu().numpy()
        live = np.arange(32)[None, :] < cnt[:, None]
        assert np.all(has[live] == depth)
        if depth:
            g1 = past[-1]
            want = g1 if depth == 1 else 2 * g1 - past[-2] if depth == 2 else 3 * g1 - 3 * past[-2] + past[-3]
            np.testing.assert_allclose(g[live], want[live], rtol=0, atol=1e-12 * np.abs(want).max())
        past.append(solver.contact_solve.contact_gamma.cpu().numpy().copy())
        state, other = other, state
        assert bool(solver.contact_solve.converged_env.all())


def test_factor_written_only_where_a_contact_is_new(cuda_device):
    """Learned start serving new contacts: the free motion writes the LDL^T
    factor only for worlds with a new contact in a live slot; the others keep
    whatever the buffer held (here NaN), and the step still converges."""
    W = 256
    model, state, control, shapes, _ = models.site_scene("humanoid", W, 43, cuda_device)
    solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
                       warm_start="learned")
    gen = ContactGenerator(shapes, solver.view, capacity=W * 32, gap=1.0e-3)
    other = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
    seen_new = seen_old = 0
    for k in range(12):
        solver.contact_jacobian.dynamics_factor_env.fill_(float("nan"))
        solver.step(state, other, control, gen.generate(state.joint_q), 2.0e-3)
        torch.cuda.synchronize()
        cnt = solver.contact_jacobian.contact_env_count.clamp(max=32)
        live = torch.arange(32, device=cuda_device)[None, :] < cnt[:, None]
        new = (live & (solver.has_history == 0)).any(1)
        diag = torch.diagonal(solver.contact_jacobian.dynamics_factor_env, dim1=1, dim2=2)
        written = torch.isfinite(diag).all(1)
        assert torch.equal(written, new), k
        seen_new += int(new.sum())
        seen_old += int((~new).sum())
        assert bool(solver.contact_solve.converged_env.all())
        state, other = other, state
    assert seen_new > 0 and seen_old > 0
