"""SolverSAP on an uneven batch: one model of worlds of different sizes (arm
+ box 13 DOF, quadruped 18, humanoid 35; models.concat_models), stepped as
one batch -- one free-motion launch, one persistent solve launch with each
world at its own DOF count, one tail launch -- against the same worlds
stepped as three homogeneous batches (previous-velocity, previous-impulse and
learned starts; with and without drive and limit terms), and a
graph-captured rollout against eager steps."""

import numpy as np
import pytest
import torch

from sap_warp_b200 import models
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SolverSAP

pytestmark = pytest.mark.gpu


def _pair(state):
    return [SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone()) for _ in range(2)]


@pytest.mark.parametrize("warm,drives", [("previous_velocity", False), ("previous_impulses", False),
                                         ("learned", False), ("previous_impulses", True), ("learned", True)])
def test_uneven_batch_steps_like_its_homogeneous_parts(cuda_device, warm, drives):
    """Also with the learned start (the network, the start velocity and the
    free motion's factor in the solve's slots) and with drive and limit terms
    (their per-DOF arrays read in the model's global order)."""
    Wk, steps = 64, 6
    model, state, control, contacts, parts = models.mixed_rollout_scene(Wk, 31, cuda_device, drives=drives)
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32", warm_start=warm)
    solver = SolverSAP(model, **kw)
    assert solver.view.uneven and list(np.unique(solver.view.dof_counts)) == [13, 18, 35]
    assert solver.view.has_pd == drives and solver.view.has_limits == drives
    a, b = _pair(state)
    for _ in range(steps):
        solver.step(a, b, control, contacts, 2.0e-3)
        a, b = b, a
    torch.cuda.synchronize()
    assert bool(solver.contact_solve.converged_env.all())
    iters = solver.contact_solve.newton_iterations_env.cpu().numpy()
    qo = qdo = w0 = 0
    for pm, ps, pc, pcon in parts:
        s = SolverSAP(pm, **kw)
        x, y = _pair(ps)
        for _ in range(steps):
            s.step(x, y, pc, pcon, 2.0e-3)
            x, y = y, x
        torch.cuda.synchronize()
        nq, nd, W = x.joint_q.numel(), x.joint_qd.numel(), int(pm.world_count)
        for got, want in ((a.joint_q[qo:qo + nq], x.joint_q), (a.joint_qd[qdo:qdo + nd], x.joint_qd)):
            err = (got - want).abs().max().item() / max(want.abs().max().item(), 1e-30)
            assert err <= 1e-9, (pm.joint_dof_count // W, err)
        it = s.contact_solve.newton_iterations_env.cpu().numpy()
        assert np.abs(iters[w0:w0 + W] - it).max() <= 1
        qo, qdo, w0 = qo + nq, qdo + nd, w0 + W


def test_uneven_batch_graph_replay_equals_eager(cuda_device):
    model, state, control, contacts, _ = models.mixed_rollout_scene(48, 32, cuda_device)
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
              warm_start="previous_impulses")
    eager = SolverSAP(model, **kw)
    a, b = _pair(state)
    for _ in range(8):
        eager.step(a, b, control, contacts, 2.0e-3)
        a, b = b, a
    g_solver = SolverSAP(model, **kw)
    ga, gb = _pair(state)
    graph = g_solver.capture_steps(ga, gb, control, contacts, 2.0e-3, warmup=1)
    for _ in range(3):
        graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(ga.joint_q, a.joint_q) and torch.equal(ga.joint_qd, a.joint_qd)
