"""The whole step through the C ABI (sapb_create / sapb_step /
sapb_get_status / sapb_destroy) against SolverSAP on the same model, in the
dense and the tree-blocked layout, and the device work-order sort against a
stable host sort."""

import ctypes

import numpy as np
import pytest
import torch

from sap_warp_b200 import _abi, models
from sap_warp_b200._lib import check, load
from sap_warp_b200.runtime import SapState
from sap_warp_b200.solver import SolverSAP

pytestmark = pytest.mark.gpu


def _p(t):
    return 0 if t is None else t.data_ptr()


def test_world_order_is_a_stable_descending_sort(cuda_device):
    lib = load()
    rng = np.random.default_rng(5)
    for W in (1, 7, 1000, 4096, 32768):
        it = rng.integers(0, 12, size=W).astype(np.int32)
        it[::97] = 40000  # clamped keys still sort first
        d_it = torch.as_tensor(it, device=cuda_device)
        order = torch.full((W,), -1, dtype=torch.int32, device=cuda_device)
        check(lib.sapb_world_order(d_it.data_ptr(), W, order.data_ptr(),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "sapb_world_order")
        torch.cuda.synchronize()
        want = np.argsort(-np.minimum(it.astype(np.int64), 0x7FFF), kind="stable")
        np.testing.assert_array_equal(order.cpu().numpy(), want)
    assert lib.sapb_world_order(d_it.data_ptr(), 32769, order.data_ptr(), None) == _abi.SAPB_ERR_UNSUPPORTED


@pytest.mark.parametrize("warm", ["previous_velocity", "previous_impulses"])
def test_c_step_equals_solver_steps(cuda_device, warm):
    W, dt, steps = 256, 2.0e-3, 4
    model, state, control, contacts, _ = models.rollout_scene("humanoid", W, 61, cuda_device)
    solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
                       warm_start=warm)
    a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    for _ in range(steps):
        solver.step(a, b, control, contacts, dt)
        a, b = b, a
    torch.cuda.synchronize()
    ref_q, ref_qd = a.joint_q.clone(), a.joint_qd.clone()
    ref_status = solver.contact_solve.ls_status.clone()
    ref_iters = solver.contact_solve.newton_iterations_env.clone()

    lib = load()
    opts = solver.c_step_options()
    handle = ctypes.c_void_p()
    check(lib.sapb_create(ctypes.byref(solver.view.desc), ctypes.byref(opts), ctypes.byref(handle)), "sapb_create")
    try:
        q = [state.joint_q.to(torch.float64).clone(), state.joint_q.to(torch.float64).clone()]
        qd = [state.joint_qd.to(torch.float64).clone(), state.joint_qd.to(torch.float64).clone()]
        dt_w = torch.full((W,), dt, dtype=torch.float64, device=cuda_device)
        jf = control.joint_f.to(torch.float64).contiguous()
        bf = state.body_f.to(torch.float64).reshape(-1, 6).contiguous()
        io = _abi.StepIO()
        inp = io.inp
        inp.joint_f, inp.body_f, inp.dt = _p(jf), _p(bf), _p(dt_w)
        inp.contact_capacity = int(contacts.rigid_contact_shape0.numel())
        inp.contact_count = _p(contacts.rigid_contact_count)
        inp.contact_shape0, inp.contact_shape1 = _p(contacts.rigid_contact_shape0), _p(contacts.rigid_contact_shape1)
        inp.contact_point0, inp.contact_point1 = _p(contacts.rigid_contact_point0d), _p(contacts.rigid_contact_point1d)
        inp.contact_normal = _p(contacts.rigid_contact_normald)
        inp.contact_margin0, inp.contact_margin1 = (_p(contacts.rigid_contact_margin0d),
                                                    _p(contacts.rigid_contact_margin1d))
        if solver.contact_solve.dof is not None:
            io.dof = ctypes.pointer(solver.contact_solve.dof)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for k in range(steps):
            src, dst = k % 2, 1 - k % 2
            inp.joint_q, inp.joint_qd = _p(q[src]), _p(qd[src])
            io.joint_q_out, io.joint_qd_out = _p(q[dst]), _p(qd[dst])
            check(lib.sapb_step(handle, ctypes.byref(io), stream), "sapb_step")
        status = torch.zeros(W, dtype=torch.int32, device=cuda_device)
        conv = np.zeros(W, np.int32)
        iters = torch.zeros(W, dtype=torch.int32, device=cuda_device)
        check(lib.sapb_get_status(handle, status.data_ptr(), conv.ctypes.data, iters.data_ptr(), stream),
              "sapb_get_status")
        torch.cuda.synchronize()
        out = _abi.SolveOutputs()
        check(lib.sapb_step_solve_outputs(handle, ctypes.byref(out)), "sapb_step_solve_outputs")
        assert out.v and out.contact_gamma and out.status
    finally:
        lib.sapb_destroy(handle)
    last = steps % 2
    assert torch.equal(q[last], ref_q.to(torch.float64)) and torch.equal(qd[last], ref_qd.to(torch.float64))
    assert torch.equal(status, ref_status) and torch.equal(iters, ref_iters)
    assert np.all(conv == 1)


def _c_steps(solver, state, control, contacts, dt, steps, device):
    """`steps` steps of the C handle made from the solver's own options;
    returns (q, qd, status, converged, newton_iterations)."""
    lib = load()
    W = solver.view.W
    opts = solver.c_step_options()
    handle = ctypes.c_void_p()
    check(lib.sapb_create(ctypes.byref(solver.view.desc), ctypes.byref(opts), ctypes.byref(handle)), "sapb_create")
    try:
        q = [state.joint_q.to(torch.float64).clone(), state.joint_q.to(torch.float64).clone()]
        qd = [state.joint_qd.to(torch.float64).clone(), state.joint_qd.to(torch.float64).clone()]
        dt_w = torch.full((W,), dt, dtype=torch.float64, device=device)
        jf = control.joint_f.to(torch.float64).contiguous()
        bf = state.body_f.to(torch.float64).reshape(-1, 6).contiguous()
        io = _abi.StepIO()
        inp = io.inp
        inp.joint_f, inp.body_f, inp.dt = _p(jf), _p(bf), _p(dt_w)
        inp.contact_capacity = int(contacts.rigid_contact_shape0.numel())
        inp.contact_count = _p(contacts.rigid_contact_count)
        inp.contact_shape0, inp.contact_shape1 = _p(contacts.rigid_contact_shape0), _p(contacts.rigid_contact_shape1)
        inp.contact_point0, inp.contact_point1 = _p(contacts.rigid_contact_point0d), _p(contacts.rigid_contact_point1d)
        inp.contact_normal = _p(contacts.rigid_contact_normald)
        inp.contact_margin0, inp.contact_margin1 = (_p(contacts.rigid_contact_margin0d),
                                                    _p(contacts.rigid_contact_margin1d))
        if solver.contact_solve.dof is not None:
            io.dof = ctypes.pointer(solver.contact_solve.dof)
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        for k in range(steps):
            src, dst = k % 2, 1 - k % 2
            inp.joint_q, inp.joint_qd = _p(q[src]), _p(qd[src])
            io.joint_q_out, io.joint_qd_out = _p(q[dst]), _p(qd[dst])
            check(lib.sapb_step(handle, ctypes.byref(io), stream), "sapb_step")
        status = torch.zeros(W, dtype=torch.int32, device=device)
        conv = np.zeros(W, np.int32)
        iters = torch.zeros(W, dtype=torch.int32, device=device)
        check(lib.sapb_get_status(handle, status.data_ptr(), conv.ctypes.data, iters.data_ptr(), stream),
              "sapb_get_status")
        torch.cuda.synchronize()
    finally:
        lib.sapb_destroy(handle)
    last = steps % 2
    return q[last], qd[last], status, conv, iters


@pytest.mark.parametrize("warm,drives", [("previous_velocity", False), ("previous_impulses", False),
                                         ("previous_impulses", True)])
def test_c_step_tree_blocked_equals_solver_steps(cuda_device, warm, drives):
    """The handle in the tree-blocked layout (an arm among 8 boxes: trees of
    7 and 6 DOFs in blocks of 7; with drives and limits on the arm) steps
    like SolverSAP(tree_blocked=True), bit for bit."""
    W, dt, steps = 128, 2.0e-3, 4
    model, state, control, contacts, _, _ = models.box_scene(W, 64, cuda_device, boxes=8, sites=(3, 5), arm=True)
    if drives:
        model, control = models.with_drives(model, state, control, np.random.default_rng(6))
    solver = SolverSAP(model, max_rigid_contact=112, contact_preset_variant="drake", hessian_precision="fp32",
                       warm_start=warm, tree_blocked=True)
    a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    for _ in range(steps):
        solver.step(a, b, control, contacts, dt)
        a, b = b, a
    torch.cuda.synchronize()
    q, qd, status, conv, iters = _c_steps(solver, state, control, contacts, dt, steps, cuda_device)
    assert torch.equal(q, a.joint_q.to(torch.float64)) and torch.equal(qd, a.joint_qd.to(torch.float64))
    assert torch.equal(status, solver.contact_solve.ls_status)
    assert torch.equal(iters, solver.contact_solve.newton_iterations_env)
    assert np.all(conv == 1)


def test_c_handle_refuses_trees_beyond_their_block(cuda_device):
    model, state, control, contacts, _, _ = models.box_scene(4, 65, cuda_device, boxes=3, sites=(2, 2), arm=True)
    solver = SolverSAP(model, max_rigid_contact=64, contact_preset_variant="drake", tree_blocked=True)
    opts = solver.c_step_options()
    opts.prepare.tree_dofs = 6  # the arm has 7 DOFs
    handle = ctypes.c_void_p()
    assert load().sapb_create(ctypes.byref(solver.view.desc), ctypes.byref(opts), ctypes.byref(handle)) == \
        _abi.SAPB_ERR_UNSUPPORTED
    assert not handle.value


@pytest.mark.parametrize("drives", [False, True])
def test_c_step_uneven_batch_equals_solver_steps(cuda_device, drives):
    """The handle on an uneven batch (arm + box 13 DOF, quadruped 18,
    humanoid 35, each world at its own DOF count; with and without drive
    and limit terms) steps like SolverSAP, bit for bit."""
    dt, steps = 2.0e-3, 4
    model, state, control, contacts, _ = models.mixed_rollout_scene(32, 66, cuda_device, drives=drives)
    solver = SolverSAP(model, max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
                       warm_start="previous_impulses")
    assert solver.view.uneven and solver.view.has_pd == drives
    a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    for _ in range(steps):
        solver.step(a, b, control, contacts, dt)
        a, b = b, a
    torch.cuda.synchronize()
    q, qd, status, conv, iters = _c_steps(solver, state, control, contacts, dt, steps, cuda_device)
    assert torch.equal(q, a.joint_q.to(torch.float64)) and torch.equal(qd, a.joint_qd.to(torch.float64))
    assert torch.equal(status, solver.contact_solve.ls_status)
    assert torch.equal(iters, solver.contact_solve.newton_iterations_env)
    assert np.all(conv == 1)


@pytest.mark.parametrize("kind", ["humanoid", "arm_boxes"])
def test_c_step_learned_equals_solver_steps(cuda_device, kind):
    """The handle's learned start (SAPB_WARM_START_LEARNED: the history's
    start plus the network's impulses on new contacts) steps like
    SolverSAP(warm_start="learned"), bit for bit, in the dense layout
    (humanoids) and the tree-blocked one (an arm among boxes)."""
    dt, steps = 2.0e-3, 4
    if kind == "humanoid":
        model, state, control, contacts, _ = models.rollout_scene("humanoid", 256, 67, cuda_device)
        kw = dict(max_rigid_contact=32)
    else:
        model, state, control, contacts, _, _ = models.box_scene(128, 68, cuda_device, boxes=8, sites=(3, 5),
                                                                 arm=True)
        kw = dict(max_rigid_contact=112, tree_blocked=True)
    solver = SolverSAP(model, contact_preset_variant="drake", hessian_precision="fp32", warm_start="learned", **kw)
    a = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                 body_f=state.body_f.clone())
    for _ in range(steps):
        solver.step(a, b, control, contacts, dt)
        a, b = b, a
    torch.cuda.synchronize()
    if kind == "humanoid":  # the start the network feeds is taken (the box stacks often keep the plain one)
        assert int(solver.contact_solve.warm_start_accepted_env.sum()) > 0
    q, qd, status, conv, iters = _c_steps(solver, state, control, contacts, dt, steps, cuda_device)
    assert torch.equal(q, a.joint_q.to(torch.float64)) and torch.equal(qd, a.joint_qd.to(torch.float64))
    assert torch.equal(status, solver.contact_solve.ls_status)
    assert torch.equal(iters, solver.contact_solve.newton_iterations_env)
    assert np.all(conv == 1)
