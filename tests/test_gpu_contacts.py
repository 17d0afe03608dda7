"""GPU contact generation (sapb_generate_contacts through the C ABI) against
the numpy restatement, and worlds of boxes stepped with contacts regenerated
from the body poses every step."""

import numpy as np
import pytest
import torch

from oracle import boundary as ob
from oracle import contacts as oc
from sap_warp_b200 import _abi, models
from sap_warp_b200.collision import ContactGenerator, ContactOverflowError, ShapeSet
from sap_warp_b200.runtime import SapContacts, SapState
from sap_warp_b200.solver import SolverSAP, _ModelView

pytestmark = pytest.mark.gpu


def _compare(gen, ref, n):
    assert int(gen.count.item()) == n == len(ref["shape0"])
    np.testing.assert_array_equal(gen.shape0[:n].cpu().numpy(), ref["shape0"])
    np.testing.assert_array_equal(gen.shape1[:n].cpu().numpy(), ref["shape1"])
    for k in ("point0", "point1", "normal", "margin0", "margin1"):
        np.testing.assert_allclose(getattr(gen, k)[:n].cpu().numpy(), ref[k], rtol=1e-12, atol=1e-12, err_msg=k)


def test_box_stacks_match_oracle(cuda_device):
    model, state, control, con, _, host = models.box_scene(4, 71, cuda_device, boxes=12, sites=(3, 5))
    shapes = models.box_shapes(host)
    gen = ContactGenerator(shapes, _ModelView(model), capacity=4096, gap=2.0e-3)
    gen.generate(state.joint_q)
    torch.cuda.synchronize()
    bq, _ = ob.eval_fk(host["g"], host["q"].reshape(-1), np.zeros(model.joint_dof_count))
    ref = oc.generate(shapes, bq, gap=2.0e-3)
    _compare(gen, ref, len(ref["shape0"]))
    ground = int((ref["shape0"] == 4 * 12).sum())
    assert ground >= 4 * 3 * 4 and ground % 4 == 0  # four corners of each bottom box, three or more sites a world
    assert len(ref["shape0"]) > ground + 48  # and the boxes stacked on them


def test_spheres_and_boxes_match_oracle(cuda_device):
    """A mixed set (spheres, rotated boxes, margins) with overlapping pairs of
    every kind against the restatement."""
    rng = np.random.default_rng(5)
    tpl = models.world_template("boxes", rng, boxes=10)
    E, B = 3, 10
    g = models.replicate(tpl, E, rng)
    q = np.zeros((E, 7 * B))
    for e in range(E):
        q7 = q[e].reshape(B, 7)
        q7[:, :3] = rng.uniform(-0.15, 0.15, size=(B, 3)) + [0.0, 0.0, 0.12]
        quat = rng.normal(size=(B, 4))
        q7[:, 3:] = quat / np.linalg.norm(quat, axis=1, keepdims=True)
    model = models.to_model(tpl, g, q, cuda_device)
    S = E * B + 1
    types = np.where(np.arange(S) % 3 == 0, _abi.SAPB_SHAPE_SPHERE, _abi.SAPB_SHAPE_BOX).astype(np.int32)
    types[-1] = _abi.SAPB_SHAPE_PLANE
    scale = rng.uniform(0.04, 0.1, size=(S, 3))
    X = np.zeros((S, 7))
    X[:, 6] = 1.0
    X[:-1, :3] = rng.normal(scale=0.01, size=(S - 1, 3))
    shapes = ShapeSet(num_worlds=E, shapes_per_world=B, num_global_shapes=1, shape_type=types, shape_scale=scale,
                      shape_X_bs=X, shape_body=np.concatenate([np.arange(E * B), [-1]]).astype(np.int32),
                      shape_margin=rng.uniform(0.0, 0.005, size=S))
    gen = ContactGenerator(shapes, _ModelView(model), capacity=8192, gap=1.0e-2)
    gen.generate(torch.as_tensor(q.reshape(-1), device=cuda_device))
    torch.cuda.synchronize()
    bq, _ = ob.eval_fk(g, q.reshape(-1), np.zeros(6 * B * E))
    ref = oc.generate(shapes, bq, gap=1.0e-2)
    kinds = {(min(types[a], types[b]), max(types[a], types[b])) for a, b in zip(ref["shape0"], ref["shape1"])}
    assert {(0, 1), (0, 2), (1, 1), (1, 2), (2, 2)} <= kinds
    _compare(gen, ref, len(ref["shape0"]))


def test_box_worlds_step_with_generated_contacts(cuda_device):
    """64-box worlds (tree-blocked step) over 20 steps with contacts
    regenerated from the current poses each step: every world converges, the
    stacks stay standing (no box sinks below the ground by more than a few
    millimetres or moves by more than a few centimetres), and two runs give
    the same trajectory bit for bit."""
    def run():
        model, state, control, _, _, host = models.box_scene(16, 72, cuda_device)
        shapes = models.box_shapes(host)
        view = _ModelView(model)
        gen = ContactGenerator(shapes, view, capacity=16 * 512, gap=2.0e-3)
        solver = SolverSAP(model, max_rigid_contact=512, contact_preset_variant="drake", hessian_precision="fp32")
        a = state
        b = SapState(joint_q=state.joint_q.clone(), joint_qd=state.joint_qd.clone(), body_q=state.body_q.clone(),
                     body_f=state.body_f.clone())
        q0 = state.joint_q.clone()
        for _ in range(20):
            solver.step(a, b, control, gen.generate(a.joint_q), 2e-3)
            assert bool(solver.contact_solve.converged_env.all())
            a, b = b, a
        return q0, a.joint_q.clone()
    q0, q1 = run()
    _, q2 = run()
    assert torch.equal(q1, q2)
    p0 = q0.reshape(-1, 7)[:, :3]
    p1 = q1.reshape(-1, 7)[:, :3]
    assert float(p1[:, 2].min()) > -5e-3
    assert float((p1 - p0).norm(dim=1).max()) < 5e-2


def test_capacity_clamps_and_keeps_the_prefix(cuda_device):
    """More contacts than slots: the count is the number found (as the
    reference's writer counts), the slots hold the oracle's first contacts in
    order, nothing past them is written, and the generator reports the
    overflow."""
    model, state, control, con, _, host = models.box_scene(2, 76, cuda_device, boxes=8, sites=(2, 3))
    shapes = models.box_shapes(host)
    bq, _ = ob.eval_fk(host["g"], host["q"].reshape(-1), np.zeros(model.joint_dof_count))
    ref = oc.generate(shapes, bq, gap=2.0e-3)
    total = len(ref["shape0"])
    cap = total // 2
    gen = ContactGenerator(shapes, _ModelView(model), capacity=cap + 5, gap=2.0e-3)
    gen.outputs.capacity = cap  # the last five slots stay outside the buffer the kernel may write
    gen.shape0.fill_(-7)
    gen.generate(state.joint_q)
    torch.cuda.synchronize()
    assert int(gen.count.item()) == total
    assert gen.overflowed()
    np.testing.assert_array_equal(gen.shape0[:cap].cpu().numpy(), ref["shape0"][:cap])
    np.testing.assert_allclose(gen.point1[:cap].cpu().numpy(), ref["point1"][:cap], rtol=1e-12, atol=1e-12)
    assert bool((gen.shape0[cap:] == -7).all())
    with pytest.raises(ContactOverflowError):
        gen.generate(state.joint_q, check_capacity=True)
    # the step reads only the slots the buffer holds
    from sap_warp_b200.solver import SapContactJacobian
    cj = SapContactJacobian(model, max_rigid_contact=64, fallback_tau_d=0.0)
    contacts = gen.generate(state.joint_q)
    cj.compute(state, SapContacts(**{k: (v[:cap] if (v is not None and v.dim() > 0 and v.shape[0] == cap + 5)
                                         else v) for k, v in vars(contacts).items()}), control=control, dt=2.0e-3)
    torch.cuda.synchronize()
    assert int(cj.contact_env_count.sum()) <= cap


def test_no_candidate_pairs(cuda_device):
    """One shape per world and no static shape: no pair, count 0."""
    model, state, control, con, _, host = models.box_scene(2, 77, cuda_device, boxes=1, sites=(1, 1))
    shapes = models.box_shapes(host)
    one = ShapeSet(num_worlds=2, shapes_per_world=1, num_global_shapes=0, shape_type=shapes.shape_type[:2],
                   shape_scale=shapes.shape_scale[:2], shape_X_bs=shapes.shape_X_bs[:2],
                   shape_body=shapes.shape_body[:2])
    gen = ContactGenerator(one, _ModelView(model), capacity=16)
    gen.count.fill_(3)
    gen.generate(state.joint_q)
    torch.cuda.synchronize()
    assert int(gen.count.item()) == 0


def test_crossed_box_edges_match_oracle(cuda_device):
    """Cubes standing on crossed edges (slightly perturbed per world): the
    edge-edge contact of the separating-axis test, bit-exact in count, pair
    and order with the restatement and within 1e-12 in geometry."""
    rng = np.random.default_rng(9)
    E, B = 4, 2
    tpl = models.world_template("boxes", rng, boxes=B)
    g = models.replicate(tpl, E, rng)
    r = np.sqrt(0.5)
    q = np.zeros((E, 7 * B))
    for e in range(E):
        q7 = q[e].reshape(B, 7)
        for k, (axis, z) in enumerate(((0, 0.0), (1, 2 * r - 1e-3 * (e + 1)))):
            rot = np.zeros(3)
            rot[axis] = np.pi / 4
            rot += rng.normal(scale=1e-3, size=3)
            ang = np.linalg.norm(rot)
            q7[k, 3:6] = np.sin(ang / 2) * rot / ang
            q7[k, 6] = np.cos(ang / 2)
            q7[k, :3] = np.array([0.0, 0.0, z]) + (rng.normal(scale=0.02, size=3) * [1, 1, 0] if k else 0.0)
    model = models.to_model(tpl, g, q, cuda_device)
    S = E * B + 1
    types = np.full(S, _abi.SAPB_SHAPE_BOX, np.int32)
    types[-1] = _abi.SAPB_SHAPE_PLANE
    scale = np.full((S, 3), 0.5)
    X = np.zeros((S, 7))
    X[:, 6] = 1.0
    X[-1, 2] = -10.0  # the ground far below
    shapes = ShapeSet(num_worlds=E, shapes_per_world=B, num_global_shapes=1, shape_type=types, shape_scale=scale,
                      shape_X_bs=X, shape_body=np.concatenate([np.arange(E * B), [-1]]).astype(np.int32))
    gen = ContactGenerator(shapes, _ModelView(model), capacity=256, gap=1.0e-4)
    gen.generate(torch.as_tensor(q.reshape(-1), device=cuda_device))
    torch.cuda.synchronize()
    bq, _ = ob.eval_fk(g, q.reshape(-1), np.zeros(6 * B * E))
    ref = oc.generate(shapes, bq, gap=1.0e-4)
    assert len(ref["shape0"]) == E  # one edge-edge contact per world, nothing else
    assert np.all(np.abs(ref["normal"][:, 2]) > 0.99)
    _compare(gen, ref, len(ref["shape0"]))
