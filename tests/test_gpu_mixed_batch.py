"""The uneven batch in one persistent launch: arm + box (13 DOF, two trees
coupled by gripper contacts), quadruped (18) and humanoid (35) worlds padded
to 35 DOF with identity blocks, taken in descending-work order; each world's
answer equals its homogeneous solve and the oracle's."""

import numpy as np
import pytest
import torch

from sap_warp_b200 import scenes
from sap_warp_b200._solve import ContactSolveBuffers, contact_solve, make_options, problem_to_device

pytestmark = pytest.mark.gpu


def solve(prob, dev, order=None, **kw):
    t = problem_to_device(prob, dev)
    buf = ContactSolveBuffers(prob.num_envs, prob.dof_per_env, prob.max_contacts, dev)
    wo = None if order is None else torch.as_tensor(order, dtype=torch.int32).to(dev)
    contact_solve(**t, buffers=buf, options=make_options("armijo_decay", **kw), world_order=wo)
    torch.cuda.synchronize()
    return buf.v.cpu().numpy().reshape(prob.num_envs, -1), buf.newton_iterations.cpu().numpy(), \
        buf.converged.cpu().numpy()


@pytest.fixture(scope="module")
def mixed():
    return scenes.mixed_contact_problem(192, seed=5)


def test_mixed_batch_equals_homogeneous_solves(cuda_device, mixed):
    prob, parts = mixed
    v, it, conv = solve(prob, cuda_device, scenes.work_order(prob))
    assert conv.all()
    off = 0
    for q in parts:
        vq, itq, _ = solve(q, cuda_device)
        E, n = q.num_envs, q.dof_per_env
        np.testing.assert_allclose(v[off:off + E, :n], vq, rtol=1e-10, atol=1e-12)
        assert np.all(v[off:off + E, n:] == 0.0)
        np.testing.assert_array_equal(it[off:off + E], itq)
        off += E


def test_mixed_batch_matches_oracle(cuda_device, oracle, mixed):
    prob, _ = mixed
    v, it, conv = solve(prob, cuda_device, scenes.work_order(prob))
    ref = oracle.solve(prob, "armijo_decay")
    vr = ref["v"].reshape(prob.num_envs, -1)
    err = np.abs(v - vr).max(1) / np.abs(vr).max(1)
    assert np.quantile(err, 0.98) <= 1e-6 and err.max() <= 1e-4, err.max()
    np.testing.assert_array_equal(conv, ref["converged"])


def test_world_order_does_not_change_the_answer(cuda_device, mixed):
    prob, _ = mixed
    v0, it0, _ = solve(prob, cuda_device)
    v1, it1, _ = solve(prob, cuda_device, scenes.work_order(prob))
    rev = np.arange(prob.num_envs, dtype=np.int32)[::-1].copy()
    v2, _, _ = solve(prob, cuda_device, rev)
    assert np.array_equal(v0, v1) and np.array_equal(v0, v2)
    np.testing.assert_array_equal(it0, it1)


def test_mixed_batch_fp32_hessian(cuda_device, oracle, mixed):
    prob, _ = mixed
    v, _, conv = solve(prob, cuda_device, scenes.work_order(prob), hessian_precision="fp32")
    assert conv.all()
    vr = oracle.solve(prob, "armijo_decay")["v"].reshape(prob.num_envs, -1)
    err = np.abs(v - vr).max(1) / np.abs(vr).max(1)
    assert np.quantile(err, 0.98) <= 1e-6 and err.max() <= 1e-4, err.max()


def test_per_world_dof_counts_without_padding(cuda_device, mixed):
    """The same batch with each world's own DOF count (dof_count, compact
    storage, no identity padding): every world equals its homogeneous solve
    (the specialised kernels of its size) to rounding, with the same Newton
    iterations up to one, and the padding of v is written as zero."""
    prob, parts = mixed
    cp = scenes.compact_problem(prob)
    t = problem_to_device(cp, cuda_device)
    buf = ContactSolveBuffers(cp.num_envs, cp.dof_per_env, cp.max_contacts, cuda_device)
    dc = torch.as_tensor(cp.dofs_active, dtype=torch.int32).to(cuda_device)
    buf.v.fill_(float("nan"))
    contact_solve(**t, buffers=buf, options=make_options("armijo_decay"), dof_count=dc,
                  world_order=torch.as_tensor(scenes.work_order(cp), dtype=torch.int32).to(cuda_device))
    torch.cuda.synchronize()
    v, it = buf.v.cpu().numpy().reshape(cp.num_envs, -1), buf.newton_iterations.cpu().numpy()
    assert buf.converged.all()
    off = 0
    for q in parts:
        vq, itq, _ = solve(q, cuda_device)
        E, n = q.num_envs, q.dof_per_env
        err = np.abs(v[off:off + E, :n] - vq).max(1) / np.maximum(np.abs(vq).max(1), 1e-300)
        assert err.max() <= 1e-9, (n, err.max())
        assert np.all(v[off:off + E, n:] == 0.0)
        assert np.abs(it[off:off + E] - itq).max() <= 1
        off += E
