"""Host side of the tree-blocked problem: the box-stack generator's blocked
arrays agree with their dense form, and the oracle solves a small world."""

import numpy as np

from sap_warp_b200 import scenes


def test_blocked_and_dense_layouts_agree():
    bp = scenes.box_stack_problem(3, seed=7, boxes=20, max_contacts=160, sites=(4, 7))
    d = bp.to_dense()
    E, n = d.num_envs, d.dof_per_env
    assert n == 120 and bp.contact_count.max() <= 160
    A = d.dynamics_matrix
    np.testing.assert_allclose(A, A.transpose(0, 2, 1), atol=1e-15)
    assert np.linalg.eigvalsh(A).min() > 0
    v = np.random.default_rng(1).normal(size=(E, n))
    vc_dense = np.einsum("ecrj,ej->ecr", d.jacobian, v)
    vb = v.reshape(E, bp.trees_per_env, 6)
    vc_blocked = np.zeros_like(vc_dense)
    for s in range(2):
        t = bp.contact_tree[..., s]
        vt = np.take_along_axis(vb, np.maximum(t, 0)[..., None], axis=1) * (t >= 0)[..., None]
        vc_blocked += np.einsum("ecrj,ecj->ecr", bp.jacobian[..., 6 * s:6 * s + 6], vt)
    np.testing.assert_allclose(vc_blocked, vc_dense, atol=1e-13)
    # contacts couple trees (stacks and side contacts) and never a tree with itself
    both = (bp.contact_tree[..., 0] >= 0) & (bp.contact_tree[..., 1] >= 0)
    assert both.any()
    assert not np.any(both & (bp.contact_tree[..., 0] == bp.contact_tree[..., 1]))


def test_oracle_solves_small_box_world(oracle):
    bp = scenes.box_stack_problem(2, seed=8, boxes=8, max_contacts=64, sites=(2, 3))
    r = oracle.solve(bp.to_dense(), "armijo_decay")
    assert np.all(r["converged"] == 1)


def _model(kind, worlds=3, boxes=4):
    import torch  # noqa: F401  (SapModel holds torch tensors)

    from sap_warp_b200 import models

    rng = np.random.default_rng(11)
    tpl = models.world_template(kind, rng, boxes=boxes)
    g = models.replicate(tpl, worlds, rng)
    return models.to_model(tpl, g, models.random_joint_q(tpl, rng, worlds), "cpu")


def test_tree_layout_of_articulated_worlds():
    """The trees of the tree-blocked layout are the articulations: an arm
    among boxes gives trees of 7 and 6 DOFs in blocks of 7, chosen by
    default beyond 60 DOFs; a world whose one tree exceeds 12 DOFs stays
    dense; uneven batches stay dense."""
    from sap_warp_b200.solver import _ModelView, tree_block_for

    v = _ModelView(_model("arm_boxes", boxes=4))
    assert v.tree_block == 7 and v.tree_eligible and not v.tree_blocked  # 31 DOFs: dense by default
    np.testing.assert_array_equal(v.tree_dof_start.numpy(), [0, 7, 13, 19, 25, 31])
    big = _ModelView(_model("arm_boxes", boxes=12))
    assert big.n == 79 and big.tree_blocked and big.tree_block == 7
    boxes = _ModelView(_model("boxes", boxes=12))
    assert boxes.tree_block == 6 and boxes.tree_blocked
    hum = _ModelView(_model("humanoid"))
    assert hum.tree_block == 0 and not hum.tree_eligible  # one 35-DOF tree
    quad = _ModelView(_model("quadruped"))
    assert tree_block_for(18) == 0 and not quad.tree_eligible
