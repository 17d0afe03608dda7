"""The Newton-array wrappers of runtime.py: zero-copy views through DLPack
(any array exposing __dlpack__, here numpy) marked with the public orders."""

import numpy as np

from sap_warp_b200.runtime import sap_contacts_from_newton, sap_control_from_newton, sap_state_from_newton


class _Arrays:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def test_wrappers_are_zero_copy_and_public():
    q, qd, bq = np.zeros(7), np.zeros(6), np.zeros((1, 7))
    st = sap_state_from_newton(_Arrays(joint_q=q, joint_qd=qd, body_q=bq, body_qd=None, body_f=None))
    assert st.joint_qd_order == "public" and st.body_f_order == "public"
    qd[2] = 5.0
    assert float(st.joint_qd[2]) == 5.0  # shares memory with the caller's array
    ctl = sap_control_from_newton(_Arrays(joint_f=np.ones(6)))
    assert ctl.joint_f_order == "public" and float(ctl.joint_f.sum()) == 6.0
    count = np.array([3], np.int32)
    con = sap_contacts_from_newton(_Arrays(rigid_contact_count=count, rigid_contact_shape0=np.zeros(4, np.int32)))
    count[0] = 2
    assert int(con.rigid_contact_count[0]) == 2 and con.rigid_contact_point0 is None


def test_with_drives_sets_drive_and_limit_terms():
    """models.with_drives: drives and +-limit limits on the revolute and
    prismatic DOFs only, targets near the state's coordinates; the model view
    then reports drive and limit terms."""
    import numpy as np

    from sap_warp_b200 import models
    from sap_warp_b200.solver import _ModelView

    rng = np.random.default_rng(3)
    tpl = models.world_template("quadruped", rng)
    g = models.replicate(tpl, 2, rng)
    q = models.random_joint_q(tpl, rng, 2)
    m = models.to_model(tpl, g, q, "cpu")
    m2, c2 = models.with_drives(m, m.state(), m.control(), rng, limit=0.25)
    on = m2.joint_target_mode.numpy() != 0
    assert on.sum() == 2 * 12 and not on.reshape(2, -1)[:, :6].any()  # the free base has none
    lo, hi = m2.joint_limit_lower.numpy(), m2.joint_limit_upper.numpy()
    np.testing.assert_allclose(hi[on] - lo[on], 0.5)
    assert np.all(np.isinf(lo[~on])) and np.all(c2.joint_target_pos.numpy()[~on] == 0)
    v = _ModelView(m2)
    assert v.has_pd and v.has_limits
