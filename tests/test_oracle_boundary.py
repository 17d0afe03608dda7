"""The numpy restatement of the public-order boundary (oracle/boundary.py):
known answers and round trips."""

import numpy as np

from oracle import boundary as ob
from sap_warp_b200 import models


def _case(kind, seed, worlds=3):
    rng = np.random.default_rng(seed)
    tpl = models.world_template(kind, rng, random_child_frames=True)
    g = models.replicate(tpl, worlds, rng)
    q = models.random_joint_q(tpl, rng, worlds).reshape(-1)
    D = g["counts"]["dofs"]
    return rng, g, q, D


def test_round_trip_is_identity():
    for kind in ("humanoid", "arm_box", "slider"):
        rng, g, q, D = _case(kind, 1)
        qd = rng.normal(size=D)
        sap, _, _ = ob.public_to_sap(g, q, qd_pub=qd)
        np.testing.assert_allclose(ob.sap_to_public_velocity(g, q, sap), qd, atol=1e-14)


def test_single_free_body_known_answers():
    """One free body with identity joint frames: body pose = joint pose,
    public body velocity = public joint velocity; SAP velocity = [w; v_com -
    w x R c]; a force f at the COM gives the SAP joint force [R c x f; f] and
    the body force [-(R c x f); -f]."""
    rng = np.random.default_rng(2)
    tpl = models.world_template("box", rng)
    g = models.replicate(tpl, 1, rng)
    g["body_com"][:] = [0.1, -0.2, 0.05]
    q = np.array([0.3, -0.1, 0.9, 0.0, 0.0, np.sin(0.4), np.cos(0.4)])
    qd = np.array([1.0, 2.0, 3.0, 0.5, -0.25, 0.125])
    bq, bqd = ob.eval_fk(g, q, qd)
    np.testing.assert_allclose(bq[0], q, atol=1e-15)
    np.testing.assert_allclose(bqd[0], qd, atol=1e-15)
    c = ob.qrot(q[3:], g["body_com"][0])
    w = qd[3:]
    sap, _, _ = ob.public_to_sap(g, q, qd_pub=qd)
    np.testing.assert_allclose(sap, np.concatenate([w, qd[:3] - np.cross(w, c)]), atol=1e-15)
    f = np.array([0.0, 0.0, -9.81])
    _, fs, bfs = ob.public_to_sap(g, q, body_q=bq, f_pub=np.concatenate([f, np.zeros(3)]),
                                  bf_pub=np.concatenate([f, np.zeros(3)])[None])
    np.testing.assert_allclose(fs, np.concatenate([np.cross(c, f), f]), atol=1e-15)
    np.testing.assert_allclose(bfs[0], -np.concatenate([np.cross(c, f), f]), atol=1e-15)
