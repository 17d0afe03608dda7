"""The two CPU restatements of the free motion, contact rows and integration
(C with OpenMP: oracle/sap_free_motion.c; numpy: oracle/free_motion.py)
agree to rounding on every model kind and both point / weight modes."""

import numpy as np
import pytest

from oracle import free_motion as ofm
from sap_warp_b200 import models


@pytest.mark.parametrize("kind", ["humanoid", "quadruped", "slider", "arm_box"])
def test_c_and_numpy_restatements_agree(oracle, kind):
    rng = np.random.default_rng(11)
    tpl = models.world_template(kind, rng, random_child_frames=kind in ("slider", "arm_box"))
    E = 6
    g = models.replicate(tpl, E, rng)
    q = models.random_joint_q(tpl, rng, E)
    n, B = tpl["dofs_per_world"], tpl["bodies_per_world"]
    qd = rng.normal(scale=0.5, size=(E, n))
    om = ofm.Model(dict(tpl, gravity=g["gravity"][0], shape_body_global=g["shape_body"],
                        shape_mu=g["shape_material_mu"], shape_ke=g["shape_material_ke"],
                        shape_tau=g["shape_material_tau"]))
    dt = np.full(E, 2e-3)
    fm = ofm.free_motion(om, q, qd, np.zeros_like(qd), np.zeros((E, B, 6)), dt)
    counts = rng.integers(4, 20, size=E)
    con = models.ground_contacts(rng, fm["pos"], fm["quat"], counts, bodies_from=B // 2,
                                 capacity=int(counts.sum()) + 3)
    hm = oracle.HostModel(tpl, g)
    for pm, wm in (("witness_point", "body_inertia"), ("contact_midpoint", "diag_delassus")):
        r = oracle.free_motion_contacts(hm, q, qd, con, dt, 12, point_mode=pm, weight_mode=wm, want_factor=True)
        ref = ofm.contact_jacobian(om, fm, con, 12, point_mode=pm, weight_mode=wm, fallback_tau=0.0)
        scale = np.abs(fm["A"]).max()
        np.testing.assert_allclose(r["A"], fm["A"], rtol=0, atol=1e-13 * scale)
        np.testing.assert_allclose(r["v_star"], fm["v_star"], rtol=1e-12, atol=1e-12)
        np.testing.assert_array_equal(r["count"], ref["count"])
        assert r["truncated"] == ref["truncated"]
        for key in ("jac", "phi0", "mu", "k", "tau", "w"):
            np.testing.assert_allclose(r[key], ref[key], rtol=1e-12, atol=1e-14, err_msg=key)
        np.testing.assert_array_equal(r["body1"], ref["body1"])
        vc = np.einsum("ecrj,ej->ecr", r["jac"], r["v_star"])
        np.testing.assert_allclose(r["vc_star"], vc, rtol=1e-12, atol=1e-12)
        # LDL^T storage of the factor reconstructs A
        for e in range(E):
            d = np.diag(r["factor"][e]).copy()
            L = np.tril(r["factor"][e], -1) / d[None, :] + np.eye(n)
            np.testing.assert_allclose(L @ np.diag(d) @ L.T, r["A"][e], rtol=0, atol=1e-12 * scale)
    for mode in ("sap_euler", "midpoint"):
        qn = oracle.integrate_positions(hm, q.reshape(-1), qd.reshape(-1), 1.1 * qd.reshape(-1), dt, mode)
        np.testing.assert_allclose(qn.reshape(E, -1), ofm.integrate(om, q, qd, 1.1 * qd, dt, mode), rtol=0,
                                   atol=1e-15)


def test_motion_subspaces_are_pose_derivatives_for_every_mobilizer():
    """Pins the numpy restatement of every mobilizer (free, ball, distance,
    D6 with 1-3 rotation axes and 1-3 translations, revolute, prismatic) to
    calculus: for joints whose velocity is the derivative of their
    coordinates (scalar coordinates: revolute, prismatic, D6), the motion
    subspace column S_k at a body origin equals the finite difference of
    that body's pose with respect to coordinate k."""
    from oracle.free_motion import JOINT_D6, JOINT_PRISMATIC, JOINT_REVOLUTE, qconj, qmul

    rng = np.random.default_rng(13)
    tpl = models.world_template("joints", rng)
    g = models.replicate(tpl, 1, rng)
    q = models.random_joint_q(tpl, rng, 1)
    n, B = tpl["dofs_per_world"], tpl["bodies_per_world"]
    om = ofm.Model(dict(tpl, gravity=g["gravity"][0]))
    zero = np.zeros((1, n))
    base = ofm.free_motion(om, q, zero, zero, np.zeros((1, B, 6)), np.full(1, 2e-3))
    checked = 0
    for j, jt in enumerate(tpl["joint_type"]):
        if jt not in (JOINT_REVOLUTE, JOINT_PRISMATIC, JOINT_D6):
            continue
        qs, ds = tpl["joint_q_start"][j], tpl["joint_qd_start"][j]
        for k in range(int(tpl["joint_dof_dim"][j].sum())):
            eps = 1e-6
            qp = q.copy()
            qp[0, qs + k] += eps
            qm = q.copy()
            qm[0, qs + k] -= eps
            fp = ofm.free_motion(om, qp, zero, zero, np.zeros((1, B, 6)), np.full(1, 2e-3))
            fmn = ofm.free_motion(om, qm, zero, zero, np.zeros((1, B, 6)), np.full(1, 2e-3))
            child = tpl["joint_child"][j]
            for b in range(B):  # every body the column moves (its own and the subtree)
                dp = (fp["pos"][0, b] - fmn["pos"][0, b]) / (2 * eps)
                dq = qmul(fp["quat"][0, b], qconj(fmn["quat"][0, b]))
                dw = 2.0 * dq[:3] * np.sign(dq[3]) / (2 * eps)
                Jcol = base["Jb"][0, b, :, ds + k]
                np.testing.assert_allclose(Jcol[:3], dw, rtol=1e-6, atol=1e-7, err_msg=f"joint {j} dof {k} body {b}")
                np.testing.assert_allclose(Jcol[3:], dp, rtol=1e-6, atol=1e-7, err_msg=f"joint {j} dof {k} body {b}")
            assert child >= 0
            checked += 1
    assert checked == 1 + 1 + 4 * 3  # revolute, prismatic, the four D6 joints of three axes each
