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
