"""Test infrastructure only (the checker): a numpy restatement of the
reference's public-order boundary of the SAP step -- the public <-> SAP
conversions of joint velocities, joint forces and body forces, and the
forward kinematics of public coordinates.

Sources restated (mardigiorgio/sap_warp):
- copy_public_to_sap_velocity_f64_from_joint_pose and the f64 force kernel
  from the joint pose: sim/sap_helpers.py:1481-1622, 1967-2057;
- _copy_public_body_force_to_sap_body_origin_kernel: sim/sap_helpers.py:2058-2073;
- _copy_sap_to_public_velocity_f64_from_joint_pose: sim/sap_helpers.py:1711-1760;
- sap_eval_single_articulation_fk: sim/sap_kinematics.py:85-229;
- the boundary driver: sim/solver_sap.py:1198-1261, 1467-1469.
Arrays follow models.replicate() (global, all worlds): joint_q [coords],
joint velocities / forces [dofs], body_q [B][7] (p, q xyzw), body forces and
velocities [B][6] (public: [f or v; tau or w]).
"""

from __future__ import annotations

import numpy as np

FREE, DISTANCE, PRISMATIC, REVOLUTE, BALL, D6 = 4, 5, 0, 1, 2, 6


def qrot(q, v):
    """Rotate v by the unit quaternion q (x, y, z, w)."""
    qv = np.asarray(q[:3], dtype=np.float64)
    t = 2.0 * np.cross(qv, v)
    return v + q[3] * t + np.cross(qv, t)


def qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + ax * bw + ay * bz - az * by, aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw, aw * bw - ax * bx - ay * by - az * bz])


def tmul(a, b):
    """Transform product (p, q) o (p, q) (sim/sap_kinematics.py: X_wp * X_pj)."""
    return (a[0] + qrot(a[1], b[0]), qmul(a[1], b[1]))


def tinv(x):
    qi = np.array([-x[1][0], -x[1][1], -x[1][2], x[1][3]])
    return (-qrot(qi, x[0]), qi)


def public_to_sap(g: dict, joint_q, body_q=None, qd_pub=None, f_pub=None, bf_pub=None):
    """(qd_sap, f_sap, bf_sap); outputs for absent inputs are None."""
    jt = g["joint_type"]
    qs, ds = g["joint_q_start"], g["joint_qd_start"]
    qd_sap = None if qd_pub is None else np.array(qd_pub, dtype=np.float64).copy()
    f_sap = None if f_pub is None else np.array(f_pub, dtype=np.float64).copy()
    for j in range(len(jt)):
        if jt[j] not in (FREE, DISTANCE):
            continue
        d, q = ds[j], joint_q[qs[j] + 3:qs[j] + 7]
        r = qrot(q, g["body_com"][g["joint_child"][j]])
        if qd_pub is not None:
            v_com, w = qd_pub[d:d + 3], qd_pub[d + 3:d + 6]
            qd_sap[d:d + 3] = w
            qd_sap[d + 3:d + 6] = v_com - np.cross(w, r)
        if f_pub is not None:
            f, tau = f_pub[d:d + 3], f_pub[d + 3:d + 6]
            f_sap[d:d + 3] = tau + np.cross(r, f)
            f_sap[d + 3:d + 6] = f
    bf_sap = None
    if bf_pub is not None:
        bf_pub = np.asarray(bf_pub, dtype=np.float64).reshape(-1, 6)
        bf_sap = np.zeros_like(bf_pub)
        for b in range(bf_pub.shape[0]):
            c = qrot(body_q[b, 3:7], g["body_com"][b])
            f, tau = bf_pub[b, :3], bf_pub[b, 3:]
            bf_sap[b, :3] = -(tau + np.cross(c, f))
            bf_sap[b, 3:] = -f
    return qd_sap, f_sap, bf_sap


def sap_to_public_velocity(g: dict, joint_q, qd_sap):
    jt = g["joint_type"]
    qs, ds = g["joint_q_start"], g["joint_qd_start"]
    out = np.array(qd_sap, dtype=np.float64).copy()
    for j in range(len(jt)):
        if jt[j] not in (FREE, DISTANCE):
            continue
        d, q = ds[j], joint_q[qs[j] + 3:qs[j] + 7]
        r = qrot(q, g["body_com"][g["joint_child"][j]])
        w, v_o = qd_sap[d:d + 3], qd_sap[d + 3:d + 6]
        out[d:d + 3] = v_o + np.cross(w, r)
        out[d + 3:d + 6] = w
    return out


def eval_fk(g: dict, joint_q, qd_pub):
    """Body poses [B][7] and public body velocities [B][6]."""
    B = g["body_mass"].shape[0]
    body_q = np.zeros((B, 7))
    body_qd = np.zeros((B, 6))
    art = g["articulation_start"]
    for a in range(len(art) - 1):
        for i in range(art[a], art[a + 1]):
            parent, child, jt = g["joint_parent"][i], g["joint_child"][i], g["joint_type"][i]
            X_pj = (g["joint_X_p"][i, :3], g["joint_X_p"][i, 3:])
            X_cj = (g["joint_X_c"][i, :3], g["joint_X_c"][i, 3:])
            X_wpj, v_wpj, w_wpj = X_pj, np.zeros(3), np.zeros(3)
            if parent >= 0:
                X_wp = (body_q[parent, :3], body_q[parent, 3:])
                X_wpj = tmul(X_wp, X_pj)
                r_p = X_wpj[0] - (X_wp[0] + qrot(X_wp[1], g["body_com"][parent]))
                w_p = body_qd[parent, 3:]
                v_wpj = body_qd[parent, :3] + np.cross(w_p, r_p)
                w_wpj = w_p
            qs, ds = g["joint_q_start"][i], g["joint_qd_start"][i]
            X_j = (np.zeros(3), np.array([0.0, 0.0, 0.0, 1.0]))
            vj, wj = np.zeros(3), np.zeros(3)
            if jt == PRISMATIC:
                ax = g["joint_axis"][ds]
                X_j = (joint_q[qs] * ax, X_j[1])
                vj = qd_pub[ds] * ax
            elif jt == REVOLUTE:
                ax = g["joint_axis"][ds]
                h = 0.5 * joint_q[qs]
                X_j = (np.zeros(3), np.concatenate([ax * np.sin(h), [np.cos(h)]]))
                wj = qd_pub[ds] * ax
            elif jt == BALL:
                X_j = (np.zeros(3), np.asarray(joint_q[qs:qs + 4], dtype=np.float64))
                wj = np.asarray(qd_pub[ds:ds + 3])
            elif jt in (FREE, DISTANCE):
                X_j = (np.asarray(joint_q[qs:qs + 3], dtype=np.float64), np.asarray(joint_q[qs + 3:qs + 7]))
                vj, wj = np.asarray(qd_pub[ds:ds + 3]), np.asarray(qd_pub[ds + 3:ds + 6])
            elif jt == D6:  # sim/sap_kinematics.py:170-215
                from oracle.free_motion import d6_transform_and_axes

                lin, ang = int(g["joint_dof_dim"][i][0]), int(g["joint_dof_dim"][i][1])
                p_, r_, ax = d6_transform_and_axes(g["joint_axis"][ds:ds + lin + ang],
                                                   np.asarray(joint_q[qs:qs + lin + ang], dtype=np.float64)[None],
                                                   lin, ang)
                X_j = (p_[0], r_[0])
                for k in range(lin):
                    vj = vj + qd_pub[ds + k] * g["joint_axis"][ds + k]
                for k in range(ang):
                    wj = wj + qd_pub[ds + lin + k] * ax[0, k]
            X_wc = tmul(tmul(X_wpj, X_j), tinv(X_cj))
            body_q[child, :3], body_q[child, 3:] = X_wc
            body_qd[child, :3] = v_wpj + qrot(X_wpj[1], vj)
            body_qd[child, 3:] = w_wpj + qrot(X_wpj[1], wj)
    return body_q, body_qd
