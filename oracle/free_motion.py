"""numpy restatement of the reference's free motion, contact Jacobian and
position integration -- TEST INFRASTRUCTURE ONLY (the checker for the CUDA
prepare/integrate kernels; see oracle/__init__.py).

Conventions of the reference: quaternions xyzw, transforms (p, q), spatial
vectors [angular; linear] at the body origin in world coordinates
(sim/sap_helpers.py:771-785).  Loops run over joints (parents before
children), vectorised over worlds.
"""

from __future__ import annotations

import numpy as np

JOINT_PRISMATIC, JOINT_REVOLUTE, JOINT_BALL, JOINT_FIXED, JOINT_FREE, JOINT_DISTANCE, JOINT_D6 = range(7)


# ---- quaternion / transform helpers (sim/sap_helpers.py:576-700) ----------------
def qmul(a, b):
    ax, ay, az, aw = np.moveaxis(a, -1, 0)
    bx, by, bz, bw = np.moveaxis(b, -1, 0)
    return np.stack([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz], -1)


def qnormalize(q):
    n = np.linalg.norm(q, axis=-1, keepdims=True)
    return np.where(n > 0, q / np.where(n > 0, n, 1.0), np.array([0.0, 0.0, 0.0, 1.0]))


def qrotate(q, v):
    qv = q[..., :3]
    t = 2.0 * np.cross(qv, v)
    return v + q[..., 3:4] * t + np.cross(qv, t)


def qconj(q):
    return np.concatenate([-q[..., :3], q[..., 3:4]], -1)


def q_axis_angle(axis, angle):
    half = 0.5 * angle
    return np.concatenate([axis * np.sin(half)[..., None], np.cos(half)[..., None]], -1)


def tcompose(ap, aq, bp, bq):
    aq = qnormalize(aq)
    bq = qnormalize(bq)
    return ap + qrotate(aq, bp), qnormalize(qmul(aq, bq))


def tinverse(p, q):
    qi = qconj(qnormalize(q))
    return -qrotate(qi, p), qi


def qmatrix(q):
    """Rotation matrices (..., 3, 3) whose columns are the rotated unit axes."""
    eye = np.eye(3)
    cols = [qrotate(q, np.broadcast_to(eye[i], q.shape[:-1] + (3,))) for i in range(3)]
    return np.stack(cols, -1)


def skew(v):
    z = np.zeros(v.shape[:-1])
    return np.stack([np.stack([z, -v[..., 2], v[..., 1]], -1),
                     np.stack([v[..., 2], z, -v[..., 0]], -1),
                     np.stack([-v[..., 1], v[..., 0], z], -1)], -2)


# ---- spatial algebra (sim/sap_helpers.py:862-1010) ----------------------------
def shift_velocity(V, p):
    return np.concatenate([V[..., :3], V[..., 3:] + np.cross(V[..., :3], p)], -1)


def shift_acceleration(A, p, w):
    return np.concatenate([A[..., :3], A[..., 3:] + np.cross(A[..., :3], p) + np.cross(w, np.cross(w, p))], -1)


def shift_force(F, p):
    return np.concatenate([F[..., :3] - np.cross(p, F[..., 3:]), F[..., 3:]], -1)


def compose_velocity(V_WP, p_PB, V_PB):
    w = V_WP[..., :3]
    return np.concatenate([w + V_PB[..., :3], V_WP[..., 3:] + np.cross(w, p_PB) + V_PB[..., 3:]], -1)


def compose_acceleration(A_WP, V_WP, p_PB, V_PB, A_PB):
    w = V_WP[..., :3]
    As = shift_acceleration(A_WP, p_PB, w)
    alpha = As[..., :3] + A_PB[..., :3] + np.cross(w, V_PB[..., :3])
    a = As[..., 3:] + A_PB[..., 3:] + 2.0 * np.cross(w, V_PB[..., 3:])
    return np.concatenate([alpha, a], -1)


def mobilizer_velocity_to_body(R_WF_q, p_MoBo_F, V_FM_F):
    w_F = V_FM_F[..., :3]
    return np.concatenate([qrotate(R_WF_q, w_F), qrotate(R_WF_q, V_FM_F[..., 3:] + np.cross(w_F, p_MoBo_F))], -1)


def mobilizer_accel_bias_to_body(R_WF_q, p_MoBo_F, V_FM_F):
    w = V_FM_F[..., :3]
    sh = shift_acceleration(np.zeros_like(V_FM_F), p_MoBo_F, w)
    return np.concatenate([qrotate(R_WF_q, sh[..., :3]), qrotate(R_WF_q, sh[..., 3:])], -1)


def quat_from_cols(c0, c1, c2):
    """_quatd_from_matrix_cols (sim/sap_helpers.py:608-655), one rotation."""
    r00, r10, r20 = c0
    r01, r11, r21 = c1
    r02, r12, r22 = c2
    tr = r00 + r11 + r22
    if tr > 0.0:
        s = np.sqrt(tr + 1.0) * 2.0
        return np.array([(r21 - r12) / s, (r02 - r20) / s, (r10 - r01) / s, 0.25 * s])
    if r00 > r11 and r00 > r22:
        s = np.sqrt(1.0 + r00 - r11 - r22) * 2.0
        return np.array([0.25 * s, (r01 + r10) / s, (r02 + r20) / s, (r21 - r12) / s])
    if r11 > r22:
        s = np.sqrt(1.0 + r11 - r00 - r22) * 2.0
        return np.array([(r01 + r10) / s, 0.25 * s, (r12 + r21) / s, (r02 - r20) / s])
    s = np.sqrt(1.0 + r22 - r00 - r11) * 2.0
    return np.array([(r02 + r20) / s, (r12 + r21) / s, 0.25 * s, (r10 - r01) / s])


def d6_transform_and_axes(axes, q, lin, ang):
    """D6 across-mobilizer transform and angular DOF axes per world
    (sim/sap_helpers.py:1109-1161 rotations, :1204-1241 X_FM, :1247-1286
    angular axes).  axes (lin + ang, 3) in F; q (E, lin + ang).  Returns
    (pos (E, 3), rot (E, 4), angular axes (E, ang, 3))."""
    E = q.shape[0]
    pos = np.zeros((E, 3))
    for k in range(lin):
        pos = pos + axes[k] * q[:, k:k + 1]
    rot = np.tile([0.0, 0.0, 0.0, 1.0], (E, 1))
    out = np.zeros((E, max(ang, 1), 3))
    if ang == 1:
        out[:, 0] = axes[lin]
        rot = q_axis_angle(axes[lin], q[:, lin])
    elif ang in (2, 3):
        c0, c1 = axes[lin], axes[lin + 1]
        c2 = axes[lin + 2] if ang == 3 else np.cross(c0, c1)
        off = np.broadcast_to(quat_from_cols(c0, c1, c2), (E, 4))
        l0 = qrotate(off, np.broadcast_to([1.0, 0.0, 0.0], (E, 3)))
        l1 = qrotate(off, np.broadcast_to([0.0, 1.0, 0.0], (E, 3)))
        l2 = qrotate(off, np.broadcast_to([0.0, 0.0, 1.0], (E, 3)))
        q0 = q_axis_angle(l0, q[:, lin])
        a1 = qrotate(q0, l1)
        q10 = qmul(q_axis_angle(a1, q[:, lin + 1]), q0)
        out[:, 0], out[:, 1] = l0, a1
        rot = q10
        if ang == 3:
            a2 = qrotate(q10, l2)
            out[:, 2] = a2
            rot = qmul(q_axis_angle(a2, q[:, lin + 2]), q10)
    return pos, rot, out


def spatial_inertia_body_origin(R, Icom, m, c_body):
    """(sim/sap_helpers.py:1027-1062) 6x6 [[I_Bo, m[c]x], [-m[c]x, m I]]."""
    c = np.einsum("...ij,...j->...i", R, c_body)
    I_com_W = R @ Icom @ np.swapaxes(R, -1, -2)
    I_Bo = I_com_W + m[..., None, None] * ((c * c).sum(-1)[..., None, None] * np.eye(3) - c[..., :, None] * c[..., None, :])
    mcx = m[..., None, None] * skew(c)
    top = np.concatenate([I_Bo, mcx], -1)
    bot = np.concatenate([-mcx, m[..., None, None] * np.eye(3)], -1)
    return np.concatenate([top, bot], -2), I_Bo, c


class Model:
    """Topology and inertial data of one world-replicated model (per world
    arrays, identical topology in every world)."""

    def __init__(self, d: dict):
        self.__dict__.update(d)


def free_motion(m: Model, joint_q, joint_qd, joint_f, body_f, dt):
    """SAP free motion (sim/free_motion.py:2094-2178): returns v*, vdot, A (E,n,n),
    body poses (p, q), body Jacobians (E,B,6,n) and the motion subspaces.

    joint_q (E, Q), joint_qd / joint_f (E, n) SAP order, body_f (E, B, 6)
    SAP order (the negated applied wrench at the body origin), dt (E,)."""
    E = joint_q.shape[0]
    B, Jn, n = m.bodies_per_world, m.joints_per_world, m.dofs_per_world
    pos = np.zeros((E, B, 3))
    quat = np.zeros((E, B, 4))
    quat[..., 3] = 1.0
    V = np.zeros((E, B, 6))
    Ab = np.zeros((E, B, 6))
    S = np.zeros((E, n, 6))
    for j in range(Jn):
        jt, parent, child = m.joint_type[j], m.joint_parent[j], m.joint_child[j]
        qs, ds = m.joint_q_start[j], m.joint_qd_start[j]
        Xp_p = np.broadcast_to(m.joint_X_p[j, :3], (E, 3))
        Xp_q = np.broadcast_to(m.joint_X_p[j, 3:], (E, 4))
        if parent >= 0:
            wf_p, wf_q = tcompose(pos[:, parent], quat[:, parent], Xp_p, Xp_q)
        else:
            wf_p, wf_q = Xp_p.copy(), Xp_q.copy()
        # across-mobilizer transform X_FM (sim/sap_helpers.py:1164-1243)
        fm_p = np.zeros((E, 3))
        fm_q = np.tile([0.0, 0.0, 0.0, 1.0], (E, 1))
        if jt == JOINT_PRISMATIC:
            fm_p = m.joint_axis[ds] * joint_q[:, qs:qs + 1]
        elif jt == JOINT_REVOLUTE:
            fm_q = q_axis_angle(m.joint_axis[ds], joint_q[:, qs])
        elif jt == JOINT_BALL:
            fm_q = joint_q[:, qs:qs + 4].copy()
        elif jt in (JOINT_FREE, JOINT_DISTANCE):
            fm_p = joint_q[:, qs:qs + 3].copy()
            fm_q = joint_q[:, qs + 3:qs + 7].copy()
        elif jt == JOINT_D6:
            lin, ang = int(m.joint_dof_dim[j, 0]), int(m.joint_dof_dim[j, 1])
            fm_p, fm_q, d6_axes = d6_transform_and_axes(m.joint_axis[ds:ds + lin + ang], joint_q[:, qs:qs + lin + ang],
                                                        lin, ang)
        elif jt != JOINT_FIXED:
            raise NotImplementedError(f"joint type {jt}")
        wm_p, wm_q = tcompose(wf_p, wf_q, fm_p, fm_q)
        Xc_p = np.broadcast_to(m.joint_X_c[j, :3], (E, 3))
        Xc_q = np.broadcast_to(m.joint_X_c[j, 3:], (E, 4))
        mb_p, mb_q = tinverse(Xc_p, Xc_q)  # X_MB = X_BM^-1
        wb_p, wb_q = tcompose(wm_p, wm_q, mb_p, mb_q)
        p_MoBo_F = qrotate(qnormalize(fm_q), mb_p)
        R_WF = qnormalize(wf_q)
        # motion subspace and joint velocity (sim/sap_helpers.py:1289-1433)
        dim = m.joint_dof_dim[j, 0] + m.joint_dof_dim[j, 1]
        zero = np.zeros((E, 6))
        if jt == JOINT_PRISMATIC:
            a = np.broadcast_to(m.joint_axis[ds], (E, 3))
            Sj = [mobilizer_velocity_to_body(R_WF, p_MoBo_F, np.concatenate([np.zeros((E, 3)), a], -1))]
            V_FM = np.concatenate([np.zeros((E, 3)), a * joint_qd[:, ds:ds + 1]], -1)
        elif jt == JOINT_REVOLUTE:
            a = np.broadcast_to(m.joint_axis[ds], (E, 3))
            Sj = [np.concatenate([qrotate(R_WF, a), qrotate(R_WF, np.cross(a, p_MoBo_F))], -1)]
            V_FM = np.concatenate([a * joint_qd[:, ds:ds + 1], np.zeros((E, 3))], -1)
        elif jt == JOINT_BALL:
            eye = np.eye(3)
            Sj = [mobilizer_velocity_to_body(R_WF, p_MoBo_F, np.concatenate([np.broadcast_to(eye[k], (E, 3)),
                                                                              np.zeros((E, 3))], -1)) for k in range(3)]
            V_FM = np.concatenate([joint_qd[:, ds:ds + 3], np.zeros((E, 3))], -1)
        elif jt in (JOINT_FREE, JOINT_DISTANCE):
            eye = np.eye(6)
            Sj = [mobilizer_velocity_to_body(R_WF, p_MoBo_F, np.broadcast_to(eye[k], (E, 6))) for k in range(6)]
            V_FM = joint_qd[:, ds:ds + 6].copy()
        elif jt == JOINT_D6:
            # sim/sap_helpers.py:1387-1431: translation columns, then the
            # angular axes at the current angles; V_FM their combination
            Sj = []
            V_FM = np.zeros((E, 6))
            for k in range(lin):
                a = np.broadcast_to(m.joint_axis[ds + k], (E, 3))
                col = np.concatenate([np.zeros((E, 3)), a], -1)
                Sj.append(mobilizer_velocity_to_body(R_WF, p_MoBo_F, col))
                V_FM = V_FM + col * joint_qd[:, ds + k:ds + k + 1]
            for k in range(ang):
                col = np.concatenate([d6_axes[:, k], np.zeros((E, 3))], -1)
                Sj.append(mobilizer_velocity_to_body(R_WF, p_MoBo_F, col))
                V_FM = V_FM + col * joint_qd[:, ds + lin + k:ds + lin + k + 1]
        else:
            Sj = []
            V_FM = zero
        for k, s in enumerate(Sj):
            S[:, ds + k] = s
        V_PB = mobilizer_velocity_to_body(R_WF, p_MoBo_F, V_FM) if dim > 0 else zero
        A_PB = mobilizer_accel_bias_to_body(R_WF, p_MoBo_F, V_FM) if dim > 0 else zero
        if jt == JOINT_REVOLUTE:
            # sim/sap_helpers.py:1320-1329: the angular part of the bias is zero
            A_PB = np.concatenate([np.zeros((E, 3)), A_PB[:, 3:]], -1)
        pos[:, child] = wb_p
        quat[:, child] = wb_q
        if parent >= 0:
            p_PB = wb_p - pos[:, parent]
            V[:, child] = compose_velocity(V[:, parent], p_PB, V_PB)
            Ab[:, child] = compose_acceleration(Ab[:, parent], V[:, parent], p_PB, V_PB, A_PB)
        else:
            V[:, child] = V_PB
            Ab[:, child] = A_PB
    # body dynamics (sim/free_motion.py:680-719)
    R = qmatrix(qnormalize(quat))
    mass = np.broadcast_to(m.body_mass, (E, B))
    I6, I_Bo, c = spatial_inertia_body_origin(R, m.body_inertia[None], mass, m.body_com[None])
    f_b = np.einsum("ebij,ebj->ebi", I6, Ab)
    w = V[..., :3]
    bias = np.concatenate([np.cross(w, np.einsum("ebij,ebj->ebi", I_Bo, w)),
                           mass[..., None] * np.cross(w, np.cross(w, c))], -1)
    g = np.broadcast_to(m.gravity, (E, 3))[:, None, :]
    f_grav = np.concatenate([np.cross(c, mass[..., None] * g), mass[..., None] * g], -1)
    f_body = f_b + bias - f_grav
    # reverse pass (sim/free_motion.py:154-220, sim/sap_helpers.py:2090-2118)
    ft = np.zeros((E, B, 6))
    tau = np.zeros((E, n))
    for j in reversed(range(Jn)):
        parent, child = m.joint_parent[j], m.joint_child[j]
        ds = m.joint_qd_start[j]
        dim = m.joint_dof_dim[j, 0] + m.joint_dof_dim[j, 1]
        f_s = f_body[:, child] + ft[:, child] + body_f[:, child]
        for k in range(dim):
            tau[:, ds + k] = -(S[:, ds + k] * f_s).sum(-1) + joint_f[:, ds + k]
        if parent >= 0:
            ft[:, parent] += shift_force(f_s, pos[:, parent] - pos[:, child])
    # body Jacobians (sim/free_motion.py:722-765) and H = sum J^T I J (:843-1179)
    Jb = np.zeros((E, B, 6, n))
    for j in range(Jn):
        child = m.joint_child[j]
        jj = j
        while jj != -1:
            col_body = m.joint_child[jj]
            ds = m.joint_qd_start[jj]
            dim = m.joint_dof_dim[jj, 0] + m.joint_dof_dim[jj, 1]
            for k in range(dim):
                Jb[:, child, :, ds + k] = shift_velocity(S[:, ds + k], pos[:, child] - pos[:, col_body])
            jj = m.joint_ancestor[jj]
    H = np.einsum("ebri,ebrs,ebsj->eij", Jb, I6, Jb)
    A = H + np.einsum("ij,ej->eij", np.eye(n), np.broadcast_to(m.joint_armature, (E, n)))
    vdot = np.linalg.solve(A, tau[..., None])[..., 0]
    v_star = joint_qd + dt[:, None] * vdot
    return dict(v_star=v_star, vdot=vdot, A=A, tau=tau, pos=pos, quat=quat, V=V, Jb=Jb, S=S)


def contact_frame_rows(nrm):
    """(t1, t2, n) rows of _sap_make_from_one_unit_vector_z (sim/sap_helpers.py:467-503)."""
    out = np.zeros(nrm.shape[:-1] + (3, 3))
    a = np.abs(nrm)
    i = np.argmin(a, axis=-1)
    # ties resolve to the lowest index like the reference's strict '<' scan
    mn = np.take_along_axis(a, i[..., None], -1)[..., 0]
    mag = np.sqrt(1.0 - mn * mn)
    r = 1.0 / mag
    umin = np.take_along_axis(nrm, i[..., None], -1)[..., 0]
    s = -r * umin
    x, y, z = nrm[..., 0], nrm[..., 1], nrm[..., 2]
    zero = np.zeros_like(x)
    v0 = np.stack([zero, -r * z, r * y], -1)
    w0 = np.stack([mag, s * y, s * z], -1)
    v1 = np.stack([r * z, zero, -r * x], -1)
    w1 = np.stack([s * x, mag, s * z], -1)
    v2 = np.stack([-r * y, r * x, zero], -1)
    w2 = np.stack([s * x, s * y, mag], -1)
    v = np.where((i == 0)[..., None], v0, np.where((i == 1)[..., None], v1, v2))
    w = np.where((i == 0)[..., None], w0, np.where((i == 1)[..., None], w1, w2))
    out[..., 0, :] = v
    out[..., 1, :] = w
    out[..., 2, :] = nrm
    return out


def combine_mu(mu0, mu1):
    d = mu0 + mu1
    return np.where(d <= 1e-12, 0.0, 2.0 * mu0 * mu1 / np.where(d <= 1e-12, 1.0, d))


def combine_k(k0, k1):
    d = k0 + k1
    return np.where(d <= 1e-12, np.maximum(k0, k1), k0 * k1 / np.where(d <= 1e-12, 1.0, d))


def contact_jacobian(m: Model, fm: dict, contacts: dict, max_contacts: int, *, point_mode="witness_point",
                     weight_mode="body_inertia", fallback_mu=None, fallback_k=1e10, fallback_tau=0.0):
    """Scatter flat contacts into per-world slots in flat order and build
    their rows (sim/contact_jacobian.py:404-562) and weights (:153-251).
    Returns per-world arrays; slot order = order of the flat buffer."""
    E, B, n, C = fm["pos"].shape[0], m.bodies_per_world, m.dofs_per_world, max_contacts
    cnt = int(np.asarray(contacts["count"]).reshape(-1)[0])
    # the FP64 mirrors when the buffer carries them (sim/sap_runtime.py:241-264)
    f64 = all(k in contacts for k in ("point0d", "point1d", "normald", "margin0d", "margin1d"))
    P0 = contacts["point0d"] if f64 else contacts["point0"]
    P1 = contacts["point1d"] if f64 else contacts["point1"]
    NR = contacts["normald"] if f64 else contacts["normal"]
    M0 = contacts["margin0d"] if f64 else contacts["margin0"]
    M1 = contacts["margin1d"] if f64 else contacts["margin1"]
    sh0, sh1 = contacts["shape0"][:cnt], contacts["shape1"][:cnt]
    b0 = np.where(sh0 >= 0, m.shape_body_global[np.maximum(sh0, 0)], -1)
    b1 = np.where(sh1 >= 0, m.shape_body_global[np.maximum(sh1, 0)], -1)
    env = np.where(b0 >= 0, b0 // B, np.where(b1 >= 0, b1 // B, -1))
    ok = env >= 0
    ok &= ~((b0 >= 0) & (b0 // B != env)) & ~((b1 >= 0) & (b1 // B != env))
    out = dict(count=np.zeros(E, np.int32), jac=np.zeros((E, C, 3, n)), phi0=np.zeros((E, C)), mu=np.zeros((E, C)),
               k=np.zeros((E, C)), tau=np.zeros((E, C)), w=np.zeros((E, C)), body0=np.full((E, C), -1, np.int32),
               body1=np.full((E, C), -1, np.int32), point=np.zeros((E, C, 3)), frame=np.zeros((E, C, 3, 3)),
               truncated=0)
    fmu = 0.0 if fallback_mu is None else float(fallback_mu)
    Ainv_diag = 1.0 / np.maximum(np.einsum("eii->ei", fm["A"]), 1e-12)
    for t in range(cnt):
        if not ok[t]:
            continue
        e = env[t]
        slot = out["count"][e]
        out["count"][e] += 1
        if slot >= C:
            out["truncated"] += 1
            continue
        x0 = np.asarray(P0[t], np.float64)
        x1 = np.asarray(P1[t], np.float64)
        p0 = p1 = np.zeros(3)
        lb0 = b0[t] - e * B if b0[t] >= 0 else -1
        lb1 = b1[t] - e * B if b1[t] >= 0 else -1
        if lb0 >= 0:
            p0 = fm["pos"][e, lb0]
            x0 = p0 + qrotate(qnormalize(fm["quat"][e, lb0]), x0)
        if lb1 >= 0:
            p1 = fm["pos"][e, lb1]
            x1 = p1 + qrotate(qnormalize(fm["quat"][e, lb1]), x1)
        nrm = np.asarray(NR[t], np.float64)
        nn = np.linalg.norm(nrm)
        nrm = nrm / nn if nn > 0 else nrm
        F = contact_frame_rows(nrm)
        def mat(arr, sh, fb):
            v = fb if sh < 0 else float(arr[sh])
            return v
        k0 = mat(m.shape_ke, sh0[t], fallback_k)
        k1 = mat(m.shape_ke, sh1[t], fallback_k)
        k0 = k0 if np.isfinite(k0) and k0 > 0 else (fallback_k if fallback_k > 0 else 1.0)
        k1 = k1 if np.isfinite(k1) and k1 > 0 else (fallback_k if fallback_k > 0 else 1.0)
        den = k0 + k1
        w0, w1 = (k0 / den, k1 / den) if den != 0 else (0.5, 0.5)
        pC = w0 * x0 + w1 * x1
        mu0 = max(mat(m.shape_mu, sh0[t], fmu), 0.0)
        mu1 = max(mat(m.shape_mu, sh1[t], fmu), 0.0)
        t0 = mat(m.shape_tau, sh0[t], fallback_tau)
        t1 = mat(m.shape_tau, sh1[t], fallback_tau)
        t0 = t0 if np.isfinite(t0) and t0 >= 0 else max(fallback_tau, 0.0)
        t1 = t1 if np.isfinite(t1) and t1 >= 0 else max(fallback_tau, 0.0)
        xj0, xj1 = (x0, x1) if point_mode == "witness_point" else (pC, pC)
        rel = np.zeros((3, n))
        if lb0 >= 0:
            Jw = fm["Jb"][e, lb0]
            rel -= Jw[3:] - skew(xj0 - p0) @ Jw[:3]
        if lb1 >= 0:
            Jw = fm["Jb"][e, lb1]
            rel += Jw[3:] - skew(xj1 - p1) @ Jw[:3]
        J = F @ rel
        out["jac"][e, slot] = J
        out["phi0"][e, slot] = (x1 - x0) @ nrm - float(M0[t]) - float(M1[t])
        out["mu"][e, slot] = combine_mu(mu0, mu1)
        out["k"][e, slot] = combine_k(k0, k1)
        out["tau"][e, slot] = t0 + t1
        out["body0"][e, slot] = b0[t]
        out["body1"][e, slot] = b1[t]
        out["point"][e, slot] = pC
        out["frame"][e, slot] = F
        if weight_mode == "diag_delassus":
            W = (J * Ainv_diag[e]) @ J.T
            out["w"][e, slot] = max(np.linalg.norm(W) / 3.0, 1e-12)
        else:
            wsum = 0.0
            for lb, xw in ((lb0, x0), (lb1, x1)):
                if lb < 0:
                    continue
                mass = m.body_mass[lb]
                if mass <= 1e-12:
                    continue
                q = qnormalize(fm["quat"][e, lb])
                com = fm["pos"][e, lb] + qrotate(q, m.body_com[lb])
                r = xw - com
                I = np.maximum(np.diag(m.body_inertia[lb]), 1e-12)
                for d in range(3):
                    cb = qrotate(qconj(q), np.cross(r, F[d]))
                    wsum += 1.0 / mass + (cb * cb / I).sum()
            out["w"][e, slot] = max(wsum / 3.0, 1e-12)
    out["count_clamped"] = np.minimum(out["count"], C)
    return out


def integrate(m: Model, joint_q, v_prev, v_new, dt, mode="sap_euler"):
    """q_{n+1} (sim/solver_sap.py:288-733) for f64 state, SAP-order velocities."""
    q = joint_q.copy()
    for j in range(m.joints_per_world):
        jt, qs, ds = m.joint_type[j], m.joint_q_start[j], m.joint_qd_start[j]
        vel = v_new if mode == "sap_euler" else 0.5 * (v_prev + v_new)
        h = dt[:, None]
        if jt in (JOINT_PRISMATIC, JOINT_REVOLUTE):
            q[:, qs] = joint_q[:, qs] + dt * vel[:, ds]
        elif jt in (JOINT_BALL, JOINT_FREE, JOINT_DISTANCE):
            o = 0 if jt == JOINT_BALL else 3
            if jt != JOINT_BALL:
                q[:, qs:qs + 3] = joint_q[:, qs:qs + 3] + h * vel[:, ds + 3:ds + 6]
            qq = joint_q[:, qs + o:qs + o + 4]
            w = vel[:, ds:ds + 3]
            if mode == "sap_euler":
                x, y, z, s = qq[:, 0], qq[:, 1], qq[:, 2], qq[:, 3]
                hd = 0.5 * dt
                nx = x + hd * (s * w[:, 0] + w[:, 1] * z - w[:, 2] * y)
                ny = y + hd * (s * w[:, 1] + w[:, 2] * x - w[:, 0] * z)
                nz = z + hd * (s * w[:, 2] + w[:, 0] * y - w[:, 1] * x)
                ns = s - hd * (w[:, 0] * x + w[:, 1] * y + w[:, 2] * z)
                qn = np.stack([nx, ny, nz, ns], -1)
                q[:, qs + o:qs + o + 4] = qnormalize(qn)
            else:
                ang = np.linalg.norm(w, axis=-1) * dt
                axis = w / np.maximum(np.linalg.norm(w, axis=-1, keepdims=True), 1e-300)
                r = q_axis_angle(axis, ang)
                qn = qnormalize(qmul(r, qq))
                q[:, qs + o:qs + o + 4] = np.where((ang > 1e-12)[:, None], qn, qq)
        elif jt == JOINT_D6:  # scalar coordinates, one per axis (sim/solver_sap.py:379-383, 504-510)
            dim = int(m.joint_dof_dim[j, 0] + m.joint_dof_dim[j, 1])
            q[:, qs:qs + dim] = joint_q[:, qs:qs + dim] + h * vel[:, ds:ds + dim]
        elif jt == JOINT_FIXED:
            pass
    return q
