"""Seeded synthetic models of the reference's workload shapes, as SapModel
(torch) and as plain numpy dictionaries, plus a ground-contact generator
that writes the flat SapContacts buffer the way the reference's collision
writer does (witness points in the body frames of their shapes, normal from
shape0 to shape1; sim/collision/pipeline.py:52-118).

No scene file or dataset is involved: the reference's robot assets are
fetched over the network and its benchmark data is synthetic, so every model
here is generated from a seed.
"""

from __future__ import annotations

import numpy as np
import torch

from .runtime import (
    SAP_JOINT_BALL,
    SAP_JOINT_D6,
    SAP_JOINT_DISTANCE,
    SAP_JOINT_FREE,
    SAP_JOINT_PRISMATIC,
    SAP_JOINT_REVOLUTE,
    SapContacts,
    SapModel,
)

_IDENT7 = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0])


def _random_unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _random_quat(rng, n):
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def _spd_inertia(rng, m, link):
    from .scenes import _random_rotations

    R = _random_rotations(rng, 1)[0]
    d = rng.uniform(0.5, 2.0, size=3) * m * link * link / 6.0
    return R @ np.diag(d) @ R.T + 1e-4 * np.eye(3)


def world_template(kind: str, rng: np.random.Generator, *, random_child_frames: bool = False,
                   boxes: int = 64) -> dict:
    """One world's topology and inertia (numpy).  kind: 'humanoid' (free base
    + 29-revolute serial chain, 35 DOF), 'quadruped' (free base + 4 legs x 3
    revolute, 18 DOF), 'box' (one free box, 6 DOF), 'boxes' (`boxes` free
    bodies, each its own tree: 6 * boxes DOF), 'arm_box' (7-revolute
    fixed-base arm + free box, 13 DOF), 'arm_boxes' (the arm and `boxes`
    free boxes: 7 + 6 * boxes DOF in 1 + boxes trees), 'slider' (free base + prismatic +
    revolute chain), 'joints' (a chain through every mobilizer kind: free
    base, ball, D6 (1 translation + 2 rotations), distance, D6 (2 + 1), D6
    (3 rotations), revolute, D6 (3 translations), prismatic; 29 DOF)."""
    joints = []  # (type, parent_body, axis or None, X_p, X_c)
    link = 0.12
    if kind == "humanoid":
        joints.append((SAP_JOINT_FREE, -1, None))
        for b in range(1, 30):
            joints.append((SAP_JOINT_REVOLUTE, b - 1, None))
    elif kind == "quadruped":
        joints.append((SAP_JOINT_FREE, -1, None))
        for leg in range(4):
            for k in range(3):
                parent = 0 if k == 0 else len(joints) - 1
                joints.append((SAP_JOINT_REVOLUTE, parent, None))
    elif kind == "box":
        joints.append((SAP_JOINT_FREE, -1, None))
    elif kind == "boxes":
        for _ in range(boxes):
            joints.append((SAP_JOINT_FREE, -1, None))
    elif kind in ("arm_box", "arm_boxes"):
        for k in range(7):
            joints.append((SAP_JOINT_REVOLUTE, k - 1, None))
        for _ in range(1 if kind == "arm_box" else boxes):
            joints.append((SAP_JOINT_FREE, -1, None))
    elif kind == "slider":
        joints.append((SAP_JOINT_FREE, -1, None))
        joints.append((SAP_JOINT_PRISMATIC, 0, None))
        for b in range(2, 6):
            joints.append((SAP_JOINT_REVOLUTE, b - 1, None))
    elif kind == "joints":
        joints.append((SAP_JOINT_FREE, -1, None))
        joints.append((SAP_JOINT_BALL, 0, None))
        joints.append((SAP_JOINT_D6, 1, (1, 2)))
        joints.append((SAP_JOINT_DISTANCE, 2, None))
        joints.append((SAP_JOINT_D6, 3, (2, 1)))
        joints.append((SAP_JOINT_D6, 4, (0, 3)))
        joints.append((SAP_JOINT_REVOLUTE, 5, None))
        joints.append((SAP_JOINT_D6, 6, (3, 0)))
        joints.append((SAP_JOINT_PRISMATIC, 7, None))
    else:
        raise ValueError(kind)
    B = len(joints)
    jtype = np.array([j[0] for j in joints], np.int32)
    parent = np.array([j[1] for j in joints], np.int32)
    axis_per_joint = _random_unit(rng, B)
    X_p = np.tile(_IDENT7, (B, 1))
    X_c = np.tile(_IDENT7, (B, 1))
    for k in range(B):
        if parent[k] >= 0:
            X_p[k, :3] = _random_unit(rng, 1)[0] * link
            if random_child_frames:
                X_p[k, 3:] = _random_quat(rng, 1)[0]
        elif jtype[k] != SAP_JOINT_FREE:
            X_p[k, :3] = [0.0, 0.0, 0.5]
        if random_child_frames:
            X_c[k, :3] = _random_unit(rng, 1)[0] * 0.03
            X_c[k, 3:] = _random_quat(rng, 1)[0]
    mass = rng.uniform(0.5, 2.0, size=B)
    if kind in ("humanoid", "quadruped", "slider", "joints"):
        mass[0] *= 4.0
    inertia = np.stack([_spd_inertia(rng, mass[b], link) for b in range(B)])
    com = rng.uniform(-0.5, 0.5, size=(B, 3)) * link * 0.5
    dofdim = np.zeros((B, 2), np.int32)
    ncoord = np.zeros(B, np.int32)
    for k in range(B):
        if jtype[k] == SAP_JOINT_FREE:
            dofdim[k] = (3, 3)
            ncoord[k] = 7
        elif jtype[k] == SAP_JOINT_REVOLUTE:
            dofdim[k] = (0, 1)
            ncoord[k] = 1
        elif jtype[k] == SAP_JOINT_PRISMATIC:
            dofdim[k] = (1, 0)
            ncoord[k] = 1
        elif jtype[k] == SAP_JOINT_BALL:
            dofdim[k] = (0, 3)
            ncoord[k] = 4
        elif jtype[k] == SAP_JOINT_DISTANCE:
            dofdim[k] = (3, 3)
            ncoord[k] = 7
        elif jtype[k] == SAP_JOINT_D6:
            dofdim[k] = joints[k][2]
            ncoord[k] = sum(joints[k][2])
    ndof = dofdim.sum(1)
    qd_start = np.concatenate([[0], np.cumsum(ndof)]).astype(np.int32)
    q_start = np.concatenate([[0], np.cumsum(ncoord)]).astype(np.int32)
    n = int(qd_start[-1])
    axis = np.zeros((n, 3))
    for k in range(B):
        if jtype[k] in (SAP_JOINT_REVOLUTE, SAP_JOINT_PRISMATIC):
            axis[qd_start[k]] = axis_per_joint[k]
        elif jtype[k] == SAP_JOINT_D6:
            lin, ang = joints[k][2]
            axis[qd_start[k]:qd_start[k] + lin] = _random_unit(rng, lin) if lin else axis[:0]
            if ang:  # rotation axes: columns of a random rotation
                qr = _random_quat(rng, 1)[0]
                cols = np.stack([_qrot(qr, e) for e in np.eye(3)])
                axis[qd_start[k] + lin:qd_start[k] + lin + ang] = cols[:ang]
    # joint ancestor: the joint whose child is this joint's parent body
    child = np.arange(B, dtype=np.int32)
    ancestor = np.array([parent[k] if parent[k] >= 0 else -1 for k in range(B)], np.int32)
    # articulations: roots start new ones (joints ordered parent before child)
    art_start = [k for k in range(B) if parent[k] < 0] + [B]
    armature = np.where(np.repeat(jtype == SAP_JOINT_FREE, ndof), 0.0, 0.01)
    return dict(kind=kind, joint_type=jtype, joint_parent=parent, joint_child=child, joint_ancestor=ancestor,
                joint_q_start=q_start, joint_qd_start=qd_start, joint_dof_dim=dofdim, joint_axis=axis,
                joint_X_p=X_p, joint_X_c=X_c, body_mass=mass, body_inertia=inertia, body_com=com,
                joint_armature=armature, articulation_start=np.array(art_start, np.int32),
                bodies_per_world=B, joints_per_world=B, dofs_per_world=n, coords_per_world=int(q_start[-1]))


def random_joint_q(tpl: dict, rng: np.random.Generator, worlds: int, spread: float = 0.05) -> np.ndarray:
    """Coordinates per world: free bases at height ~1 m with random yaw/tilt,
    revolute/prismatic coordinates ~ N(0, spread) around a random rest pose."""
    Q = tpl["coords_per_world"]
    q = np.zeros((worlds, Q))
    rest = rng.uniform(-1.0, 1.0, size=Q)
    for k, jt in enumerate(tpl["joint_type"]):
        qs = tpl["joint_q_start"][k]
        if jt == SAP_JOINT_FREE:
            q[:, qs:qs + 3] = np.stack([rng.uniform(-1, 1, worlds), rng.uniform(-1, 1, worlds),
                                        rng.uniform(0.8, 1.2, worlds)], -1)
            q[:, qs + 3:qs + 7] = _random_quat(rng, worlds)
        elif jt == SAP_JOINT_BALL:
            q[:, qs:qs + 4] = _random_quat(rng, worlds)
        elif jt == SAP_JOINT_DISTANCE:
            q[:, qs:qs + 3] = rng.normal(scale=0.05, size=(worlds, 3))
            q[:, qs + 3:qs + 7] = _random_quat(rng, worlds)
        elif jt == SAP_JOINT_D6:
            dim = int(tpl["joint_dof_dim"][k].sum())
            q[:, qs:qs + dim] = rest[qs:qs + dim] + rng.normal(scale=spread, size=(worlds, dim))
        else:
            q[:, qs] = rest[qs] + rng.normal(scale=spread, size=worlds)
    return q


def replicate(tpl: dict, worlds: int, rng: np.random.Generator, *, gravity=(0.0, 0.0, -9.81),
              mu_range=(0.3, 1.0), stiffness=1.0e5, tau_d=0.005) -> dict:
    """Global (all-worlds) numpy arrays in the reference's layout: equal
    contiguous per-world blocks of joints, bodies, coordinates and DOFs.  Each
    body owns one shape; shape index S-1 is a static ground (body -1)."""
    B, Jw, n, Q = tpl["bodies_per_world"], tpl["joints_per_world"], tpl["dofs_per_world"], tpl["coords_per_world"]
    E = worlds
    g = {}
    off = lambda a, step: (a[None, :] + step * np.arange(E)[:, None]).reshape(-1)
    g["joint_type"] = np.tile(tpl["joint_type"], E)
    g["joint_parent"] = np.where(np.tile(tpl["joint_parent"], E) >= 0, off(tpl["joint_parent"], B), -1).astype(np.int32)
    g["joint_child"] = off(tpl["joint_child"], B).astype(np.int32)
    g["joint_ancestor"] = np.where(np.tile(tpl["joint_ancestor"], E) >= 0, off(tpl["joint_ancestor"], Jw),
                                   -1).astype(np.int32)
    g["joint_articulation"] = np.zeros(E * Jw, np.int32)
    qs = np.concatenate([off(tpl["joint_q_start"][:-1], Q), [E * Q]]).astype(np.int32)
    ds = np.concatenate([off(tpl["joint_qd_start"][:-1], n), [E * n]]).astype(np.int32)
    g["joint_q_start"], g["joint_qd_start"] = qs, ds
    g["joint_dof_dim"] = np.tile(tpl["joint_dof_dim"], (E, 1))
    g["joint_axis"] = np.tile(tpl["joint_axis"], (E, 1))
    g["joint_X_p"] = np.tile(tpl["joint_X_p"], (E, 1))
    g["joint_X_c"] = np.tile(tpl["joint_X_c"], (E, 1))
    g["joint_armature"] = np.tile(tpl["joint_armature"], E)
    arts = tpl["articulation_start"]
    A_w = len(arts) - 1
    starts = (arts[:-1][None, :] + Jw * np.arange(E)[:, None]).reshape(-1)
    g["articulation_start"] = np.concatenate([starts, [E * Jw]]).astype(np.int32)
    for a in range(E * A_w):
        g["joint_articulation"][g["articulation_start"][a]:g["articulation_start"][a + 1]] = a
    g["body_mass"] = np.tile(tpl["body_mass"], E)
    g["body_inertia"] = np.tile(tpl["body_inertia"], (E, 1, 1))
    g["body_com"] = np.tile(tpl["body_com"], (E, 1))
    g["body_world"] = np.repeat(np.arange(E, dtype=np.int32), B)
    g["gravity"] = np.tile(np.asarray(gravity, np.float64), (E, 1))
    S = E * B + 1
    g["shape_body"] = np.concatenate([np.arange(E * B), [-1]]).astype(np.int32)
    g["shape_material_mu"] = np.concatenate([rng.uniform(*mu_range, E * B), [1.0]])
    g["shape_material_ke"] = np.full(S, 2.0 * stiffness)  # series combination halves it
    g["shape_material_tau"] = np.full(S, tau_d)
    g["counts"] = dict(joints=E * Jw, dofs=E * n, coords=E * Q, bodies=E * B, articulations=E * A_w, worlds=E,
                       shapes=S)
    return g


def to_model(tpl: dict, g: dict, joint_q: np.ndarray, device) -> SapModel:
    """SapModel (torch) from the numpy arrays of `replicate`."""
    c = g["counts"]
    t64 = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=device)
    t32 = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device=device)
    ti = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.int32, device=device)
    D = c["dofs"]
    return SapModel(
        device=device, joint_count=c["joints"], joint_dof_count=D, joint_coord_count=c["coords"],
        body_count=c["bodies"], articulation_count=c["articulations"], world_count=c["worlds"],
        shape_count=c["shapes"], requires_grad=False,
        joint_type=ti(g["joint_type"]), joint_articulation=ti(g["joint_articulation"]),
        joint_parent=ti(g["joint_parent"]), joint_child=ti(g["joint_child"]),
        joint_q_start=ti(g["joint_q_start"]), joint_qd_start=ti(g["joint_qd_start"]),
        joint_dof_dim=ti(g["joint_dof_dim"]), joint_axis=t64(g["joint_axis"]), joint_X_p=t64(g["joint_X_p"]),
        joint_X_c=t64(g["joint_X_c"]), joint_ancestor=ti(g["joint_ancestor"]),
        articulation_start=ti(g["articulation_start"]), joint_q=t64(joint_q.reshape(-1)),
        joint_qd=torch.zeros(D, dtype=torch.float64, device=device),
        body_q=torch.zeros(c["bodies"], 7, dtype=torch.float64, device=device),
        body_qd=torch.zeros(c["bodies"], 6, dtype=torch.float64, device=device),
        body_mass=t64(g["body_mass"]), body_inertia=t64(g["body_inertia"]), body_com=t64(g["body_com"]),
        body_flags=torch.ones(c["bodies"], dtype=torch.int32, device=device), body_world=ti(g["body_world"]),
        gravity=t64(g["gravity"]), joint_armature=t64(g["joint_armature"]), shape_body=ti(g["shape_body"]),
        shape_material_mu=t64(g["shape_material_mu"]), shape_material_ke=t64(g["shape_material_ke"]),
        shape_material_tau=t64(g["shape_material_tau"]),
        joint_target_mode=torch.zeros(D, dtype=torch.int32, device=device),
        joint_target_ke=torch.zeros(D, dtype=torch.float32, device=device),
        joint_target_kd=torch.zeros(D, dtype=torch.float32, device=device),
        joint_target_pos=torch.zeros(D, dtype=torch.float32, device=device),
        joint_target_vel=torch.zeros(D, dtype=torch.float32, device=device),
        joint_f=torch.zeros(D, dtype=torch.float64, device=device),
        joint_act=torch.zeros(D, dtype=torch.float32, device=device),
        joint_effort_limit=torch.zeros(D, dtype=torch.float32, device=device),
        joint_limit_lower=torch.full((D,), -np.inf, dtype=torch.float64, device=device),
        joint_limit_upper=torch.full((D,), np.inf, dtype=torch.float64, device=device),
        joint_limit_ke=torch.zeros(D, dtype=torch.float64, device=device),
        joint_limit_kd=torch.zeros(D, dtype=torch.float64, device=device),
    )


def _qrot(q, v):
    qv = q[..., :3]
    t = 2.0 * np.cross(qv, v)
    return v + q[..., 3:4] * t + np.cross(qv, t)


def ground_contacts(rng: np.random.Generator, body_pos: np.ndarray, body_quat: np.ndarray, per_world, *,
                    bodies_from: int = 0, phi0_range=(-2e-3, 0.0), tilt: float = 0.1, shuffle: bool = True,
                    capacity: int | None = None) -> dict:
    """Flat contact buffer of body-vs-ground contacts.  body_pos (E,B,3),
    body_quat (E,B,4) are the body poses of the step's start state;
    per_world: int or (E,) counts.  shape0 = ground (static), shape1 = the
    body's shape, point1 in the body frame, point0 in world (its shape is
    static), normal ~ +z from ground to body, (x1 - x0).n = phi0."""
    E, B = body_pos.shape[:2]
    counts = np.broadcast_to(np.asarray(per_world), (E,)).astype(np.int64)
    N = int(counts.sum())
    world = np.repeat(np.arange(E), counts)
    body = rng.integers(bodies_from, B, size=N)
    r_local = rng.normal(size=(N, 3))
    r_local *= (rng.uniform(0.0, 0.05, size=N) / np.linalg.norm(r_local, axis=1))[:, None]
    q = body_quat[world, body]
    q = q / np.linalg.norm(q, axis=1, keepdims=True)
    x1 = body_pos[world, body] + _qrot(q, r_local)
    nrm = np.array([0.0, 0.0, 1.0]) + rng.normal(scale=tilt, size=(N, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    phi0 = rng.uniform(*phi0_range, size=N)
    x0 = x1 - phi0[:, None] * nrm
    order = rng.permutation(N) if shuffle else np.arange(N)
    cap = max(capacity or N, N)
    def pad(a, fill=0):
        out = np.full((cap,) + a.shape[1:], fill, dtype=a.dtype)
        out[:N] = a[order]
        return out
    ground_shape = E * B
    return dict(
        count=np.array([N], np.int32),
        shape0=pad(np.full(N, ground_shape, np.int32), -1),
        shape1=pad((world * B + body).astype(np.int32), -1),
        point0=pad(x0.astype(np.float32)), point1=pad(r_local.astype(np.float32)),
        normal=pad(nrm.astype(np.float32)),
        margin0=pad(np.zeros(N, np.float32)), margin1=pad(np.zeros(N, np.float32)),
        point0d=pad(x0), point1d=pad(r_local), normald=pad(nrm),
        margin0d=pad(np.zeros(N)), margin1d=pad(np.zeros(N)),
    )


def contacts_to_torch(c: dict, device, *, with_f64: bool = True) -> SapContacts:
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=device)
    kw = dict(
        rigid_contact_count=t(c["count"], torch.int32), rigid_contact_shape0=t(c["shape0"], torch.int32),
        rigid_contact_shape1=t(c["shape1"], torch.int32), rigid_contact_point0=t(c["point0"], torch.float32),
        rigid_contact_point1=t(c["point1"], torch.float32), rigid_contact_normal=t(c["normal"], torch.float32),
        rigid_contact_margin0=t(c["margin0"], torch.float32), rigid_contact_margin1=t(c["margin1"], torch.float32),
    )
    if with_f64:
        kw.update(rigid_contact_point0d=t(c["point0d"], torch.float64),
                  rigid_contact_point1d=t(c["point1d"], torch.float64),
                  rigid_contact_normald=t(c["normald"], torch.float64),
                  rigid_contact_margin0d=t(c["margin0d"], torch.float64),
                  rigid_contact_margin1d=t(c["margin1d"], torch.float64))
    return SapContacts(**kw)


def rollout_scene(kind: str, worlds: int, seed: int, device, *, contacts=(8, 32), qd_std: float = 0.5,
                  phi0_range=(-2.0e-3, 0.0), mu_range=(0.3, 1.0), stiffness: float = 1.0e5, tau_d: float = 0.01,
                  tilt: float = 0.1, dt: float = 2.0e-3):
    """A batch of `worlds` copies of `kind` with random poses, joint
    velocities ~ N(0, qd_std) and C ~ U{contacts} body-vs-ground point
    contacts per world on the distal half of the bodies, phi0 ~ U[phi0_range]
    at the start, pair stiffness `stiffness`, pair dissipation time `tau_d`.
    Body poses come from one free-motion pass on the device.  Returns
    (model, state, control, contacts (SapContacts), host contact dict)."""
    from .runtime import SapContacts, SapControl, SapState
    from .solver import SapContactJacobian

    rng = np.random.default_rng(seed)
    tpl = world_template(kind, rng)
    g = replicate(tpl, worlds, rng, mu_range=mu_range, stiffness=stiffness, tau_d=0.5 * tau_d)
    q = random_joint_q(tpl, rng, worlds)
    n, B = tpl["dofs_per_world"], tpl["bodies_per_world"]
    model = to_model(tpl, g, q, device)
    qd = rng.normal(scale=qd_std, size=(worlds, n))
    state = SapState(joint_q=torch.as_tensor(q.reshape(-1), dtype=torch.float64, device=device),
                     joint_qd=torch.as_tensor(qd.reshape(-1), dtype=torch.float64, device=device),
                     body_q=model.body_q.clone(),
                     body_f=torch.zeros(model.body_count, 6, dtype=torch.float64, device=device))
    control = SapControl(joint_f=torch.zeros(model.joint_dof_count, dtype=torch.float64, device=device))
    cj = SapContactJacobian(model, max_rigid_contact=1, fallback_tau_d=0.0)
    cj.compute(state, SapContacts(), control=control, dt=dt)
    bq = cj.body_q_sap.reshape(worlds, B, 7).cpu().numpy()
    counts = rng.integers(contacts[0], contacts[1] + 1, size=worlds)
    con = ground_contacts(rng, bq[..., :3], bq[..., 3:], counts, bodies_from=B // 2, phi0_range=phi0_range,
                          tilt=tilt, capacity=int(counts.sum()))
    return model, state, control, contacts_to_torch(con, device), con


def _quat_from_z(n: np.ndarray) -> np.ndarray:
    """Unit quaternions (xyzw) rotating +z onto the unit vectors n (N, 3)."""
    z = np.array([0.0, 0.0, 1.0])
    axis = np.cross(z, n)
    s = np.linalg.norm(axis, axis=1)
    c = n[:, 2]
    ang = np.arctan2(s, c)
    u = np.where(s[:, None] > 1e-15, axis / np.maximum(s, 1e-300)[:, None], np.array([1.0, 0.0, 0.0]))
    return np.concatenate([u * np.sin(0.5 * ang)[:, None], np.cos(0.5 * ang)[:, None]], axis=1)


def site_scene(kind: str, worlds: int, seed: int, device, *, sites: int = 32, contacts=(8, 32),
               radius: float = 0.01, qd_std: float = 0.5, phi0_range=(-2.0e-3, 0.0), lift_range=(5.0e-3, 3.0e-2),
               mu_range=(0.3, 1.0), stiffness: float = 1.0e5, tau_d: float = 0.01, tilt: float = 0.1):
    """A batch of `kind` worlds whose contacts come from collision shapes and
    are regenerated from the pose every step: `sites` spheres of radius
    `radius` on the distal half of each world's bodies, each over its own
    static ground patch (a plane through a ground point, normal ~ +z tilted
    by `tilt`), a sphere and its patch sharing a collision group so that
    only those pairs are tested.  At the start C ~ U{contacts} sites per
    world touch their patch (phi0 ~ U[phi0_range]) and the others hover
    U[lift_range] above theirs; as the bodies move, contacts vanish and
    appear.  Materials as rollout_scene's (pair stiffness, dissipation).
    Returns (model, state, control, shapes (collision.ShapeSet), host)."""
    from ._abi import SAPB_SHAPE_PLANE, SAPB_SHAPE_SPHERE
    from .collision import ShapeSet
    from .runtime import SapContacts, SapControl, SapState
    from .solver import SapContactJacobian

    rng = np.random.default_rng(seed)
    tpl = world_template(kind, rng)
    g = replicate(tpl, worlds, rng, mu_range=mu_range, stiffness=stiffness, tau_d=0.5 * tau_d)
    q = random_joint_q(tpl, rng, worlds)
    n, B = tpl["dofs_per_world"], tpl["bodies_per_world"]
    E, K = worlds, int(sites)
    # shapes: per world K spheres (on bodies), then K static patches
    S = E * 2 * K
    shape_body = np.full(S, -1, np.int32)
    bodies = rng.integers(B // 2, B, size=(E, K))
    gidx = (np.arange(E)[:, None] * B + bodies)
    sph = (np.arange(E)[:, None] * 2 * K + np.arange(K)[None, :])
    shape_body[sph.reshape(-1)] = gidx.reshape(-1)
    g["shape_body"] = shape_body
    g["shape_material_mu"] = np.ones(S)
    g["shape_material_mu"][sph.reshape(-1)] = rng.uniform(*mu_range, E * K)
    g["shape_material_ke"] = np.full(S, 2.0 * stiffness)
    g["shape_material_tau"] = np.full(S, 0.5 * tau_d)
    g["counts"] = dict(g["counts"], shapes=S)
    model = to_model(tpl, g, q, device)
    qd = rng.normal(scale=qd_std, size=(worlds, n))
    state = SapState(joint_q=torch.as_tensor(q.reshape(-1), dtype=torch.float64, device=device),
                     joint_qd=torch.as_tensor(qd.reshape(-1), dtype=torch.float64, device=device),
                     body_q=model.body_q.clone(),
                     body_f=torch.zeros(model.body_count, 6, dtype=torch.float64, device=device))
    control = SapControl(joint_f=torch.zeros(model.joint_dof_count, dtype=torch.float64, device=device))
    cj = SapContactJacobian(model, max_rigid_contact=1, fallback_tau_d=0.0)
    cj.compute(state, SapContacts(), control=control, dt=2.0e-3)
    bq = cj.body_q_sap.reshape(worlds, B, 7).cpu().numpy()
    counts = rng.integers(contacts[0], contacts[1] + 1, size=worlds)
    # sites: a point on the body (within 5 cm of its origin), its patch
    # through the point moved by phi along the patch normal
    r_local = rng.normal(size=(E, K, 3))
    r_local *= (rng.uniform(0.0, 0.05, size=(E, K)) / np.linalg.norm(r_local, axis=2))[..., None]
    bp = bq[np.arange(E)[:, None], bodies]
    bquat = bp[..., 3:] / np.linalg.norm(bp[..., 3:], axis=-1, keepdims=True)
    x1 = bp[..., :3] + _qrot(bquat, r_local)
    nrm = np.array([0.0, 0.0, 1.0]) + rng.normal(scale=tilt, size=(E, K, 3))
    nrm /= np.linalg.norm(nrm, axis=2, keepdims=True)
    touching = np.arange(K)[None, :] < counts[:, None]
    phi = np.where(touching, rng.uniform(*phi0_range, size=(E, K)), rng.uniform(*lift_range, size=(E, K)))
    x0 = x1 - phi[..., None] * nrm
    # sphere centre = the site point plus the radius along the normal, in the body frame
    conj = bquat * np.array([-1.0, -1.0, -1.0, 1.0])
    centre_local = r_local + _qrot(conj, radius * nrm)
    X = np.zeros((S, 7))
    scale = np.zeros((S, 3))
    types = np.full(S, SAPB_SHAPE_PLANE, np.int32)
    groups = np.zeros(S, np.int32)
    for w in range(E):
        base = w * 2 * K
        X[base:base + K, :3] = centre_local[w]
        X[base:base + K, 6] = 1.0
        X[base + K:base + 2 * K, :3] = x0[w]
        X[base + K:base + 2 * K, 3:] = _quat_from_z(nrm[w])
        scale[base:base + K, 0] = radius
        types[base:base + K] = SAPB_SHAPE_SPHERE
        groups[base:base + K] = 1 + np.arange(K)
        groups[base + K:base + 2 * K] = 1 + np.arange(K)
    shapes = ShapeSet(num_worlds=E, shapes_per_world=2 * K, num_global_shapes=0, shape_type=types,
                      shape_scale=scale, shape_X_bs=X, shape_body=shape_body, shape_collision_group=groups)
    host = dict(tpl=tpl, g=g, q=q, qd=qd, counts=counts, phi=phi, sites=K)
    return model, state, control, shapes, host


def _quat_z(yaw: np.ndarray) -> np.ndarray:
    """Quaternions (x, y, z, w) of rotations about +z."""
    z = np.zeros_like(yaw)
    return np.stack([z, z, np.sin(0.5 * yaw), np.cos(0.5 * yaw)], -1)


def box_scene(worlds: int, seed: int, device, *, boxes: int = 64, sites=(12, 20), points_per_pair=(4, 8),
              side_pairs=(2, 8), size_range=(0.05, 0.2), density_range=(500.0, 2000.0), v_std: float = 0.05,
              phi0_range=(-2.0e-3, 0.0), mu_range=(0.3, 1.0), stiffness: float = 1.0e5, tau_d: float = 0.01,
              arm: bool = False, gripper=(2, 8)):
    """Worlds of `boxes` free boxes stacked on a grid of sites on the ground
    (the model behind scenes.box_stack_problem, as a SapModel with a flat
    contact buffer): box sizes U[size_range] m per axis, density
    U[density_range], small random yaw, body origin at the centre of the
    bottom face; 4-8 contact points between each box and the box below it
    (or the ground), plus a few side contacts between boxes of neighbouring
    stacks; witness points in the body frames of their shapes, normal from
    shape0 to shape1, phi0 ~ U[phi0_range]; joint velocities ~ N(0, v_std).
    arm: the world also holds a 7-revolute fixed-base arm (bodies 0-6, the
    boxes after it: 7 + 6 * boxes DOFs in 1 + boxes trees) whose last link
    grips one box through U{gripper} contacts, which couple the arm's tree
    with the box's.
    Returns (model, state, control, contacts, host contact dict, host arrays
    dict(tpl, g, q, qd))."""
    from .runtime import SapControl, SapState
    from .scenes import _axis_angle

    rng = np.random.default_rng(seed)
    E, B = worlds, boxes
    a0 = 7 if arm else 0  # first box body
    Bt = B + a0           # bodies (and shapes) per world
    tpl = world_template("arm_boxes" if arm else "boxes", rng, boxes=B)
    g = replicate(tpl, E, rng, mu_range=mu_range, stiffness=stiffness, tau_d=0.5 * tau_d)
    Q = tpl["coords_per_world"]
    q = np.zeros((E, Q))
    ground = E * Bt
    rows = []  # (world, lower box or -1, upper box, x1 world, normal)
    pos_all = np.zeros((E, B, 3))
    R_all = np.zeros((E, B, 3, 3))
    dims_all = np.zeros((E, B, 3))
    for e in range(E):
        S = int(rng.integers(sites[0], sites[1] + 1))
        grid = int(np.ceil(np.sqrt(S)))
        site_xy = np.stack([(np.arange(S) % grid) * 0.35, (np.arange(S) // grid) * 0.35], -1)
        site_of = rng.integers(0, S, size=B)
        dims = rng.uniform(*size_range, size=(B, 3))
        dims_all[e] = dims
        mass = rng.uniform(*density_range, size=B) * dims.prod(-1)
        yaw = rng.uniform(-0.3, 0.3, size=B)
        R = _axis_angle(np.array([0.0, 0.0, 1.0]), yaw)
        origin = np.zeros((B, 3))
        below = np.full(B, -1)
        top_z = np.zeros(S)
        top_box = np.full(S, -1)
        for k in range(B):
            st = site_of[k]
            origin[k] = [site_xy[st, 0] + rng.normal(scale=0.01), site_xy[st, 1] + rng.normal(scale=0.01), top_z[st]]
            below[k] = top_box[st]
            top_z[st] += dims[k, 2]
            top_box[st] = k
        sl = slice(e * Bt + a0, (e + 1) * Bt)
        a, b, c = dims[:, 0], dims[:, 1], dims[:, 2]
        g["body_mass"][sl] = mass
        g["body_inertia"][sl] = (mass / 12.0)[:, None, None] * np.stack(
            [np.diag(v) for v in np.stack([b * b + c * c, a * a + c * c, a * a + b * b], -1)])
        g["body_com"][sl] = np.stack([np.zeros(B), np.zeros(B), 0.5 * c], -1)
        q7 = q[e, a0:].reshape(B, 7)
        q7[:, :3] = origin
        q7[:, 3:] = _quat_z(yaw)
        pos_all[e], R_all[e] = origin, R
        for k in range(B):
            lo = below[k]
            hx = 0.45 * min(dims[k, 0], dims[lo, 0] if lo >= 0 else 1.0)
            hy = 0.45 * min(dims[k, 1], dims[lo, 1] if lo >= 0 else 1.0)
            npts = int(rng.integers(points_per_pair[0], points_per_pair[1] + 1))
            local = np.array([[hx, hy], [-hx, hy], [-hx, -hy], [hx, -hy]])
            if npts > 4:
                local = np.concatenate([local, rng.uniform(-1, 1, size=(npts - 4, 2)) * [hx, hy]])
            for p2 in local[:npts]:
                x1 = origin[k] + R[k] @ np.array([p2[0], p2[1], 0.0])
                nrm = np.array([0.0, 0.0, 1.0]) + (rng.normal(scale=0.02, size=3) if lo >= 0 else 0.0)
                rows.append((e, lo, k, x1, nrm / np.linalg.norm(nrm)))
        for _ in range(int(rng.integers(side_pairs[0], side_pairs[1] + 1))):
            s0 = int(rng.integers(0, S))
            nb = [t for t in (s0 + 1, s0 + grid) if t < S and (t != s0 + 1 or (s0 + 1) % grid != 0)]
            if not nb:
                continue
            s1 = nb[int(rng.integers(0, len(nb)))]
            in0, in1 = np.nonzero(site_of == s0)[0], np.nonzero(site_of == s1)[0]
            if len(in0) == 0 or len(in1) == 0:
                continue
            u, w = int(rng.choice(in0)), int(rng.choice(in1))
            d = origin[w] - origin[u]
            d[2] = 0.0
            nrm = d / max(np.linalg.norm(d), 1e-9)
            mid = 0.5 * (origin[u] + origin[w])
            zlo = max(origin[u, 2], origin[w, 2])
            for _p in range(int(rng.integers(2, 5))):
                x1 = np.array([mid[0], mid[1], zlo + rng.uniform(0.0, 0.05)])
                x1[:2] += rng.normal(scale=0.02, size=2) * np.array([-nrm[1], nrm[0]])
                rows.append((e, u, w, x1, nrm))
    N = len(rows)
    phi0 = rng.uniform(*phi0_range, size=N)
    shape0 = np.array([r[0] * Bt + a0 + r[1] if r[1] >= 0 else ground for r in rows], np.int32)
    shape1 = np.array([r[0] * Bt + a0 + r[2] for r in rows], np.int32)
    x1 = np.stack([r[3] for r in rows])
    nrm = np.stack([r[4] for r in rows])
    x0 = x1 - phi0[:, None] * nrm
    ew = np.array([r[0] for r in rows])
    lo = np.array([r[1] for r in rows])
    up = np.array([r[2] for r in rows])
    Ru = R_all[ew, up]
    p1 = np.einsum("nji,nj->ni", Ru, x1 - pos_all[ew, up])
    Rl = R_all[ew, np.maximum(lo, 0)]
    p0 = np.where((lo >= 0)[:, None], np.einsum("nji,nj->ni", Rl, x0 - pos_all[ew, np.maximum(lo, 0)]), x0)
    if arm:
        q[:, :a0] = rng.uniform(-1.0, 1.0, size=a0)[None, :] + rng.normal(scale=0.05, size=(E, a0))
    model = to_model(tpl, g, q, device)
    if arm:
        # the arm's last link grips one box: x1 inside the box, x0 = x1 -
        # phi0 n in the link's frame (its pose from one free-motion pass)
        from .runtime import SapContacts as _SC
        from .solver import SapContactJacobian

        st0 = SapState(joint_q=torch.as_tensor(q.reshape(-1), dtype=torch.float64, device=device),
                       joint_qd=torch.zeros(model.joint_dof_count, dtype=torch.float64, device=device),
                       body_q=model.body_q.clone())
        ctl0 = SapControl(joint_f=torch.zeros(model.joint_dof_count, dtype=torch.float64, device=device))
        cj = SapContactJacobian(model, max_rigid_contact=1, fallback_tau_d=0.0)
        cj.compute(st0, _SC(), control=ctl0, dt=2.0e-3)
        link = cj.body_q_sap.reshape(E, Bt, 7)[:, a0 - 1].cpu().numpy()
        gs, gp0, gp1, gn = [], [], [], []
        for e in range(E):
            u = int(rng.integers(0, B))
            Rl6 = _quat_to_matrix(link[e, 3:])
            for _ in range(int(rng.integers(gripper[0], gripper[1] + 1))):
                r = rng.uniform(-0.4, 0.4, size=3) * dims_all[e, u] + np.array([0.0, 0.0, 0.5 * dims_all[e, u, 2]])
                xb = pos_all[e, u] + R_all[e, u] @ r
                nv = _random_unit(rng, 1)[0]
                ph = rng.uniform(*phi0_range)
                xa = xb - ph * nv
                gs.append((e * Bt + a0 - 1, e * Bt + a0 + u))
                gp0.append(Rl6.T @ (xa - link[e, :3]))
                gp1.append(r)
                gn.append(nv)
        M = len(gs)
        shape0 = np.concatenate([shape0, np.array([t[0] for t in gs], np.int32)])
        shape1 = np.concatenate([shape1, np.array([t[1] for t in gs], np.int32)])
        p0 = np.concatenate([p0, np.stack(gp0)])
        p1 = np.concatenate([p1, np.stack(gp1)])
        nrm = np.concatenate([nrm, np.stack(gn)])
        N += M
    z = np.zeros(N)
    con = dict(count=np.array([N], np.int32), shape0=shape0, shape1=shape1, point0=p0.astype(np.float32),
               point1=p1.astype(np.float32), normal=nrm.astype(np.float32), margin0=z.astype(np.float32),
               margin1=z.astype(np.float32), point0d=p0, point1d=p1, normald=nrm, margin0d=z, margin1d=z.copy())
    qd = rng.normal(scale=v_std, size=(E, tpl["dofs_per_world"]))
    state = SapState(joint_q=torch.as_tensor(q.reshape(-1), dtype=torch.float64, device=device),
                     joint_qd=torch.as_tensor(qd.reshape(-1), dtype=torch.float64, device=device),
                     body_q=model.body_q.clone(),
                     body_f=torch.zeros(model.body_count, 6, dtype=torch.float64, device=device))
    control = SapControl(joint_f=torch.zeros(model.joint_dof_count, dtype=torch.float64, device=device))
    return model, state, control, contacts_to_torch(con, device), con, dict(tpl=tpl, g=g, q=q, qd=qd, dims=dims_all)


def _quat_to_matrix(q: np.ndarray) -> np.ndarray:
    """Rotation matrix of a unit quaternion (x, y, z, w)."""
    x, y, z, w = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def box_shapes(host: dict):
    """collision.ShapeSet of a box_scene: one box shape per body (centred half
    a height above the body origin, which sits at the bottom face) and a
    static ground plane z = 0 shared by all worlds."""
    from .collision import ShapeSet
    from ._abi import SAPB_SHAPE_BOX, SAPB_SHAPE_PLANE

    if host["tpl"]["kind"] != "boxes":
        raise ValueError("box_shapes takes the host arrays of a box_scene without an arm")
    dims = host["dims"]
    E, B = dims.shape[:2]
    X = np.zeros((E * B + 1, 7))
    X[:, 6] = 1.0
    X[:E * B, 2] = 0.5 * dims.reshape(-1, 3)[:, 2]
    scale = np.zeros((E * B + 1, 3))
    scale[:E * B] = 0.5 * dims.reshape(-1, 3)
    return ShapeSet(num_worlds=E, shapes_per_world=B, num_global_shapes=1,
                    shape_type=np.concatenate([np.full(E * B, SAPB_SHAPE_BOX), [SAPB_SHAPE_PLANE]]).astype(np.int32),
                    shape_scale=scale, shape_X_bs=X,
                    shape_body=np.concatenate([np.arange(E * B), [-1]]).astype(np.int32))


def concat_models(parts) -> SapModel:
    """One uneven batch from models of equal-block worlds (each of one or
    more worlds, of any sizes): the global arrays concatenated, their body,
    joint, DOF, coordinate, articulation and world indices shifted, and the
    per-world offsets (world_*_start) set."""
    import dataclasses

    dev = parts[0].device
    cat = lambda name: torch.cat([getattr(m, name) for m in parts])
    offs = {k: np.cumsum([0] + [int(getattr(m, k)) for m in parts]) for k in
            ("joint_count", "body_count", "joint_dof_count", "joint_coord_count", "articulation_count",
             "world_count", "shape_count")}

    def shifted(name, key, keep_negative=True):
        out = []
        for i, m in enumerate(parts):
            t = getattr(m, name)
            o = int(offs[key][i])
            out.append(torch.where(t >= 0, t + o, t) if keep_negative else t + o)
        return torch.cat(out)

    def starts(name, key):  # [N+1] prefix arrays
        out = [getattr(m, name)[:-1] + int(offs[key][i]) for i, m in enumerate(parts)]
        out.append(torch.tensor([int(offs[key][-1])], dtype=parts[0].__getattribute__(name).dtype, device=dev))
        return torch.cat(out)

    def world_starts(key):
        w = []
        for i, m in enumerate(parts):
            W = int(m.world_count)
            per = int(getattr(m, key)) // W
            w.extend(int(offs[key][i]) + per * np.arange(W))
        w.append(int(offs[key][-1]))
        return torch.as_tensor(np.asarray(w), dtype=torch.int32, device=dev)

    f = {fl.name: getattr(parts[0], fl.name) for fl in dataclasses.fields(SapModel)}
    for name in ("joint_count", "body_count", "joint_dof_count", "joint_coord_count", "articulation_count",
                 "world_count", "shape_count"):
        f[name] = int(offs[name][-1])
    for name in ("joint_type", "joint_dof_dim", "joint_axis", "joint_X_p", "joint_X_c", "joint_q", "joint_qd",
                 "body_q", "body_qd", "body_mass", "body_inertia", "body_com", "body_flags", "gravity",
                 "joint_armature", "joint_target_mode", "joint_target_ke", "joint_target_kd", "joint_target_pos",
                 "joint_target_vel", "joint_f", "joint_act", "joint_effort_limit", "joint_limit_lower",
                 "joint_limit_upper", "joint_limit_ke", "joint_limit_kd"):
        f[name] = cat(name)
    for name in ("shape_material_mu", "shape_material_ke", "shape_material_tau"):
        f[name] = None if any(getattr(m, name) is None for m in parts) else cat(name)
    f["joint_parent"] = shifted("joint_parent", "body_count")
    f["joint_child"] = shifted("joint_child", "body_count")
    f["joint_ancestor"] = shifted("joint_ancestor", "joint_count")
    f["joint_articulation"] = shifted("joint_articulation", "articulation_count")
    f["body_world"] = shifted("body_world", "world_count", keep_negative=False)
    f["shape_body"] = shifted("shape_body", "body_count")
    f["joint_q_start"] = starts("joint_q_start", "joint_coord_count")
    f["joint_qd_start"] = starts("joint_qd_start", "joint_dof_count")
    f["articulation_start"] = starts("articulation_start", "joint_count")
    f["world_joint_start"] = world_starts("joint_count")
    f["world_body_start"] = world_starts("body_count")
    f["world_dof_start"] = world_starts("joint_dof_count")
    f["world_articulation_start"] = world_starts("articulation_count")
    f["body_label"], f["joint_label"] = (), ()
    return SapModel(**f)


def concat_contacts(parts, shape_offsets) -> "SapContacts":
    """The live contacts of several flat buffers in one (shape indices
    shifted by each part's shape offset); synchronous (test and bench set-up)."""
    from .runtime import SapContacts

    names = [k for k in vars(parts[0]) if isinstance(getattr(parts[0], k), torch.Tensor) and k != "rigid_contact_count"]
    counts = [int(c.rigid_contact_count.item()) for c in parts]
    out = {}
    for k in names:
        seg = []
        for c, n, o in zip(parts, counts, shape_offsets):
            t = getattr(c, k)[:n]
            if k in ("rigid_contact_shape0", "rigid_contact_shape1"):
                t = torch.where(t >= 0, t + int(o), t)
            seg.append(t)
        out[k] = torch.cat(seg).contiguous()
    cnt = torch.tensor([sum(counts)], dtype=torch.int32, device=parts[0].rigid_contact_count.device)
    return SapContacts(rigid_contact_count=cnt, **out)


def with_drives(model: SapModel, state, control, rng: np.random.Generator, *, ke=(10.0, 1.0e3), kd=(0.1, 10.0),
                effort: float = 5.0, limit: float = 0.3, limit_ke: float = 1.0e4, limit_kd: float = 10.0):
    """The model with a drive on every revolute and prismatic DOF (gains
    U[ke], U[kd], effort limit `effort`) and joint limits +-`limit` around
    the state's coordinate there (stiffness limit_ke, damping limit_kd), and
    the control with drive targets near that coordinate (target velocities
    ~ N(0, 1)).  Returns (model, control)."""
    import dataclasses

    from .runtime import SapControl

    jt = model.joint_type.cpu().numpy()
    ds, qs = model.joint_qd_start.cpu().numpy(), model.joint_q_start.cpu().numpy()
    q = state.joint_q.cpu().numpy()
    D = int(model.joint_dof_count)
    on = np.zeros(D, bool)
    q_at = np.zeros(D)
    for j, t in enumerate(jt):
        if t in (SAP_JOINT_REVOLUTE, SAP_JOINT_PRISMATIC):
            on[ds[j]] = True
            q_at[ds[j]] = q[qs[j]]
    dev = model.joint_type.device
    f32 = lambda a: torch.as_tensor(np.asarray(a, np.float32), device=dev)
    f64 = lambda a: torch.as_tensor(np.asarray(a, np.float64), device=dev)
    m2 = dataclasses.replace(
        model, joint_target_mode=torch.as_tensor(on.astype(np.int32), device=dev),
        joint_target_ke=f32(np.where(on, rng.uniform(*ke, D), 0.0)),
        joint_target_kd=f32(np.where(on, rng.uniform(*kd, D), 0.0)),
        joint_effort_limit=f32(np.where(on, effort, 0.0)),
        joint_limit_lower=f64(np.where(on, q_at - limit, -np.inf)),
        joint_limit_upper=f64(np.where(on, q_at + limit, np.inf)),
        joint_limit_ke=f64(np.where(on, limit_ke, 0.0)), joint_limit_kd=f64(np.where(on, limit_kd, 0.0)))
    c2 = SapControl(joint_f=control.joint_f, joint_target_pos=f32(np.where(on, q_at + rng.uniform(-0.2, 0.2, D), 0.0)),
                    joint_target_vel=f32(np.where(on, rng.normal(size=D), 0.0)))
    return m2, c2


def mixed_rollout_scene(worlds_per_kind, seed: int, device, kinds=("arm_box", "quadruped", "humanoid"),
                        drives: bool = False, **kw):
    """An uneven batch of rollout scenes: `worlds_per_kind` worlds of each
    kind (arm + box 13 DOF, quadruped 18, humanoid 35 by default), their
    models, states, controls and contacts concatenated; drives: each part
    with_drives (seeded).  Returns (model, state, control, contacts, parts)
    with parts the per-kind (model, state, control, contacts)."""
    from .runtime import SapControl, SapState

    parts = [rollout_scene(k, worlds_per_kind, seed + i, device, **kw)[:4] for i, k in enumerate(kinds)]
    if drives:
        rng = np.random.default_rng(seed + 100)
        driven = []
        for pm, ps, pc, pcon in parts:
            dm, dc = with_drives(pm, ps, pc, rng)
            driven.append((dm, ps, dc, pcon))
        parts = driven
    models_ = [p[0] for p in parts]
    model = concat_models(models_)
    state = SapState(joint_q=torch.cat([p[1].joint_q for p in parts]), joint_qd=torch.cat([p[1].joint_qd for p in parts]),
                     body_q=torch.cat([p[1].body_q for p in parts]), body_f=torch.cat([p[1].body_f for p in parts]))
    cat = lambda name: (torch.cat([getattr(p[2], name) for p in parts])
                        if all(getattr(p[2], name) is not None for p in parts) else None)
    control = SapControl(joint_f=cat("joint_f"), joint_target_pos=cat("joint_target_pos"),
                         joint_target_vel=cat("joint_target_vel"))
    shape_offs = np.cumsum([0] + [int(m.shape_count) for m in models_])[:-1]
    contacts = concat_contacts([p[3] for p in parts], shape_offs)
    return model, state, control, contacts, parts
