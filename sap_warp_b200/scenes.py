"""Seeded synthetic SAP problems with the shapes of the reference's workloads.

No public dataset or scene file is involved: the reference ships no benchmark
data, so every input here is generated from a seed.  The generators build a
real kinematic tree (free base + revolute chain), its mass matrix
A = M(q) + diag(armature) by the composite-rigid-body sum sum_b J_b^T I_b J_b,
and contact rows J_c = R_WC^T J_point(p) at random points of random bodies,
so A is SPD and J has the sparsity and scale of an articulated robot.

Conventions follow the reference: spatial velocities are [omega; v] at the
body origin, angular first (sim/sap_helpers.py:771-785); the free joint's six
DOFs come first in SAP order; contact rows are (t1, t2, n) with the normal
pointing from body0 (the ground, -1) to body1 (sim/contact_jacobian.py:404-562).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def _skew(v: np.ndarray) -> np.ndarray:
    """[v]x for a (..., 3) array -> (..., 3, 3)."""
    z = np.zeros(v.shape[:-1], dtype=v.dtype)
    return np.stack(
        [
            np.stack([z, -v[..., 2], v[..., 1]], -1),
            np.stack([v[..., 2], z, -v[..., 0]], -1),
            np.stack([-v[..., 1], v[..., 0], z], -1),
        ],
        -2,
    )


def _axis_angle(axis: np.ndarray, angle: np.ndarray) -> np.ndarray:
    """Rotation matrices (..., 3, 3) for unit axes (3,) or (...,3) and angles (...)."""
    axis = np.broadcast_to(axis, angle.shape + (3,))
    K = _skew(axis)
    s = np.sin(angle)[..., None, None]
    c = np.cos(angle)[..., None, None]
    eye = np.eye(3)
    return eye + s * K + (1.0 - c) * (K @ K)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    x, y, z, w = q.T
    return np.stack(
        [
            np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
            np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
            np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
        ],
        -2,
    )


@dataclass
class ChainModel:
    """A floating-base serial chain: body 0 is the base, body k>0 hangs from k-1
    by a revolute joint about `axis[k]` (parent frame) at offset `offset[k]`."""

    masses: np.ndarray  # (B,)
    inertia: np.ndarray  # (B, 3, 3) body-frame inertia about the COM
    com: np.ndarray  # (B, 3) COM in the body frame
    axis: np.ndarray  # (B, 3) joint axis in the parent frame (row 0 unused)
    offset: np.ndarray  # (B, 3) joint origin in the parent frame (row 0 unused)
    armature: float

    @property
    def bodies(self) -> int:
        return int(self.masses.shape[0])

    @property
    def dofs(self) -> int:
        return 6 + self.bodies - 1


def make_chain(rng: np.random.Generator, bodies: int, mass_range=(0.5, 2.0), link=0.12) -> ChainModel:
    masses = rng.uniform(*mass_range, size=bodies)
    masses[0] *= 4.0  # heavier torso/base
    # diagonal-dominant SPD inertia: R diag(d) R^T + delta I
    R = _random_rotations(rng, bodies)
    d = rng.uniform(0.5, 2.0, size=(bodies, 3)) * masses[:, None] * link * link / 6.0
    inertia = np.einsum("bij,bj,bkj->bik", R, d, R) + 1e-4 * np.eye(3)[None]
    com = rng.uniform(-0.5, 0.5, size=(bodies, 3)) * link * 0.5
    axis = rng.normal(size=(bodies, 3))
    axis /= np.linalg.norm(axis, axis=1, keepdims=True)
    off = rng.normal(size=(bodies, 3))
    off /= np.linalg.norm(off, axis=1, keepdims=True)
    off *= link
    return ChainModel(masses, inertia, com, axis, off, armature=0.01)


def chain_kinematics(model: ChainModel, q_base_R: np.ndarray, q_base_p: np.ndarray, q_joint: np.ndarray):
    """World rotations (E,B,3,3), origins (E,B,3) and the body Jacobians
    (E,B,6,n) mapping SAP-order generalized velocities to [omega; v_origin]."""
    E = q_joint.shape[0]
    B = model.bodies
    n = model.dofs
    Rw = np.zeros((E, B, 3, 3))
    ow = np.zeros((E, B, 3))
    Rw[:, 0] = q_base_R
    ow[:, 0] = q_base_p
    axes_w = np.zeros((E, B, 3))
    for k in range(1, B):
        Rp = Rw[:, k - 1]
        ow[:, k] = ow[:, k - 1] + np.einsum("eij,j->ei", Rp, model.offset[k])
        axes_w[:, k] = np.einsum("eij,j->ei", Rp, model.axis[k])
        Rw[:, k] = Rp @ _axis_angle(model.axis[k], q_joint[:, k - 1])
    Jb = np.zeros((E, B, 6, n))
    eye = np.eye(3)
    for k in range(B):
        # base angular DOFs 0..2 and linear DOFs 3..5 (world frame, base origin)
        Jb[:, k, 0:3, 0:3] = eye
        Jb[:, k, 3:6, 0:3] = -_skew(ow[:, k] - ow[:, 0])  # e x r = -[r]x e
        Jb[:, k, 3:6, 3:6] = eye
        for j in range(1, k + 1):
            a = axes_w[:, j]
            Jb[:, k, 0:3, 5 + j] = a
            Jb[:, k, 3:6, 5 + j] = np.cross(a, ow[:, k] - ow[:, j])
    return Rw, ow, Jb


def chain_mass_matrix(model: ChainModel, Rw: np.ndarray, ow: np.ndarray, Jb: np.ndarray) -> np.ndarray:
    """A = sum_b J_b^T I_b J_b + diag(armature on revolute DOFs), spatial
    inertia about the body origin in the world frame, angular first."""
    E, B = Rw.shape[:2]
    n = model.dofs
    A = np.zeros((E, n, n))
    for k in range(B):
        m = model.masses[k]
        c = np.einsum("eij,j->ei", Rw[:, k], model.com[k])  # COM offset, world
        Ic = Rw[:, k] @ model.inertia[k] @ np.swapaxes(Rw[:, k], -1, -2)
        cx = _skew(c)
        I6 = np.zeros((E, 6, 6))
        I6[:, 0:3, 0:3] = Ic + m * np.swapaxes(cx, -1, -2) @ cx
        I6[:, 0:3, 3:6] = m * cx
        I6[:, 3:6, 0:3] = m * np.swapaxes(cx, -1, -2)
        I6[:, 3:6, 3:6] = m * np.eye(3)
        A += np.swapaxes(Jb[:, k], -1, -2) @ I6 @ Jb[:, k]
    A[:, 6:, 6:] += model.armature * np.eye(n - 6)
    return 0.5 * (A + np.swapaxes(A, -1, -2))


def contact_frames(normals: np.ndarray) -> np.ndarray:
    """Rows (t1, t2, n) of an orthonormal frame with third axis = normal."""
    n = normals / np.linalg.norm(normals, axis=-1, keepdims=True)
    helper = np.where(np.abs(n[..., 0:1]) < 0.9, np.array([1.0, 0.0, 0.0]), np.array([0.0, 1.0, 0.0]))
    t1 = np.cross(helper, n)
    t1 /= np.linalg.norm(t1, axis=-1, keepdims=True)
    t2 = np.cross(n, t1)
    return np.stack([t1, t2, n], axis=-2)


@dataclass
class ContactProblemArrays:
    """Host arrays of one sapb_contact_problem (FP64 unless noted)."""

    num_envs: int
    dof_per_env: int
    max_contacts: int
    bodies_per_env: int
    contact_count: np.ndarray  # int32 (E,)
    dynamics_matrix: np.ndarray  # (E, n, n)
    jacobian: np.ndarray  # (E, C, 3, n)
    phi0: np.ndarray  # (E, C)
    w_eff: np.ndarray
    mu: np.ndarray
    stiffness: np.ndarray
    tau_d: np.ndarray
    body0: np.ndarray  # int32 (E, C)
    body1: np.ndarray
    body_dof_start: np.ndarray  # int32 (E*B,)
    body_dof_count: np.ndarray
    v_star: np.ndarray  # (E*n,)
    v0: np.ndarray
    dt: np.ndarray  # (E,)
    normal_up: np.ndarray | None = None  # (E, C) world-up component of the contact normal
    dofs_active: np.ndarray | None = None  # (E,) DOFs of each world before padding (mixed batches)

    def subset(self, worlds: np.ndarray) -> "ContactProblemArrays":
        """The same problem restricted to a list of worlds (bodies renumbered)."""
        worlds = np.asarray(worlds, dtype=np.int64)
        E, n, B = len(worlds), self.dof_per_env, self.bodies_per_env
        remap = lambda b: np.where(b >= 0, (b % B) + np.arange(E)[:, None] * B, -1).astype(np.int32)
        body_idx = (worlds[:, None] * B + np.arange(B)[None]).reshape(-1)
        dof_idx = (worlds[:, None] * n + np.arange(n)[None]).reshape(-1)
        return ContactProblemArrays(
            E, n, self.max_contacts, B,
            self.contact_count[worlds].copy(), self.dynamics_matrix[worlds].copy(), self.jacobian[worlds].copy(),
            self.phi0[worlds].copy(), self.w_eff[worlds].copy(), self.mu[worlds].copy(),
            self.stiffness[worlds].copy(), self.tau_d[worlds].copy(),
            remap(self.body0[worlds]), remap(self.body1[worlds]),
            self.body_dof_start[body_idx].copy(), self.body_dof_count[body_idx].copy(),
            self.v_star[dof_idx].copy(), self.v0[dof_idx].copy(), self.dt[worlds].copy(),
            None if self.normal_up is None else self.normal_up[worlds].copy(),
            None if self.dofs_active is None else self.dofs_active[worlds].copy(),
        )


def diag_delassus_weight(jac: np.ndarray, A: np.ndarray) -> np.ndarray:
    """w = max(||J diag(A)^-1 J^T||_F / 3, 1e-12) per contact
    (sim/contact_jacobian.py:153-251, the diag_delassus mode)."""
    dinv = 1.0 / np.clip(np.einsum("eii->ei", A), 1e-12, None)  # (E, n)
    W = np.einsum("ecrj,ej,eckj->ecrk", jac, dinv, jac)
    return np.maximum(np.linalg.norm(W, axis=(-2, -1)) / 3.0, 1e-12)


def humanoid_contact_problem(
    num_worlds: int,
    seed: int = 2,
    *,
    revolute: int = 29,
    contacts: tuple[int, int] = (8, 32),
    max_contacts: int = 32,
    dt: float = 2.0e-3,
    phi0_range=(-2.0e-3, 0.0),
    mu_range=(0.3, 1.0),
    v_star_std: float = 0.5,
    stiffness: float = 1.0e5,
    tau_d: float = 0.01,
    mass_range=(0.5, 2.0),
    counts: np.ndarray | None = None,
) -> ContactProblemArrays:
    """Batched floating-base serial-chain 'humanoid' worlds (6 + `revolute`
    DOFs, one tree per world) with a random pose q, A = M(q) + armature,
    C ~ U{contacts} foot/hand-style point contacts against the ground and
    v* ~ N(0, v_star_std)."""
    rng = np.random.default_rng(seed)
    model = make_chain(rng, revolute + 1, mass_range=mass_range)
    E, B, n, C = num_worlds, model.bodies, model.dofs, max_contacts
    base_R = _random_rotations(rng, E)
    base_p = np.stack([rng.uniform(-1, 1, E), rng.uniform(-1, 1, E), rng.uniform(0.8, 1.2, E)], -1)
    qj = rng.uniform(-1.0, 1.0, size=(E, B - 1))
    Rw, ow, Jb = chain_kinematics(model, base_R, base_p, qj)
    A = chain_mass_matrix(model, Rw, ow, Jb)

    count = rng.integers(contacts[0], contacts[1] + 1, size=E).astype(np.int32)
    if counts is not None:
        count = np.asarray(counts, dtype=np.int32).copy()
    count = np.minimum(count, C)
    # contacts favour the distal half of the chain (feet / hands)
    bodies = rng.integers(B // 2, B, size=(E, C))
    r_local = rng.normal(size=(E, C, 3))
    r_local *= (rng.uniform(0.0, 0.05, size=(E, C)) / np.linalg.norm(r_local, axis=-1))[..., None]
    Rb = np.take_along_axis(Rw, bodies[..., None, None], axis=1)  # (E,C,3,3)
    r_world = np.einsum("ecij,ecj->eci", Rb, r_local)
    normals = np.array([0.0, 0.0, 1.0]) + rng.normal(scale=0.1, size=(E, C, 3))
    frame = contact_frames(normals)  # (E,C,3,3) rows t1,t2,n
    Jsel = np.take_along_axis(Jb, bodies[..., None, None], axis=1)  # (E,C,6,n)
    J_point = Jsel[:, :, 3:6, :] - np.einsum("ecij,ecjk->ecik", _skew(r_world), Jsel[:, :, 0:3, :])
    jac = np.einsum("ecrj,ecjk->ecrk", frame, J_point)
    live = np.arange(C)[None, :] < count[:, None]
    jac *= live[..., None, None]

    phi0 = rng.uniform(*phi0_range, size=(E, C)) * live
    mu = rng.uniform(*mu_range, size=(E, C)) * live
    w_eff = diag_delassus_weight(jac, A) * live
    k = np.full((E, C), stiffness) * live
    tau = np.full((E, C), tau_d) * live
    body1 = np.where(live, bodies + np.arange(E)[:, None] * B, -1).astype(np.int32)
    body0 = np.full((E, C), -1, dtype=np.int32)
    v_star = rng.normal(scale=v_star_std, size=(E, n))
    v0 = v_star + rng.normal(scale=0.01, size=(E, n))
    return ContactProblemArrays(
        num_envs=E,
        dof_per_env=n,
        max_contacts=C,
        bodies_per_env=B,
        contact_count=count,
        dynamics_matrix=A,
        jacobian=jac,
        phi0=phi0,
        w_eff=w_eff,
        mu=mu,
        stiffness=k,
        tau_d=tau,
        body0=body0,
        body1=body1,
        body_dof_start=np.zeros(E * B, dtype=np.int32),
        body_dof_count=np.full(E * B, n, dtype=np.int32),
        v_star=v_star.reshape(-1),
        v0=v0.reshape(-1),
        dt=np.full(E, dt),
        normal_up=frame[:, :, 2, 2] * live,
    )


def quadruped_contact_problem(num_worlds: int, seed: int = 1, **kw) -> ContactProblemArrays:
    """18-DOF floating-base stand-in (6 + 12 revolute) with <= 16 contacts."""
    kw.setdefault("contacts", (4, 16))
    kw.setdefault("max_contacts", 16)
    kw.setdefault("mu_range", (0.5, 1.0))
    return humanoid_contact_problem(num_worlds, seed, revolute=12, **kw)


def arm_box_contact_problem(num_worlds: int, seed: int = 3, *, contacts=(2, 8), max_contacts: int = 8,
                            dt: float = 2.0e-3, phi0_range=(-2.0e-3, 0.0), mu_range=(0.3, 1.0),
                            v_star_std: float = 0.5, stiffness: float = 1.0e5, tau_d: float = 0.01,
                            counts: np.ndarray | None = None) -> ContactProblemArrays:
    """A 7-DOF fixed-base arm (serial chain, DOFs 0..6) and a 6-DOF free box
    (DOFs 7..12, [omega; v] at the box origin) held by gripper contacts
    between the arm's last link (body 7, shape0) and the box (body 8,
    shape1): two trees coupled into one clique by J = R (V_box(x) - V_arm(x)).
    A = blockdiag(M_arm(q), I_box) + armature on the arm."""
    rng = np.random.default_rng(seed)
    arm = make_chain(rng, 8)
    E, C, B = num_worlds, max_contacts, 9
    base_R = np.broadcast_to(np.eye(3), (E, 3, 3)).copy()
    base_p = np.tile([0.0, 0.0, 0.5], (E, 1))
    qj = rng.uniform(-1.0, 1.0, size=(E, 7))
    Rw, ow, Jb = chain_kinematics(arm, base_R, base_p, qj)
    A_arm = chain_mass_matrix(arm, Rw, ow, Jb)[:, 6:, 6:]  # the fixed base removes DOFs 0..5
    J_arm = Jb[:, :, :, 6:]  # (E, 8, 6, 7)
    m_box = rng.uniform(0.5, 2.0, size=E)
    R_box = _random_rotations(rng, E)
    d_box = rng.uniform(0.5, 2.0, size=(E, 3)) * m_box[:, None] * 0.1 ** 2 / 6.0
    I_box = np.einsum("eij,ej,ekj->eik", R_box, d_box, R_box)
    p_box = ow[:, 7] + rng.normal(scale=0.03, size=(E, 3))
    n = 13
    A = np.zeros((E, n, n))
    A[:, :7, :7] = A_arm
    A[:, 7:10, 7:10] = I_box
    A[:, 10:, 10:] = m_box[:, None, None] * np.eye(3)
    count = rng.integers(contacts[0], contacts[1] + 1, size=E).astype(np.int32)
    if counts is not None:
        count = np.asarray(counts, dtype=np.int32).copy()
    count = np.minimum(count, C)
    r_local = rng.normal(size=(E, C, 3))
    r_local *= (rng.uniform(0.0, 0.05, size=(E, C)) / np.linalg.norm(r_local, axis=-1))[..., None]
    x = p_box[:, None, :] + r_local
    normals = rng.normal(size=(E, C, 3))
    frame = contact_frames(normals)
    eye = np.broadcast_to(np.eye(3), (E, C, 3, 3))
    J_box = np.concatenate([-_skew(x - p_box[:, None, :]), eye], -1)  # v + w x r
    Jl = J_arm[:, 7]  # last link
    J_a = Jl[:, None, 3:6, :] - np.einsum("ecij,ejk->ecik", _skew(x - ow[:, 7][:, None, :]), Jl[:, 0:3, :])
    J_point = np.concatenate([-J_a, J_box], -1)  # (E, C, 3, 13): V1 - V0, body1 = box
    jac = np.einsum("ecrj,ecjk->ecrk", frame, J_point)
    live = np.arange(C)[None, :] < count[:, None]
    jac *= live[..., None, None]
    phi0 = rng.uniform(*phi0_range, size=(E, C)) * live
    mu = rng.uniform(*mu_range, size=(E, C)) * live
    w_eff = diag_delassus_weight(jac, A) * live
    env = np.arange(E)[:, None]
    body0 = np.where(live, env * B + 7, -1).astype(np.int32)
    body1 = np.where(live, env * B + 8, -1).astype(np.int32)
    start = np.tile(np.array([-1, 0, 0, 0, 0, 0, 0, 0, 7], np.int32), E)
    cnt_dof = np.tile(np.array([0, 7, 7, 7, 7, 7, 7, 7, 6], np.int32), E)
    v_star = rng.normal(scale=v_star_std, size=(E, n))
    return ContactProblemArrays(
        num_envs=E, dof_per_env=n, max_contacts=C, bodies_per_env=B, contact_count=count, dynamics_matrix=A,
        jacobian=jac, phi0=phi0, w_eff=w_eff, mu=mu, stiffness=np.full((E, C), stiffness) * live,
        tau_d=np.full((E, C), tau_d) * live, body0=body0, body1=body1, body_dof_start=start,
        body_dof_count=cnt_dof, v_star=v_star.reshape(-1),
        v0=(v_star + rng.normal(scale=0.01, size=(E, n))).reshape(-1), dt=np.full(E, dt),
        normal_up=frame[:, :, 2, 2] * live)


def pad_problem(p: ContactProblemArrays, n_max: int, C_max: int, B_max: int) -> ContactProblemArrays:
    """The same worlds with n_max DOFs, C_max slots and B_max bodies: the
    extra DOFs get an identity block in A, zero Jacobian columns and
    v* = v0 = 0, so they take no part in the solve and stay at zero; the
    solution of the real DOFs is unchanged."""
    E, n, C, B = p.num_envs, p.dof_per_env, p.max_contacts, p.bodies_per_env
    assert n <= n_max and C <= C_max and B <= B_max
    A = np.zeros((E, n_max, n_max))
    A[:, :n, :n] = p.dynamics_matrix
    A[:, n:, n:] = np.eye(n_max - n)
    J = np.zeros((E, C_max, 3, n_max))
    J[:, :C, :, :n] = p.jacobian
    pad_c = lambda a: np.pad(a, ((0, 0), (0, C_max - C)))
    remap = lambda b: np.where(b >= 0, (b // B) * B_max + b % B, -1).astype(np.int32)
    body_start = np.full((E, B_max), -1, np.int32)
    body_count = np.zeros((E, B_max), np.int32)
    body_start[:, :B] = p.body_dof_start.reshape(E, B)
    body_count[:, :B] = p.body_dof_count.reshape(E, B)
    pad_v = lambda v: np.pad(v.reshape(E, n), ((0, 0), (0, n_max - n))).reshape(-1)
    return ContactProblemArrays(
        num_envs=E, dof_per_env=n_max, max_contacts=C_max, bodies_per_env=B_max,
        contact_count=p.contact_count.copy(), dynamics_matrix=A, jacobian=J, phi0=pad_c(p.phi0),
        w_eff=pad_c(p.w_eff), mu=pad_c(p.mu), stiffness=pad_c(p.stiffness), tau_d=pad_c(p.tau_d),
        body0=np.pad(remap(p.body0), ((0, 0), (0, C_max - C)), constant_values=-1),
        body1=np.pad(remap(p.body1), ((0, 0), (0, C_max - C)), constant_values=-1),
        body_dof_start=body_start.reshape(-1), body_dof_count=body_count.reshape(-1), v_star=pad_v(p.v_star),
        v0=pad_v(p.v0), dt=p.dt.copy(), normal_up=None if p.normal_up is None else pad_c(p.normal_up),
        dofs_active=np.full(E, n, np.int32) if p.dofs_active is None else p.dofs_active.copy())


def concat_problems(parts) -> ContactProblemArrays:
    """One batch of problems with equal n, C and B (body indices renumbered)."""
    n, C, B = parts[0].dof_per_env, parts[0].max_contacts, parts[0].bodies_per_env
    assert all(q.dof_per_env == n and q.max_contacts == C and q.bodies_per_env == B for q in parts)
    offs = np.cumsum([0] + [q.num_envs for q in parts])
    shift = lambda b, o: np.where(b >= 0, b + o * B, -1).astype(np.int32)
    cat = lambda name: np.concatenate([getattr(q, name) for q in parts])
    return ContactProblemArrays(
        num_envs=int(offs[-1]), dof_per_env=n, max_contacts=C, bodies_per_env=B, contact_count=cat("contact_count"),
        dynamics_matrix=cat("dynamics_matrix"), jacobian=cat("jacobian"), phi0=cat("phi0"), w_eff=cat("w_eff"),
        mu=cat("mu"), stiffness=cat("stiffness"), tau_d=cat("tau_d"),
        body0=np.concatenate([shift(q.body0, o) for q, o in zip(parts, offs)]),
        body1=np.concatenate([shift(q.body1, o) for q, o in zip(parts, offs)]),
        body_dof_start=cat("body_dof_start"), body_dof_count=cat("body_dof_count"), v_star=cat("v_star"),
        v0=cat("v0"), dt=cat("dt"),
        normal_up=None if any(q.normal_up is None for q in parts) else cat("normal_up"),
        dofs_active=np.concatenate([q.dofs_active if q.dofs_active is not None else
                                    np.full(q.num_envs, q.dof_per_env, np.int32) for q in parts]))


def poisson_counts(rng: np.random.Generator, E: int, lam: float = 12.0, lo: int = 1, hi: int = 64) -> np.ndarray:
    return np.clip(rng.poisson(lam, size=E), lo, hi).astype(np.int32)


def mixed_contact_problem(num_worlds: int, seed: int = 3, max_contacts: int = 64):
    """The uneven batch: a third each of arm + box (13 DOF, 2-8 gripper
    contacts), quadruped (18 DOF) and humanoid (35 DOF) worlds, contacts of
    the last two ~ min(Poisson(12), max_contacts) (at least 1), padded to 35
    DOF and max_contacts slots.  Returns (problem, parts): parts are the
    unpadded per-kind problems in batch order."""
    rng = np.random.default_rng(seed)
    k = num_worlds // 3
    sizes = [k, k, num_worlds - 2 * k]
    arm = arm_box_contact_problem(sizes[0], seed=seed)
    quad = humanoid_contact_problem(sizes[1], seed=seed + 1, revolute=12, max_contacts=max_contacts,
                                    counts=poisson_counts(rng, sizes[1], hi=max_contacts), mu_range=(0.5, 1.0))
    hum = humanoid_contact_problem(sizes[2], seed=seed + 2, max_contacts=max_contacts,
                                   counts=poisson_counts(rng, sizes[2], hi=max_contacts))
    parts = [arm, quad, hum]
    B_max = max(q.bodies_per_env for q in parts)
    prob = concat_problems([pad_problem(q, 35, max_contacts, B_max) for q in parts])
    return prob, parts


def compact_problem(p: ContactProblemArrays) -> ContactProblemArrays:
    """A padded mixed batch (dofs_active set) in the layout of per-world DOF
    counts (sapb_contact_problem.dof_count): world e's A block and Jacobian
    rows stored compact, row stride dofs_active[e], at the start of its
    slots; per-DOF arrays unchanged (the world's DOFs first in its slots).
    The padding's identity block and zero columns are dropped."""
    assert p.dofs_active is not None
    E, n, C = p.num_envs, p.dof_per_env, p.max_contacts
    A = np.zeros((E, n * n))
    J = np.zeros((E, C * 3 * n))
    for e in range(E):
        ne = int(p.dofs_active[e])
        A[e, :ne * ne] = p.dynamics_matrix[e, :ne, :ne].reshape(-1)
        J[e, :C * 3 * ne] = p.jacobian[e, :, :, :ne].reshape(-1)
    q = ContactProblemArrays(**{f: getattr(p, f) for f in p.__dataclass_fields__})
    q.dynamics_matrix = A.reshape(E, n, n)
    q.jacobian = J.reshape(E, C, 3, n)
    return q


def work_order(prob: ContactProblemArrays) -> np.ndarray:
    """Worlds by descending estimated solve work n^3/3 + C n^2 (n the
    world's own DOF count): the order a persistent kernel should take them in
    so the biggest worlds do not finish last."""
    n = prob.dofs_active if prob.dofs_active is not None else np.full(prob.num_envs, prob.dof_per_env)
    C = np.minimum(prob.contact_count, prob.max_contacts).astype(np.float64)
    work = n.astype(np.float64) ** 3 / 3.0 + C * n.astype(np.float64) ** 2
    return np.argsort(-work, kind="stable").astype(np.int32)


@dataclass
class BlockedProblemArrays:
    """Host arrays of one sapb_blocked_problem: worlds of `trees_per_env`
    trees of `tree_dofs` DOFs, DOF order tree by tree (FP64 unless noted)."""

    num_envs: int
    trees_per_env: int
    tree_dofs: int
    max_contacts: int
    contact_count: np.ndarray  # int32 (E,)
    tree_mass: np.ndarray  # (E, T, NB, NB) diagonal blocks of A
    jacobian: np.ndarray  # (E, C, 3, 2 NB): columns of contact_tree[..., 0], then of [..., 1]
    contact_tree: np.ndarray  # int32 (E, C, 2), -1: static side
    phi0: np.ndarray  # (E, C)
    w_eff: np.ndarray
    mu: np.ndarray
    stiffness: np.ndarray
    tau_d: np.ndarray
    v_star: np.ndarray  # (E*n,)
    v0: np.ndarray
    dt: np.ndarray  # (E,)

    @property
    def dof_per_env(self) -> int:
        return self.trees_per_env * self.tree_dofs

    def to_dense(self) -> ContactProblemArrays:
        """The same problem in the dense layout of sapb_contact_problem (A with
        its zero blocks between trees, J rows over all n DOFs; body = tree)."""
        E, T, NB, C = self.num_envs, self.trees_per_env, self.tree_dofs, self.max_contacts
        n = T * NB
        A = np.zeros((E, T, NB, T, NB))
        idx = np.arange(T)
        A[:, idx, :, idx, :] = self.tree_mass.transpose(1, 0, 2, 3)
        Jd = np.zeros((E, C, 3, T, NB))
        for s in range(2):
            t = self.contact_tree[..., s]
            e_i, c_i = np.nonzero(t >= 0)
            Jd[e_i, c_i, :, t[e_i, c_i]] += self.jacobian[e_i, c_i, :, s * NB:(s + 1) * NB]
        body = lambda s: np.where(self.contact_tree[..., s] >= 0,
                                  self.contact_tree[..., s] + np.arange(E)[:, None] * T, -1).astype(np.int32)
        return ContactProblemArrays(
            num_envs=E, dof_per_env=n, max_contacts=C, bodies_per_env=T,
            contact_count=self.contact_count.astype(np.int32), dynamics_matrix=A.reshape(E, n, n),
            jacobian=Jd.reshape(E, C, 3, n), phi0=self.phi0, w_eff=self.w_eff, mu=self.mu,
            stiffness=self.stiffness, tau_d=self.tau_d, body0=body(0), body1=body(1),
            body_dof_start=np.tile((np.arange(T) * NB).astype(np.int32), E),
            body_dof_count=np.full(E * T, NB, dtype=np.int32), v_star=self.v_star, v0=self.v0, dt=self.dt,
        )

    def subset(self, worlds) -> "BlockedProblemArrays":
        worlds = np.asarray(worlds, dtype=np.int64)
        n = self.dof_per_env
        dof_idx = (worlds[:, None] * n + np.arange(n)[None]).reshape(-1)
        return BlockedProblemArrays(
            len(worlds), self.trees_per_env, self.tree_dofs, self.max_contacts,
            self.contact_count[worlds].copy(), self.tree_mass[worlds].copy(), self.jacobian[worlds].copy(),
            self.contact_tree[worlds].copy(), self.phi0[worlds].copy(), self.w_eff[worlds].copy(),
            self.mu[worlds].copy(), self.stiffness[worlds].copy(), self.tau_d[worlds].copy(),
            self.v_star[dof_idx].copy(), self.v0[dof_idx].copy(), self.dt[worlds].copy(),
        )


def _free_body_inertia(m: float, inertia_world: np.ndarray, r: np.ndarray) -> np.ndarray:
    """6x6 mass matrix of a free body in SAP coordinates [omega; v_origin]
    (world frame) with the COM at r from the body origin: [[I_c + m [r]x^T [r]x,
    m [r]x], [-m [r]x, m I]]."""
    S = _skew(r)
    M = np.zeros((6, 6))
    M[:3, :3] = inertia_world + m * S.T @ S
    M[:3, 3:] = m * S
    M[3:, :3] = -m * S
    M[3:, 3:] = m * np.eye(3)
    return M


def box_stack_problem(
    num_worlds: int,
    seed: int = 4,
    *,
    boxes: int = 64,
    max_contacts: int = 448,
    sites: tuple[int, int] = (12, 20),
    points_per_pair: tuple[int, int] = (4, 8),
    side_pairs: tuple[int, int] = (2, 8),
    size_range=(0.05, 0.2),
    density_range=(500.0, 2000.0),
    dt: float = 2.0e-3,
    phi0_range=(-2.0e-3, 0.0),
    mu_range=(0.3, 1.0),
    stiffness: float = 1.0e5,
    tau_d: float = 0.01,
    v_std: float = 0.05,
    gravity: float = -9.81,
) -> BlockedProblemArrays:
    """Worlds of `boxes` free boxes (6-DOF trees: n = 6 * boxes) stacked on a
    grid of sites on the ground.  Sizes U[size_range] m per axis, density
    U[density_range] kg/m^3, small random yaw; body origin at the centre of
    the bottom face (so each 6x6 block couples rotation and translation).
    Contacts: 4-8 points (<= 8 per touching pair) between each box and the
    box below it or the ground, plus a few side contacts (2-4 points,
    horizontal normal) between boxes of neighbouring stacks, which couple
    stacks and create fill in the factor.  v0 ~ N(0, v_std); v* = v0 + dt
    M^-1 f_gravity."""
    rng = np.random.default_rng(seed)
    E, T, NB, C = num_worlds, boxes, 6, max_contacts
    tm = np.zeros((E, T, NB, NB))
    jac = np.zeros((E, C, 3, 2 * NB))
    ct = np.full((E, C, 2), -1, dtype=np.int32)
    count = np.zeros(E, dtype=np.int32)
    v0 = rng.normal(scale=v_std, size=(E, T * NB))
    v_star = v0.copy()
    g = np.array([0.0, 0.0, gravity])
    for e in range(E):
        S = int(rng.integers(sites[0], sites[1] + 1))
        grid = int(np.ceil(np.sqrt(S)))
        site_xy = np.stack([(np.arange(S) % grid) * 0.35, (np.arange(S) // grid) * 0.35], -1)
        site_of = rng.integers(0, S, size=T)
        dims = rng.uniform(*size_range, size=(T, 3))
        rho = rng.uniform(*density_range, size=T)
        mass = rho * dims.prod(-1)
        yaw = rng.uniform(-0.3, 0.3, size=T)
        R = _axis_angle(np.array([0.0, 0.0, 1.0]), yaw)
        origin = np.zeros((T, 3))
        below = np.full(T, -1)
        top_z = np.zeros(S)
        top_box = np.full(S, -1)
        for k in range(T):
            s = site_of[k]
            origin[k] = [site_xy[s, 0] + rng.normal(scale=0.01), site_xy[s, 1] + rng.normal(scale=0.01), top_z[s]]
            below[k] = top_box[s]
            top_z[s] += dims[k, 2]
            top_box[s] = k
        for k in range(T):
            a, b, c = dims[k]
            Ic = mass[k] / 12.0 * np.diag([b * b + c * c, a * a + c * c, a * a + b * b])
            r = R[k] @ np.array([0.0, 0.0, 0.5 * c])
            M = _free_body_inertia(mass[k], R[k] @ Ic @ R[k].T, r)
            tm[e, k] = M
            f = np.concatenate([np.cross(r, mass[k] * g), mass[k] * g])
            v_star[e, k * NB:(k + 1) * NB] += dt * np.linalg.solve(M, f)
        rows = []  # (tree0, tree1, point, normal)
        for k in range(T):
            lo = below[k]
            hx = 0.45 * min(dims[k, 0], dims[lo, 0] if lo >= 0 else 1.0)
            hy = 0.45 * min(dims[k, 1], dims[lo, 1] if lo >= 0 else 1.0)
            npts = int(rng.integers(points_per_pair[0], points_per_pair[1] + 1))
            local = np.array([[hx, hy], [-hx, hy], [-hx, -hy], [hx, -hy]])
            if npts > 4:
                local = np.concatenate([local, rng.uniform(-1, 1, size=(npts - 4, 2)) * [hx, hy]])
            for p2 in local[:npts]:
                p = origin[k] + R[k] @ np.array([p2[0], p2[1], 0.0])
                nrm = np.array([0.0, 0.0, 1.0]) + (rng.normal(scale=0.02, size=3) if lo >= 0 else 0.0)
                rows.append((lo, k, p, nrm / np.linalg.norm(nrm)))
        for _ in range(int(rng.integers(side_pairs[0], side_pairs[1] + 1))):
            s0 = int(rng.integers(0, S))
            nb = [s for s in (s0 + 1, s0 + grid) if s < S and (s != s0 + 1 or (s0 + 1) % grid != 0)]
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
                p = mid + np.array([0.0, 0.0, zlo + rng.uniform(0.0, 0.05)]) - np.array([0.0, 0.0, mid[2]])
                p[:2] += rng.normal(scale=0.02, size=2) * np.array([-nrm[1], nrm[0]])
                rows.append((u, w, p, nrm))
        cnt = min(len(rows), C)
        count[e] = cnt
        for c, (t0, t1, p, nrm) in enumerate(rows[:cnt]):
            fr = contact_frames(nrm[None])[0]
            ct[e, c] = (t0, t1)
            for s, t in ((0, t0), (1, t1)):
                if t < 0:
                    continue
                Jp = np.concatenate([-_skew(p - origin[t]), np.eye(3)], axis=1)  # v_p = v_o + w x (p - o)
                jac[e, c, :, s * NB:(s + 1) * NB] = (1.0 if s == 1 else -1.0) * fr @ Jp
    live = np.arange(C)[None, :] < count[:, None]
    # diag_delassus weights over the columns of the contact's trees
    dA = np.einsum("etii->eti", tm)
    dinv = 1.0 / np.clip(dA, 1e-12, None)  # (E, T, NB)
    W = np.zeros((E, C, 3, 3))
    for s in range(2):
        t = np.maximum(ct[..., s], 0)
        d = np.take_along_axis(dinv, t[..., None], axis=1) * (ct[..., s] >= 0)[..., None]  # (E, C, NB)
        Js = jac[..., s * NB:(s + 1) * NB]
        W += np.einsum("ecrj,ecj,eckj->ecrk", Js, d, Js)
    w_eff = np.maximum(np.linalg.norm(W, axis=(-2, -1)) / 3.0, 1e-12) * live
    return BlockedProblemArrays(
        num_envs=E, trees_per_env=T, tree_dofs=NB, max_contacts=C, contact_count=count,
        tree_mass=tm, jacobian=jac, contact_tree=ct,
        phi0=rng.uniform(*phi0_range, size=(E, C)) * live, w_eff=w_eff,
        mu=rng.uniform(*mu_range, size=(E, C)) * live, stiffness=np.full((E, C), stiffness) * live,
        tau_d=np.full((E, C), tau_d) * live, v_star=v_star.reshape(-1), v0=v0.reshape(-1), dt=np.full(E, dt),
    )
