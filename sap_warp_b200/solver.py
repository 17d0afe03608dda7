"""Drop-in SAP step API: SolverSAP and its components, mirroring
sim/solver_sap.py, sim/free_motion.py, sim/contact_jacobian.py and
sim/contact_solve.py of the reference (constructor keywords, presets,
result dataclasses, errors), running on the native library only.

Every buffer is allocated in the constructors; `step` / `compute` / `solve`
only launch kernels on the current torch stream (no host synchronisation,
no allocation), so a whole step can be captured in a CUDA graph.
"""

from __future__ import annotations

import ctypes
import os
import warnings
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._lib import check, load
from ._solve import F32, F64, I32, normalize_sap_line_search_mode
from .runtime import (
    SAP_JOINT_D6,
    SAP_JOINT_DISTANCE,
    SAP_JOINT_FREE,
    SAP_JOINT_PRISMATIC,
    SAP_JOINT_REVOLUTE,
    SAP_JOINT_TARGET_NONE,
    SapContacts,
    SapControl,
    SapModel,
    SapState,
    sap_contacts_from_newton,
)

SAP_CONTACT_PRESET_VARIANTS = ("approx32", "approx64", "drake")

# sim/solver_sap.py:75-106
_CONTACT_PRESET_KWARGS = {
    "approx32": dict(use_f64_boundary_pose=False, free_motion_solve_precision="fp32", contact_solve_precision="fp64",
                     contact_linear_solve_precision="fp32", sap_contact_weight_precision="fp32",
                     contact_weight_mode="body_inertia", contact_point_mode="witness_point",
                     position_integration="midpoint"),
    "approx64": dict(use_f64_boundary_pose=True, free_motion_solve_precision="fp64", contact_solve_precision="fp64",
                     contact_linear_solve_precision="fp64", sap_contact_weight_precision="fp64",
                     contact_weight_mode="body_inertia", contact_point_mode="witness_point",
                     position_integration="midpoint"),
    "drake": dict(use_f64_boundary_pose=True, free_motion_solve_precision="fp64", contact_solve_precision="fp64",
                  contact_linear_solve_precision="fp64", sap_contact_weight_precision="fp64",
                  contact_weight_mode="diag_delassus", contact_point_mode="contact_midpoint",
                  position_integration="sap_euler"),
}


def _normalize_precision_knob(value: str, *, option_name: str) -> str:
    """sim/solver_sap.py:62-70"""
    p = str(value).strip().lower()
    p = {"f32": "fp32", "f64": "fp64"}.get(p, p)
    if p not in ("fp32", "fp64"):
        raise ValueError(f"{option_name} must be 'fp32'/'f32' or 'fp64'/'f64', got {value!r}.")
    return p


def _normalize_contact_preset_variant(value: str | None) -> str:
    """sim/solver_sap.py:109-120"""
    if value is None:
        return "approx32"
    v = str(value).strip().lower().replace("-", "_")
    v = {"approx_32": "approx32", "approx_64": "approx64"}.get(v, v)
    if v not in _CONTACT_PRESET_KWARGS:
        raise ValueError(f"contact_preset_variant must be one of {', '.join(SAP_CONTACT_PRESET_VARIANTS)}, "
                         f"got {value!r}.")
    return v


def _ptr(t: torch.Tensor | None) -> int:
    return 0 if t is None else t.data_ptr()


def _f64(t: torch.Tensor) -> torch.Tensor:
    return t if t.dtype == F64 and t.is_contiguous() else t.to(F64).contiguous()


class _ModelView:
    """Per-world sizes, host maps and the sapb_model_desc of a SapModel."""

    def __init__(self, model: SapModel):
        if not isinstance(model, SapModel):
            raise TypeError("SolverSAP requires SapModel; convert frontend data before constructing the solver.")
        W = max(int(model.world_count), 1)
        J, B, D, Q = int(model.joint_count), int(model.body_count), int(model.joint_dof_count), int(
            model.joint_coord_count)
        if J <= 0 or D <= 0:
            raise ValueError("SolverSAP requires a model with articulated joint DOFs.")
        self.uneven = getattr(model, "world_joint_start", None) is not None
        self.model = model
        if self.uneven:
            # worlds of different sizes: per-world blocks from the offsets;
            # the *_per_world sizes are the largest world's
            off = {k: getattr(model, "world_" + k + "_start").cpu().numpy().astype(np.int64)
                   for k in ("joint", "body", "dof", "articulation")}
            for k, tot in (("joint", J), ("body", B), ("dof", D), ("articulation", int(model.articulation_count))):
                o = off[k]
                if len(o) != W + 1 or o[0] != 0 or o[-1] != tot or np.any(np.diff(o) < 0):
                    raise ValueError(f"world_{k}_start must be {W + 1} nondecreasing offsets from 0 to {tot}")
            self.world_offsets = off
            self.dof_counts = np.diff(off["dof"]).astype(np.int32)
            self.W, self.Jw, self.Bw = W, int(np.diff(off["joint"]).max()), int(np.diff(off["body"]).max())
            self.n, self.Aw = int(self.dof_counts.max()), int(np.diff(off["articulation"]).max())
            self.Qw = int(Q)  # coordinates follow joint_q_start
        else:
            if J % W or B % W or D % W or Q % W or int(model.articulation_count) % W:
                raise ValueError("SolverSAP requires contiguous equal-sized per-world joint/body/dof/coord blocks "
                                 f"(worlds={W}, joints={J}, bodies={B}, dofs={D}, coords={Q}) or the world "
                                 "offsets of an uneven batch.")
            self.W, self.Jw, self.Bw, self.n, self.Qw = W, J // W, B // W, D // W, Q // W
            self.Aw = int(model.articulation_count) // W
            self.dof_counts = None
        jt = model.joint_type.cpu().numpy()
        parent_joint = model.joint_ancestor.cpu().numpy()
        if np.any(parent_joint >= np.arange(J)):
            raise ValueError("joints must be ordered parents before children")
        self.device = model.joint_type.device
        # the tree-blocked layout: the trees are the world's articulations
        # (a free body, an arm), each in a block of tree_block DOFs (6, 7 or
        # 12: the smallest holding the largest tree); worlds of equal blocks
        # with <= 64 bodies may use it, and by default those beyond the dense
        # solve's 60 DOFs do
        self.tree_dof_start, self.tree_block = None, 0
        if not self.uneven and self.Bw <= 64 and 1 <= self.Aw <= 64:
            art = model.articulation_start.cpu().numpy()[:self.Aw + 1]
            ds0 = model.joint_qd_start.cpu().numpy()
            tds = np.array([int(ds0[int(a)]) for a in art], np.int64)
            if tds[0] == 0 and tds[-1] == self.n and np.all(np.diff(tds) >= 0):
                self.tree_block = tree_block_for(int(np.diff(tds).max()))
                self.tree_dof_start = torch.as_tensor(tds.astype(np.int32), device=model.joint_type.device)
        self.tree_eligible = self.tree_block > 0
        self.tree_blocked = self.tree_eligible and self.n > 60
        d = _abi.ModelDesc()
        d.num_worlds, d.joints_per_world, d.bodies_per_world = W, self.Jw, self.Bw
        d.dofs_per_world, d.coords_per_world, d.articulations_per_world = self.n, self.Qw, self.Aw
        d.num_shapes = int(model.shape_body.numel()) if model.shape_body is not None else 0
        self._keep = {}

        def k(name, t, dtype):
            t = t.to(dtype).contiguous()
            self._keep[name] = t
            return t.data_ptr()

        def k_(name, t):
            return k(name, t, I32)

        for name in ("joint_type", "joint_parent", "joint_child", "joint_ancestor", "joint_q_start",
                     "joint_qd_start", "articulation_start"):
            setattr(d, name, k(name, getattr(model, name), I32))
        d.joint_dof_dim = k("joint_dof_dim", model.joint_dof_dim.reshape(-1), I32)
        for name in ("joint_axis", "joint_X_p", "joint_X_c", "joint_armature", "body_mass", "body_inertia",
                     "body_com", "gravity"):
            setattr(d, name, k(name, getattr(model, name).reshape(-1), F64))
        if d.num_shapes:
            d.shape_body = k("shape_body", model.shape_body, I32)
            for name in ("shape_material_mu", "shape_material_ke", "shape_material_tau"):
                t = getattr(model, name)
                setattr(d, name, k(name, t, F64) if t is not None else 0)
        if self.uneven:
            for kind in ("joint", "body", "dof", "articulation"):
                setattr(d, f"world_{kind}_start", k_(f"world_{kind}_start", getattr(model, f"world_{kind}_start")))
            d.body_world = k_("body_world", model.body_world)
            d.total_joints, d.total_bodies, d.total_dofs = J, B, D
            d.total_articulations = int(model.articulation_count)
            self.dof_count_t = torch.as_tensor(self.dof_counts, dtype=I32, device=self.device)
        else:
            self.dof_count_t = None
        self.desc = d
        self._build_dof_maps(jt)

    def _build_dof_maps(self, jt):
        """sim/contact_solve.py:3681-3758: DOF -> coordinate, drive target and
        limit support; body -> articulation DOF range (world-local)."""
        m = self.model
        D = int(m.joint_dof_count)
        qs = m.joint_q_start.cpu().numpy()
        ds = m.joint_qd_start.cpu().numpy()
        dim = m.joint_dof_dim.cpu().numpy().reshape(-1, 2)
        coord = np.full(D, -1, np.int32)
        target = np.arange(D, dtype=np.int32)
        limit_ok = np.zeros(D, np.int32)
        for j, t in enumerate(jt):
            d0 = int(ds[j])
            if t in (SAP_JOINT_FREE, SAP_JOINT_DISTANCE):
                for a in range(3):
                    target[d0 + a] = d0 + a + 3
                    target[d0 + a + 3] = d0 + a
            if t not in (SAP_JOINT_PRISMATIC, SAP_JOINT_REVOLUTE, SAP_JOINT_D6):
                continue
            cnt = int(dim[j].sum())
            for a in range(cnt):
                coord[d0 + a] = int(qs[j]) + a
                if cnt == 1:
                    limit_ok[d0 + a] = 1
        child = m.joint_child.cpu().numpy()
        art = m.articulation_start.cpu().numpy()
        B = int(m.body_count)
        bstart = np.full(B, -1, np.int32)
        bcount = np.zeros(B, np.int32)
        for a in range(len(art) - 1):
            js = range(int(art[a]), int(art[a + 1]))
            counts = [int(dim[j].sum()) for j in js]
            starts = [int(ds[j]) for j, c in zip(js, counts) if c > 0]
            tot = sum(counts)
            if not starts or tot <= 0:
                continue
            s0 = min(starts)
            for j in js:
                b = int(child[j])
                if 0 <= b < B:
                    if self.uneven:
                        env = int(np.searchsorted(self.world_offsets["body"], b, side="right") - 1)
                        bstart[b] = s0 - int(self.world_offsets["dof"][env])
                    else:
                        env = b // self.Bw
                        bstart[b] = s0 - env * self.n
                    bcount[b] = tot
        dev = self.device
        self.dof_coord_index = torch.as_tensor(coord, device=dev)
        self.dof_target_index = torch.as_tensor(target, device=dev)
        self.limit_supported = torch.as_tensor(limit_ok, device=dev)
        self.body_dof_start = torch.as_tensor(bstart, device=dev)
        self.body_dof_count = torch.as_tensor(bcount, device=dev)
        mode = m.joint_target_mode.cpu().numpy()
        ke = m.joint_target_ke.cpu().numpy()
        kd = m.joint_target_kd.cpu().numpy()
        self.has_pd = bool(np.any((mode != SAP_JOINT_TARGET_NONE) & ((ke > 0) | (kd > 0))))
        lo = m.joint_limit_lower.cpu().numpy()
        hi = m.joint_limit_upper.cpu().numpy()
        lke = m.joint_limit_ke.cpu().numpy()
        self.has_limits = bool(np.any((limit_ok != 0) & (lke > 0) & (np.isfinite(lo) | np.isfinite(hi))))


def _checked_order(order: torch.Tensor | None, W: int) -> torch.Tensor | None:
    if order is not None and (order.dtype != I32 or not order.is_contiguous() or order.numel() != W):
        raise TypeError(f"world_order must be a contiguous int32 tensor of {W} world indices")
    return order


def tree_block_for(tree_dofs: int) -> int:
    """The block size of the tree-blocked solve for trees of up to tree_dofs
    DOFs: the smallest of 6, 7 and 12 that holds them, 0 if none does (the
    rule of sapb_blocked_tree_block)."""
    for nb in (6, 7, 12):
        if 0 <= tree_dofs <= nb:
            return nb
    return 0


def _pick_tree_blocked(view: _ModelView, tree_blocked: bool | None) -> bool:
    if tree_blocked is None:
        return view.tree_blocked
    if tree_blocked and not view.tree_eligible:
        raise ValueError("the tree-blocked layout needs equal worlds of <= 64 bodies whose articulations hold at "
                         "most 12 DOFs each")
    return bool(tree_blocked)


@dataclass(frozen=True)
class SapFreeMotionResult:
    """sim/free_motion.py:63-68"""

    v_star: torch.Tensor
    vdot: torch.Tensor
    dynamics_matrix: torch.Tensor | None


@dataclass(frozen=True)
class SapContactJacobianResult:
    """Views into buffers owned by SapContactJacobian (sim/contact_jacobian.py:51-84)."""

    contact_count: int
    truncated_contact_count: int
    contact_env_count: torch.Tensor
    contact_env_phi0: torch.Tensor
    contact_env_jacobian: torch.Tensor
    contact_env_w_eff: torch.Tensor
    contact_env_mu: torch.Tensor
    contact_env_stiffness: torch.Tensor
    contact_env_R_WC: torch.Tensor
    contact_env_point: torch.Tensor
    contact_env_witness0: torch.Tensor | None
    contact_env_witness1: torch.Tensor | None
    contact_env_body0: torch.Tensor
    contact_env_body1: torch.Tensor
    body_jacobian_local: torch.Tensor | None
    dynamics_matrix_env: torch.Tensor
    contact_env_tau_d: torch.Tensor | None = None
    # LDL^T of dynamics_matrix_env from the free-motion solve (no counterpart
    # in the reference's result), or None when not requested
    dynamics_factor_env: torch.Tensor | None = None
    # tree-blocked layout (no counterpart in the reference): the diagonal
    # blocks of A, one per articulation [W, T, NB, NB] (the identity beyond a
    # tree's own DOFs), and the tree of each contact side [W, C, 2];
    # contact_env_jacobian is then [W, C, 3, 2 NB] and dynamics_matrix_env is
    # None
    tree_mass_env: torch.Tensor | None = None
    contact_env_tree: torch.Tensor | None = None


@dataclass(frozen=True)
class SapContactSolveResult:
    """Views into buffers owned by SapContactSolve (sim/contact_solve.py:188-232)."""

    v_env: torch.Tensor
    v_flat: torch.Tensor
    cost: torch.Tensor
    contact_gamma: torch.Tensor
    contact_mode: torch.Tensor
    newton_iterations_env: torch.Tensor
    line_search_iterations_env: torch.Tensor
    converged_env: torch.Tensor
    line_search_status_env: torch.Tensor
    grad_norm_env: torch.Tensor
    iterations: int
    line_search_iterations: int
    converged: bool


class SapContactJacobian:
    """Free motion + contact Jacobian of every world in two launches
    (SapContactJacobian, sim/contact_jacobian.py:1242-1985, which owns the
    SapFreeMotion of sim/free_motion.py)."""

    def __init__(self, model: SapModel, *, max_rigid_contact: int = 128, fallback_mu: float | None = None,
                 fallback_stiffness: float = 1.0e10, fallback_tau_d: float = 0.1,
                 contact_weight_mode: str = "diag_delassus", contact_point_mode: str = "contact_midpoint",
                 capture_local_snapshots: bool = False, use_f64_boundary_pose: bool = True,
                 free_motion_solve_precision: str = "fp64", sap_contact_weight_precision: str = "fp64",
                 tree_blocked: bool | None = None, _view: _ModelView | None = None):
        """tree_blocked: None picks the tree-blocked layout for worlds of free
        bodies with more than 60 DOFs; True asks for it (worlds of free
        bodies only), False for the dense one."""
        self.view = _view or _ModelView(model)
        v = self.view
        self.tree_blocked = _pick_tree_blocked(v, tree_blocked)
        self.model = model
        self.max_rigid_contact = max(int(max_rigid_contact), 1)
        wm = str(contact_weight_mode).strip().lower()
        if wm not in ("body_inertia", "diag_delassus"):
            raise ValueError(f"contact_weight_mode must be 'body_inertia' or 'diag_delassus', got {contact_weight_mode!r}")
        pm = str(contact_point_mode).strip().lower()
        if pm not in ("witness_point", "contact_midpoint"):
            raise ValueError(f"contact_point_mode must be 'witness_point' or 'contact_midpoint', got {contact_point_mode!r}")
        self.contact_weight_mode, self.contact_point_mode = wm, pm
        if fallback_mu is None:  # _infer_contact_mu_fallback (sim/sap_helpers.py:40-45)
            mu = model.shape_material_mu.cpu().numpy() if model.shape_material_mu is not None else np.zeros(0)
            pos = mu[mu > 0.0]
            fallback_mu = float(pos.min()) if pos.size else 0.1
        self.opts = _abi.PrepareOptions()
        self.opts.max_contacts = self.max_rigid_contact
        self.opts.contact_weight_mode = (_abi.SAPB_WEIGHT_DIAG_DELASSUS if wm == "diag_delassus"
                                         else _abi.SAPB_WEIGHT_BODY_INERTIA)
        self.opts.contact_point_mode = _abi.SAPB_POINT_MIDPOINT if pm == "contact_midpoint" else _abi.SAPB_POINT_WITNESS
        self.opts.fallback_mu = float(fallback_mu)
        self.opts.fallback_stiffness = float(fallback_stiffness)
        self.opts.fallback_tau_d = float(fallback_tau_d)
        self.opts.tree_blocked = 1 if self.tree_blocked else 0
        self.opts.tree_dofs = v.tree_block if self.tree_blocked else 0
        W, n, C, dev = v.W, v.n, self.max_rigid_contact, v.device
        z = lambda *s, dt=F64: torch.zeros(*s, dtype=dt, device=dev)
        self.v_star = z(W * n)
        self.vdot = z(W * n)
        if self.tree_blocked:
            self.dynamics_matrix_env = None
            NB = v.tree_block
            self.tree_mass_env = z(W, v.Aw, NB, NB)
            self.contact_env_tree = torch.full((W, C, 2), -1, dtype=I32, device=dev)
            self.contact_env_jacobian = z(W, C, 3, 2 * NB)
        else:
            self.dynamics_matrix_env = z(W, n, n)
            self.tree_mass_env = self.contact_env_tree = None
            self.contact_env_jacobian = z(W, C, 3, n)
        self.contact_env_count = z(W, dt=I32)
        self.contact_env_phi0 = z(W, C)
        self.contact_env_w_eff = z(W, C)
        self.contact_env_mu = z(W, C)
        self.contact_env_stiffness = z(W, C)
        self.contact_env_tau_d = z(W, C)
        self.contact_env_body0 = torch.full((W, C), -1, dtype=I32, device=dev)
        self.contact_env_body1 = torch.full((W, C), -1, dtype=I32, device=dev)
        self.contact_env_point = z(W, C, 3)
        self.contact_env_R_WC = z(W, C, 3, 3)
        self.truncated = z(1, dt=I32)
        self.body_q_sap = z(int(model.body_count), 7)
        # uneven batches: the start-of-step velocities in the solve's slots
        self.qd_slots = z(W * n) if v.uneven else None
        self.dynamics_factor_env = None  # allocated by keep_dynamics_factor()
        self.dt_world = z(W)
        ws = int(load().sapb_prepare_workspace_size(ctypes.byref(v.desc), C))
        self.workspace = torch.zeros(max(ws, 16), dtype=torch.uint8, device=dev)
        self._contact_f64 = None
        o = _abi.PrepareOutputs()
        o.v_star, o.vdot, o.dynamics_matrix = _ptr(self.v_star), _ptr(self.vdot), _ptr(self.dynamics_matrix_env)
        o.jacobian, o.contact_count = _ptr(self.contact_env_jacobian), _ptr(self.contact_env_count)
        o.phi0, o.w_eff, o.mu = _ptr(self.contact_env_phi0), _ptr(self.contact_env_w_eff), _ptr(self.contact_env_mu)
        o.stiffness, o.tau_d = _ptr(self.contact_env_stiffness), _ptr(self.contact_env_tau_d)
        o.body0, o.body1 = _ptr(self.contact_env_body0), _ptr(self.contact_env_body1)
        o.point, o.frame = _ptr(self.contact_env_point), _ptr(self.contact_env_R_WC)
        o.truncated_count, o.body_q = _ptr(self.truncated), _ptr(self.body_q_sap)
        o.tree_mass, o.contact_tree = _ptr(self.tree_mass_env), _ptr(self.contact_env_tree)
        o.qd_slots = _ptr(self.qd_slots)
        self.outputs = o

    def keep_dynamics_factor(self) -> None:
        """Also write the free-motion LDL^T of A and the free-motion contact
        velocities J_c v* (for candidate starts and the warm-start network)."""
        if self.tree_blocked:
            raise NotImplementedError("the tree-blocked layout keeps no dense factor of A")
        if self.dynamics_factor_env is None:
            v = self.view
            self.dynamics_factor_env = torch.zeros(v.W, v.n, v.n, dtype=F64, device=v.device)
            self.outputs.dynamics_factor = _ptr(self.dynamics_factor_env)
        self.keep_contact_velocities()

    def keep_contact_velocities(self) -> None:
        """Also write the free-motion contact velocities J_c v* (the
        warm-start network's inputs); in either layout."""
        if getattr(self, "contact_env_vc_star", None) is None:
            v = self.view
            self.contact_env_vc_star = torch.zeros(v.W, self.max_rigid_contact, 3, dtype=F64, device=v.device)
            self.outputs.vc_star = _ptr(self.contact_env_vc_star)

    def keep_contact_source(self) -> None:
        """Also write the flat contact index of each slot (contact_env_source,
        [W][C], -1 past a world's count): the key of the contact history."""
        if getattr(self, "contact_env_source", None) is None:
            v = self.view
            self.contact_env_source = torch.full((v.W, self.max_rigid_contact), -1, dtype=I32, device=v.device)
            self.outputs.contact_source = _ptr(self.contact_env_source)

    def set_history(self, history, v_start: torch.Tensor | None = None, factor_new_contacts_only: bool = False) -> None:
        """Run the contact history (an _abi.ContactHistory over persistent
        buffers, or None) inside the launch, between the contact scatter and
        the free motion; with v_start ((W*n,) FP64) also write the candidate
        start v* + A^-1 J^T gamma_start there; factor_new_contacts_only: the
        kept LDL^T factor only for worlds with a new contact."""
        self._history = history  # the launch reads it by address
        self.outputs.history = ctypes.addressof(history) if history is not None else None
        self.outputs.v_start = _ptr(v_start)
        self.opts.factor_new_contacts_only = 1 if factor_new_contacts_only else 0

    def set_dt(self, dt) -> None:
        """Per-world time step (scalar or [W] tensor), sim/solver_sap.py:975-992."""
        if isinstance(dt, torch.Tensor):
            if dt.numel() != self.view.W:
                raise ValueError(f"per-world dt length {dt.numel()} != num_envs {self.view.W}")
            self.dt_world.copy_(dt.reshape(-1))
        else:
            self.dt_world.fill_(float(dt))

    def _contact_arrays(self, contacts: SapContacts):
        if contacts is None or contacts.rigid_contact_count is None:
            return None
        if contacts.has_f64_rigid_contacts:
            return (contacts.rigid_contact_point0d, contacts.rigid_contact_point1d, contacts.rigid_contact_normald,
                    contacts.rigid_contact_margin0d, contacts.rigid_contact_margin1d)
        N = int(contacts.rigid_contact_shape0.numel())
        if self._contact_f64 is None or self._contact_f64[0].shape[0] != N:
            dev = self.view.device
            self._contact_f64 = [torch.zeros(N, 3, dtype=F64, device=dev), torch.zeros(N, 3, dtype=F64, device=dev),
                                 torch.zeros(N, 3, dtype=F64, device=dev), torch.zeros(N, dtype=F64, device=dev),
                                 torch.zeros(N, dtype=F64, device=dev)]
        srcs = (contacts.rigid_contact_point0, contacts.rigid_contact_point1, contacts.rigid_contact_normal,
                contacts.rigid_contact_margin0, contacts.rigid_contact_margin1)
        for dst, src in zip(self._contact_f64, srcs):
            if src is None:
                dst.zero_()
            else:
                dst.copy_(src.reshape(dst.shape))
        return tuple(self._contact_f64)

    def compute(self, state: SapState, contacts: SapContacts, *, control: SapControl | None = None, dt=None):
        """Free motion and contact rows for `state` and the flat `contacts`."""
        if not isinstance(state, SapState):
            raise TypeError("SapContactJacobian.compute requires SapState.")
        if getattr(state, "joint_qd_order", "sap") != "sap" or (control is not None and
                                                                getattr(control, "joint_f_order", "sap") != "sap"):
            raise NotImplementedError("public-order boundary conversion is not supported; pass SAP-order arrays.")
        if dt is not None:
            self.set_dt(dt)
        self._q = _f64(state.joint_q)
        self._qd = _f64(state.joint_qd)
        jf = _f64(control.joint_f) if control is not None and control.joint_f is not None else None
        bf = _f64(state.body_f.reshape(-1, 6)) if state.body_f is not None else None
        inp = _abi.StepInputs()
        inp.joint_q, inp.joint_qd, inp.joint_f, inp.body_f = _ptr(self._q), _ptr(self._qd), _ptr(jf), _ptr(bf)
        inp.dt = _ptr(self.dt_world)
        arrays = self._contact_arrays(contacts)
        if arrays is not None:
            inp.contact_capacity = int(contacts.rigid_contact_shape0.numel())
            inp.contact_count = _ptr(contacts.rigid_contact_count)
            inp.contact_shape0 = _ptr(contacts.rigid_contact_shape0)
            inp.contact_shape1 = _ptr(contacts.rigid_contact_shape1)
            inp.contact_point0, inp.contact_point1, inp.contact_normal = (_ptr(a) for a in arrays[:3])
            inp.contact_margin0, inp.contact_margin1 = _ptr(arrays[3]), _ptr(arrays[4])
        self._inputs = inp
        status = load().sapb_free_motion_contacts(ctypes.byref(self.view.desc), ctypes.byref(inp),
                                                  ctypes.byref(self.opts), ctypes.byref(self.outputs),
                                                  self.workspace.data_ptr(), self.workspace.numel(),
                                                  ctypes.c_void_p(torch.cuda.current_stream(self.view.device).cuda_stream))
        check(status, "sapb_free_motion_contacts")
        return self.result()

    def result(self) -> SapContactJacobianResult:
        return SapContactJacobianResult(
            contact_count=-1, truncated_contact_count=-1,  # device counters; read without a host sync
            contact_env_count=self.contact_env_count, contact_env_phi0=self.contact_env_phi0,
            contact_env_jacobian=self.contact_env_jacobian, contact_env_w_eff=self.contact_env_w_eff,
            contact_env_mu=self.contact_env_mu, contact_env_stiffness=self.contact_env_stiffness,
            contact_env_R_WC=self.contact_env_R_WC, contact_env_point=self.contact_env_point,
            contact_env_witness0=None, contact_env_witness1=None, contact_env_body0=self.contact_env_body0,
            contact_env_body1=self.contact_env_body1, body_jacobian_local=None,
            dynamics_matrix_env=self.dynamics_matrix_env, contact_env_tau_d=self.contact_env_tau_d,
            dynamics_factor_env=self.dynamics_factor_env, tree_mass_env=self.tree_mass_env,
            contact_env_tree=self.contact_env_tree)

    @property
    def free_motion_result(self) -> SapFreeMotionResult:
        return SapFreeMotionResult(v_star=self.v_star, vdot=self.vdot, dynamics_matrix=None)


class SapFreeMotion:
    """SapFreeMotion.compute (sim/free_motion.py:2180-2208): v* and vdot in
    SAP order.  Runs the same fused launch as SapContactJacobian with no
    contacts."""

    def __init__(self, model: SapModel, **kwargs):
        self._cj = SapContactJacobian(model, max_rigid_contact=1, **kwargs)

    def compute(self, state: SapState, control: SapControl | None, dt, *, assemble_dynamics_matrix: bool = False):
        if control is None or not isinstance(control, SapControl):
            raise TypeError("SapFreeMotion.compute requires SapControl; convert before entering SAP components.")
        self._cj.compute(state, SapContacts(), control=control, dt=dt)
        r = self._cj.free_motion_result
        if assemble_dynamics_matrix:
            if self._cj.tree_blocked:
                raise NotImplementedError("assemble_dynamics_matrix is not available in the tree-blocked layout")
            W, n = self._cj.view.W, self._cj.view.n
            A = torch.zeros(W * n, W * n, dtype=F64, device=self._cj.view.device)
            for e in range(W):
                A[e * n:(e + 1) * n, e * n:(e + 1) * n] = self._cj.dynamics_matrix_env[e]
            return SapFreeMotionResult(r.v_star, r.vdot, A)
        return r


class SapContactSolve:
    """Stage-2 Newton solve (sim/contact_solve.py:3291-6341) in one launch."""

    def __init__(self, model: SapModel, *, max_rigid_contact: int = 128, contact_beta: float = 1.0,
                 contact_sigma: float = 1.0e-3, contact_tau_d: float = 0.1, block_size: int | None = None,
                 diag_shift: float = 0.0, contact_assembly_tile_size: int = 256, solve_precision: str = "fp64",
                 linear_solve_precision: str = "fp64", hessian_precision: str | None = None,
                 tree_blocked: bool | None = None, _view: _ModelView | None = None):
        self.view = _view or _ModelView(model)
        v = self.view
        self.autotuner = None  # autotune.SolveAutotuner: picks the dense solve's resident CTAs per SM
        self._device_props = None
        self.tree_blocked = _pick_tree_blocked(v, tree_blocked)
        if v.n > 60 and not self.tree_blocked:
            raise NotImplementedError(f"the dense on-chip solve supports up to 60 DOFs per world, got {v.n} "
                                      "(worlds of free bodies use the tree-blocked solve)")
        self.model = model
        self.max_rigid_contact = max(int(max_rigid_contact), 1)
        self.contact_beta, self.contact_sigma = float(contact_beta), float(contact_sigma)
        self.contact_tau_d, self.diag_shift = float(contact_tau_d), float(diag_shift)
        self.solve_precision = _normalize_precision_knob(solve_precision, option_name="solve_precision")
        if self.solve_precision != "fp64":
            raise NotImplementedError("the contact objective is always evaluated in fp64")
        self.linear_solve_precision = _normalize_precision_knob(linear_solve_precision,
                                                                option_name="linear_solve_precision")
        self.hessian_precision = _normalize_precision_knob(hessian_precision or self.linear_solve_precision,
                                                           option_name="hessian_precision")
        W, n, C, dev = v.W, v.n, self.max_rigid_contact, v.device
        z = lambda *s, dt=F64: torch.zeros(*s, dtype=dt, device=dev)
        self.v_flat = z(W * n)
        self.v_env = self.v_flat.view(W, n)
        self.contact_gamma = z(W, C, 3)
        self.contact_mode = z(W, C, dt=I32)
        self.cost = z(W)
        self.newton_iterations_env = z(W, dt=I32)
        self.ls_iterations_total = z(W, dt=I32)
        self.converged_env = z(W, dt=I32)
        self.ls_status = z(W, dt=I32)
        self.grad_norm = z(W)
        self.warm_start_accepted_env = z(W, dt=I32)
        self.dt_world = z(W)
        ws = int(load().sapb_blocked_solve_workspace_size(W, v.Aw, C) if self.tree_blocked
                 else load().sapb_contact_solve_workspace_size(W, n, C))
        self.workspace = torch.zeros(max(ws, 16), dtype=torch.uint8, device=dev)
        self.zero_f32 = z(W * n, dt=F32)
        out = _abi.SolveOutputs()
        out.v, out.contact_gamma, out.contact_mode = _ptr(self.v_flat), _ptr(self.contact_gamma), _ptr(self.contact_mode)
        out.cost, out.newton_iterations = _ptr(self.cost), _ptr(self.newton_iterations_env)
        out.line_search_iterations, out.converged = _ptr(self.ls_iterations_total), _ptr(self.converged_env)
        out.status, out.grad_norm = _ptr(self.ls_status), _ptr(self.grad_norm)
        out.warm_start_accepted = _ptr(self.warm_start_accepted_env)
        self.outputs = out
        self.dof = None
        if v.has_pd or v.has_limits:
            m = model
            self.dof = _abi.DofTerms()
            self.dof.has_pd, self.dof.has_limits = int(v.has_pd), int(v.has_limits)
            self.dof.joint_coord_count = int(m.joint_coord_count)
            self._dof_keep = dict(
                dof_coord_index=v.dof_coord_index, dof_target_index=v.dof_target_index,
                limit_supported=v.limit_supported, joint_target_mode=m.joint_target_mode.to(I32).contiguous(),
                joint_target_ke=m.joint_target_ke.to(F32).contiguous(),
                joint_target_kd=m.joint_target_kd.to(F32).contiguous(),
                joint_effort_limit=m.joint_effort_limit.to(F32).contiguous(),
                joint_limit_lower=_f64(m.joint_limit_lower), joint_limit_upper=_f64(m.joint_limit_upper),
                joint_limit_ke=_f64(m.joint_limit_ke), joint_limit_kd=_f64(m.joint_limit_kd))
            for k, t in self._dof_keep.items():
                setattr(self.dof, k, t.data_ptr())
            if v.uneven:
                # per-DOF arrays in the model's global order, each world's
                # from its DOF offset (the solve runs in slots)
                self.dof.world_dof_start = v._keep["world_dof_start"].data_ptr()

    def options(self, line_search_variant, **kw) -> _abi.SolveOptions:
        from ._solve import make_options

        return make_options(line_search_variant, contact_beta=self.contact_beta, contact_sigma=self.contact_sigma,
                            contact_tau_d=self.contact_tau_d, diag_shift=self.diag_shift,
                            linear_solve_precision=self.linear_solve_precision,
                            hessian_precision=self.hessian_precision, **kw)

    def solve_options(self, line_search_variant: str = "monotone_decay", *, max_iterations: int = 100,
                      optimality_abs_tol: float = 1.0e-14, optimality_rel_tol: float = 1.0e-6,
                      cost_abs_tol: float | None = None, cost_rel_tol: float | None = None,
                      line_search_max_iterations: int = 40, armijo_c: float = 1.0e-4, rho: float = 0.8,
                      line_search_relative_slop: float | None = None):
        """(variant, sapb_solve_options) of solve() with the reference's
        variant-dependent defaults (sim/contact_solve.py:6163-6182)."""
        variant = normalize_sap_line_search_mode(line_search_variant)
        if variant == "armijo_decay" and not (0.0 < float(rho) < 1.0):
            raise ValueError(f"rho must lie in (0, 1), got {rho!r}.")
        if variant == "exact_root" and int(line_search_max_iterations) == 40:
            line_search_max_iterations = 100
        if cost_abs_tol is None:
            cost_abs_tol = 0.0 if variant == "monotone_decay" else 1.0e-30
        if cost_rel_tol is None:
            cost_rel_tol = 5.0e-3 if variant == "monotone_decay" else 1.0e-15
        if line_search_relative_slop is None:
            line_search_relative_slop = 1000.0 * np.finfo(np.float64).eps
        opts = self.options(variant, max_iterations=int(max_iterations), optimality_abs_tol=float(optimality_abs_tol),
                            optimality_rel_tol=float(optimality_rel_tol), cost_abs_tol=float(cost_abs_tol),
                            cost_rel_tol=float(cost_rel_tol),
                            line_search_max_iterations=int(line_search_max_iterations), armijo_c=float(armijo_c),
                            rho=float(rho), line_search_relative_slop=float(line_search_relative_slop))
        return variant, opts

    def _launch_shape(self, P, opts, variant: str, stream,
                      guess: torch.Tensor | None = None) -> tuple[int, int, int]:
        """(resident CTAs per SM, LDL^T block width, threads per CTA) for this
        problem: (0, 0, 0) -- the occupancy bound, the default width and
        kernel -- without an autotuner; with one, its choice for the
        problem's key among every CTA count up to the bound and every width
        the kernel is built with, and every CTA count of the 256-thread
        runtime-size kernel, timed here on this very problem the first time
        the key is seen
        (never while a graph is being captured: then the defaults).  The solve
        writes its start back into the warm-start guess `guess` (and the
        guess may be the output velocity itself), so the guess is saved
        before the timed solves and restored before each of them and after:
        every timed solve, and the real one, starts from the same guess."""
        from .autotune import tuning_key

        if self.autotuner is None:
            return 0, 0, 0
        v = self.view
        fp32 = opts.hessian_precision == _abi.SAPB_FP32 or opts.linear_solve_precision == _abi.SAPB_FP32
        if self._device_props is None:
            self._device_props = torch.cuda.get_device_properties(v.device)
        props = self._device_props
        key = tuning_key(v.n, P.max_contacts, "fp32" if fp32 else "fp64", variant, props.name,
                         props.multi_processor_count)
        known = self.autotuner.lookup(key)
        if known is not None:
            known = known if isinstance(known, tuple) else (known,)
            return tuple(known) + (0,) * (3 - len(known))
        if torch.cuda.is_current_stream_capturing():
            return 0, 0, 0
        lib = load()
        occ = int(lib.sapb_contact_solve_occupancy(v.n, int(P.max_contacts),
                                                   _abi.SAPB_FP32 if fp32 else _abi.SAPB_FP64,
                                                   int(opts.line_search_variant)))
        if occ < 1:
            check(occ, "sapb_contact_solve_occupancy")
        cur = torch.cuda.current_stream(v.device)
        saved = guess.clone() if guess is not None else None
        widths = (ctypes.c_int32 * 8)()
        nw = max(min(int(lib.sapb_contact_solve_ldlt_blocks(v.n, widths, 8)), 8), 1)

        def time_ms(shape) -> float:
            o = _abi.SolveOptions.from_buffer_copy(opts)
            o.ctas_per_sm, o.ldlt_block, o.threads_per_cta = shape
            if saved is not None:
                guess.copy_(saved)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(cur)
            check(lib.sapb_contact_solve(ctypes.byref(P), ctypes.byref(o), ctypes.byref(self.outputs),
                                         self.workspace.data_ptr(), self.workspace.numel(), stream),
                  "sapb_contact_solve")
            e1.record(cur)
            e1.synchronize()
            return e0.elapsed_time(e1)

        cands = [(k, int(widths[b]), 128) for b in range(nw) for k in range(1, occ + 1)]
        # the runtime-size kernel with eight warps per world (its default
        # width), where its shared memory fits
        occ_wide = int(lib.sapb_contact_solve_occupancy_threads(v.n, int(P.max_contacts),
                                                                _abi.SAPB_FP32 if fp32 else _abi.SAPB_FP64,
                                                                int(opts.line_search_variant), 256))
        if occ_wide >= 1:
            gw = (ctypes.c_int32 * 8)()
            lib.sapb_contact_solve_ldlt_blocks(1, gw, 8)  # the runtime-size kernel's widths
            cands += [(k, int(gw[0]), 256) for k in range(1, occ_wide + 1)]
        chosen = self.autotuner.tune(key, cands, time_ms, default=(occ, int(widths[0]), 128))
        if saved is not None:
            guess.copy_(saved)
        return chosen

    def solve(self, contact_result: SapContactJacobianResult, state: SapState, control: SapControl | None, dt,
              v_star: torch.Tensor, *, v0: torch.Tensor | None = None, v_guess: torch.Tensor | None = None,
              v_guess_active: torch.Tensor | None = None, max_iterations: int = 100,
              optimality_abs_tol: float = 1.0e-14, optimality_rel_tol: float = 1.0e-6,
              cost_abs_tol: float | None = None, cost_rel_tol: float | None = None,
              line_search_max_iterations: int = 40, armijo_c: float = 1.0e-4, rho: float = 0.8,
              line_search_relative_slop: float | None = None, line_search_variant: str = "monotone_decay",
              collect_iteration_stats: bool = True, check_line_search_errors: bool = True,
              graph_conditional: bool = True, static_loop: bool = False,
              gamma0: torch.Tensor | None = None, world_order: torch.Tensor | None = None,
              v_candidates: torch.Tensor | None = None,
              gamma0_base: torch.Tensor | None = None, skip_plain_start: bool = False) -> SapContactSolveResult:
        """sim/contact_solve.py:6129-6285.  Candidate starts (no counterpart
        in the reference), tried against the plain start on the cost:
        v_candidates (W*n,) or (K, W*n) FP64 start velocities, then gamma0
        (W, C, 3) or (K, W, C, 3) FP64 starting impulses, each mapped to
        gamma0_base (or v*) + A^-1 J^T gamma; skip_plain_start: start from the
        best candidate without trying the plain start (kept as the fallback
        when no candidate's cost is finite).  world_order (W,) int32: the
        order in which the persistent kernel takes the worlds (a permutation;
        results do not depend on it)."""
        if not bool(graph_conditional):
            raise ValueError("SapContactSolve only supports graph_conditional=True; "
                             "the Python Newton-loop fallback has been removed.")
        variant, opts = self.solve_options(
            line_search_variant, max_iterations=max_iterations, optimality_abs_tol=optimality_abs_tol,
            optimality_rel_tol=optimality_rel_tol, cost_abs_tol=cost_abs_tol, cost_rel_tol=cost_rel_tol,
            line_search_max_iterations=line_search_max_iterations, armijo_c=armijo_c, rho=rho,
            line_search_relative_slop=line_search_relative_slop)
        if isinstance(dt, torch.Tensor):
            self.dt_world.copy_(dt.reshape(-1))
        else:
            self.dt_world.fill_(float(dt))
        if v0 is None:
            v0 = v_guess if v_guess is not None else v_star
        v = self.view
        W, n, C = v.W, v.n, self.max_rigid_contact
        if self.tree_blocked:
            return self._solve_blocked(contact_result, opts, v_star, v0, v_guess, v_guess_active, world_order,
                                       gamma0, state=state, control=control)
        P = _abi.ContactProblem()
        P.num_envs, P.dof_per_env, P.max_contacts = W, n, int(contact_result.contact_env_jacobian.shape[1])
        P.num_bodies = int(v.body_dof_start.numel())
        r = contact_result
        P.contact_count, P.dynamics_matrix = _ptr(r.contact_env_count), _ptr(r.dynamics_matrix_env)
        P.world_order = _ptr(_checked_order(world_order, W))
        P.dof_count = _ptr(v.dof_count_t)  # uneven batches: each world's own DOF count
        P.jacobian, P.phi0, P.w_eff = _ptr(r.contact_env_jacobian), _ptr(r.contact_env_phi0), _ptr(r.contact_env_w_eff)
        P.mu, P.stiffness, P.tau_d = _ptr(r.contact_env_mu), _ptr(r.contact_env_stiffness), _ptr(r.contact_env_tau_d)
        P.body0, P.body1 = _ptr(r.contact_env_body0), _ptr(r.contact_env_body1)
        P.body_dof_start, P.body_dof_count = _ptr(v.body_dof_start), _ptr(v.body_dof_count)
        self._vs, self._v0 = _f64(v_star), _f64(v0)
        P.v_star, P.v0, P.dt = _ptr(self._vs), _ptr(self._v0), _ptr(self.dt_world)
        if v_guess is not None:
            if v_guess.dtype != F64 or not v_guess.is_contiguous():
                raise TypeError("v_guess must be a contiguous float64 tensor (it is written back)")
            P.v_guess = _ptr(v_guess)
            P.v_guess_active = _ptr(v_guess_active)
        if gamma0 is not None:
            per_set = W * P.max_contacts * 3
            if gamma0.dtype != F64 or not gamma0.is_contiguous() or gamma0.numel() < per_set:
                raise TypeError("gamma0 must be a contiguous float64 (W, C, 3) or (K, W, C, 3) tensor")
            P.gamma0 = _ptr(gamma0)
            P.gamma0_count = int(gamma0.numel() // per_set)
            if getattr(contact_result, "dynamics_factor_env", None) is not None:
                P.dynamics_factor = _ptr(contact_result.dynamics_factor_env)
            if gamma0_base is not None:
                if gamma0_base.dtype != F64 or not gamma0_base.is_contiguous() or gamma0_base.numel() != W * n:
                    raise TypeError("gamma0_base must be a contiguous float64 (W*n,) tensor")
                P.gamma0_base = _ptr(gamma0_base)
        if v_candidates is not None:
            if v_candidates.dtype != F64 or not v_candidates.is_contiguous() or v_candidates.numel() % (W * n) != 0 \
                    or v_candidates.numel() == 0:
                raise TypeError("v_candidates must be a contiguous float64 (W*n,) or (K, W*n) tensor")
            P.v_candidates = _ptr(v_candidates)
            P.v_candidate_count = int(v_candidates.numel() // (W * n))
        if self.dof is not None:
            self._set_dof_inputs(state, control)
            P.dof = ctypes.pointer(self.dof)
        stream = ctypes.c_void_p(torch.cuda.current_stream(v.device).cuda_stream)
        opts.skip_plain_start = 1 if skip_plain_start else 0
        opts.ctas_per_sm, opts.ldlt_block, opts.threads_per_cta = self._launch_shape(P, opts, variant, stream,
                                                                                      v_guess)
        status = load().sapb_contact_solve(ctypes.byref(P), ctypes.byref(opts), ctypes.byref(self.outputs),
                                           self.workspace.data_ptr(), self.workspace.numel(), stream)
        check(status, "sapb_contact_solve")
        return self.result()

    def _set_dof_inputs(self, state, control) -> None:
        """This step's coordinates and drive targets into the drive / limit
        terms (sapb_dof_terms reads them by address)."""
        self._jq = _f64(state.joint_q)
        self.dof.joint_q = _ptr(self._jq)
        for name, t in (("joint_target_pos", getattr(control, "joint_target_pos", None)),
                        ("joint_target_vel", getattr(control, "joint_target_vel", None)),
                        ("joint_act", getattr(control, "joint_act", None))):
            tt = t.to(F32).contiguous() if t is not None else None
            self._dof_keep["_" + name] = tt
            setattr(self.dof, name, _ptr(tt))

    def _solve_blocked(self, r: SapContactJacobianResult, opts, v_star, v0, v_guess, v_guess_active,
                       world_order=None, gamma0=None, state=None, control=None):
        """The tree-blocked solve (sapb_blocked_contact_solve) on the
        tree-blocked result of SapContactJacobian; gamma0 (W, C, 3): one set
        of candidate starting impulses."""
        if r.tree_mass_env is None or r.contact_env_tree is None:
            raise ValueError("the tree-blocked solve needs a tree-blocked SapContactJacobianResult")
        v = self.view
        P = _abi.BlockedProblem()
        P.num_envs, P.trees_per_env, P.tree_dofs = v.W, v.Aw, v.tree_block
        P.tree_dof_start, P.dofs_per_world = _ptr(v.tree_dof_start), v.n
        if self.dof is not None:
            self._set_dof_inputs(state, control)
            P.dof = ctypes.pointer(self.dof)
        P.max_contacts = int(r.contact_env_jacobian.shape[1])
        P.contact_count, P.tree_mass = _ptr(r.contact_env_count), _ptr(r.tree_mass_env)
        P.world_order = _ptr(_checked_order(world_order, v.W))
        P.jacobian, P.contact_tree = _ptr(r.contact_env_jacobian), _ptr(r.contact_env_tree)
        P.phi0, P.w_eff, P.mu = _ptr(r.contact_env_phi0), _ptr(r.contact_env_w_eff), _ptr(r.contact_env_mu)
        P.stiffness, P.tau_d = _ptr(r.contact_env_stiffness), _ptr(r.contact_env_tau_d)
        self._vs, self._v0 = _f64(v_star), _f64(v0)
        P.v_star, P.v0, P.dt = _ptr(self._vs), _ptr(self._v0), _ptr(self.dt_world)
        if v_guess is not None:
            if v_guess.dtype != F64 or not v_guess.is_contiguous():
                raise TypeError("v_guess must be a contiguous float64 tensor (it is written back)")
            P.v_guess = _ptr(v_guess)
            P.v_guess_active = _ptr(v_guess_active)
        if gamma0 is not None:
            per_set = v.W * int(P.max_contacts) * 3
            if gamma0.dtype != F64 or not gamma0.is_contiguous() or gamma0.numel() != per_set:
                raise TypeError("the tree-blocked solve takes one contiguous float64 (W, C, 3) impulse set")
            P.gamma0, P.gamma0_count = _ptr(gamma0), 1
        status = load().sapb_blocked_contact_solve(ctypes.byref(P), ctypes.byref(opts), ctypes.byref(self.outputs),
                                                   self.workspace.data_ptr(), self.workspace.numel(),
                                                   ctypes.c_void_p(torch.cuda.current_stream(v.device).cuda_stream))
        check(status, "sapb_blocked_contact_solve")
        return self.result()

    def result(self) -> SapContactSolveResult:
        return SapContactSolveResult(
            v_env=self.v_env, v_flat=self.v_flat, cost=self.cost, contact_gamma=self.contact_gamma,
            contact_mode=self.contact_mode, newton_iterations_env=self.newton_iterations_env,
            line_search_iterations_env=self.ls_iterations_total, converged_env=self.converged_env,
            line_search_status_env=self.ls_status, grad_norm_env=self.grad_norm,
            iterations=-1, line_search_iterations=-1, converged=True)


class HostStepGraph:
    """A captured pair of host-fed steps (SolverSAP.capture_host_steps):
    replay() advances the rollout by two steps, copies included."""

    def __init__(self, graph: "torch.cuda.CUDAGraph", device_contacts: tuple, copy_stream: "torch.cuda.Stream"):
        self.graph = graph
        self.device_contacts = device_contacts  # the two device contact buffers the graph reads
        self.copy_stream = copy_stream

    def replay(self) -> None:
        self.graph.replay()


class SolverSAP:
    """SAP timestepper (sim/solver_sap.py:736-1512): free motion and contact
    Jacobian, the stage-2 solve and position integration, three native
    launches per step (plus small memsets)."""

    def __init__(self, model: SapModel, *, max_rigid_contact: int = 128, fallback_mu: float | None = None,
                 fallback_stiffness: float = 1.0e10, contact_beta: float = 1.0, contact_sigma: float = 1.0e-3,
                 contact_tau_d: float | None = None, block_size: int | None = None, diag_shift: float = 0.0,
                 max_iterations: int = 100, optimality_abs_tol: float = 1.0e-14, optimality_rel_tol: float = 1.0e-6,
                 cost_abs_tol: float | None = None, cost_rel_tol: float | None = None,
                 line_search_max_iterations: int = 40, armijo_c: float = 1.0e-4, rho: float = 0.8,
                 line_search_relative_slop: float | None = None, line_search_variant: str = "armijo_decay",
                 contact_preset_variant: str | None = None, contact_weight_mode: str | None = None,
                 contact_point_mode: str | None = None, capture_contact_jacobian_snapshots: bool = False,
                 use_f64_boundary_pose: bool | None = None, free_motion_solve_precision: str | None = None,
                 contact_solve_precision: str | None = None, contact_linear_solve_precision: str | None = None,
                 sap_contact_weight_precision: str | None = None, collect_iteration_stats: bool = False,
                 check_line_search_errors: bool = False, graph_conditional: bool = True,
                 static_substep: bool = False, static_substep_iterations: int = 8,
                 static_substep_line_search_iterations: int = 6, position_integration: str | None = None,
                 hessian_precision: str | None = None, warm_start: str = "previous_velocity",
                 learned_warm_start=None, learned_candidates: str = "new_contacts", impulse_history: int = 3,
                 plain_start: bool = False,
                 tree_blocked: bool | None = None,
                 work_order: str = "previous_iterations", autotune: bool | str | os.PathLike | None = None):
        """Keyword arguments of the reference's SolverSAP (sim/solver_sap.py:
        749-791) plus: hessian_precision ("fp64" / "fp32": J^T G J assembly and
        factorization precision; the gradient, cost, line search and
        convergence test stay FP64); warm_start, one of
          "previous_velocity"  the reference's: start from the last solution;
          "previous_impulses"  also try v* + A^-1 J^T gamma0, gamma0 the
                               start impulses of the contact history;
          "learned"            also try starts from the per-contact network
                               (learned_warm_start: a LearnedWarmStart, a
                               weights path, or None for the packaged
                               weights); learned_candidates "new_contacts"
                               (default): one start v* + A^-1 J^T gamma0 with
                               gamma0 the history's start impulse where the
                               contact existed last step and the network's
                               where it is new (tiles without a new contact
                               skip the network); "all_contacts": two starts,
                               the network's gamma0 on every contact and the
                               history's start impulses;
        previous impulses are carried to this step's contact slots by
        contact identity (shape pair and witness point), so slots may shift
        as contacts appear and vanish; impulse_history (1, 2 or 3, default
        3): how many past impulses of each contact make its start impulse --
        1 the last one, 2 their linear extrapolation to this step, 3 the
        quadratic one (fewer where the contact is younger); plain_start
        (False): whether the previous-velocity start also competes with the
        candidate on the cost (it wins in about 0.1 % of world-steps on the
        rollouts measured, at the price of one more cost evaluation per
        world); without it the previous velocity is only the fallback when
        the candidate's cost is not finite;
        the candidate start is taken (with plain_start, the lower-cost of it
        and the previous velocity), and Newton always runs to the same
        tolerance;
        work_order ("previous_iterations", the default, or "index"): the
        order in which the persistent solve kernel takes the worlds -- by the
        previous step's Newton iterations, most first, so long solves start
        early instead of trailing at the end of the launch (results do not
        depend on it); tree_blocked (None: automatic) selects the tree-blocked layout for
        worlds made only of free bodies (default beyond 60 DOFs per world:
        A as 6 x 6 blocks, contact rows over the two touching bodies, a block
        sparse Newton factorization), which takes the previous-velocity or
        previous-impulses warm start; autotune (True, or a JSON cache path)
        times the dense solve's resident CTAs per SM on the first solve of
        each problem shape and keeps the fastest (autotune.SolveAutotuner;
        results do not depend on it)."""
        view = _ModelView(model)
        tree_blocked = _pick_tree_blocked(view, tree_blocked)
        preset = dict(_CONTACT_PRESET_KWARGS[_normalize_contact_preset_variant(contact_preset_variant)])
        self.contact_preset_variant = _normalize_contact_preset_variant(contact_preset_variant)
        pick = lambda v, k: preset[k] if v is None else v
        contact_weight_mode = pick(contact_weight_mode, "contact_weight_mode")
        contact_point_mode = pick(contact_point_mode, "contact_point_mode")
        position_integration = pick(position_integration, "position_integration")
        self.contact_linear_solve_precision = _normalize_precision_knob(
            pick(contact_linear_solve_precision, "contact_linear_solve_precision"),
            option_name="contact_linear_solve_precision")
        self.contact_solve_precision = _normalize_precision_knob(pick(contact_solve_precision,
                                                                      "contact_solve_precision"),
                                                                 option_name="contact_solve_precision")
        self.free_motion_solve_precision = _normalize_precision_knob(
            pick(free_motion_solve_precision, "free_motion_solve_precision"),
            option_name="free_motion_solve_precision")
        self.sap_contact_weight_precision = _normalize_precision_knob(
            pick(sap_contact_weight_precision, "sap_contact_weight_precision"),
            option_name="sap_contact_weight_precision")
        self.use_f64_boundary_pose = bool(pick(use_f64_boundary_pose, "use_f64_boundary_pose"))
        self.model = model
        self.max_rigid_contact = int(max_rigid_contact)
        self.max_iterations = int(max_iterations)
        self.optimality_abs_tol, self.optimality_rel_tol = float(optimality_abs_tol), float(optimality_rel_tol)
        self.armijo_c, self.rho = float(armijo_c), float(rho)
        self.line_search_relative_slop = line_search_relative_slop
        self.line_search_variant = normalize_sap_line_search_mode(line_search_variant)
        if self.line_search_variant == "armijo_decay" and not (0.0 < float(rho) < 1.0):
            raise ValueError(f"rho must lie in (0, 1), got {rho!r}.")
        if cost_abs_tol is None:
            cost_abs_tol = 0.0 if self.line_search_variant == "monotone_decay" else 1.0e-30
        if cost_rel_tol is None:
            cost_rel_tol = 5.0e-3 if self.line_search_variant == "monotone_decay" else 1.0e-15
        self.cost_abs_tol, self.cost_rel_tol = float(cost_abs_tol), float(cost_rel_tol)
        self.line_search_max_iterations = int(line_search_max_iterations)
        if self.line_search_variant == "exact_root" and self.line_search_max_iterations == 40:
            self.line_search_max_iterations = 100
        if not bool(graph_conditional):
            raise ValueError("SolverSAP only supports graph_conditional=True; "
                             "the Python contact-solve loop has been removed.")
        self.static_substep = bool(static_substep)
        self.static_substep_iterations = int(static_substep_iterations)
        self.static_substep_line_search_iterations = int(static_substep_line_search_iterations)
        self.position_integration = str(position_integration).strip().lower().replace("-", "_")
        if self.position_integration not in ("sap_euler", "midpoint"):
            raise ValueError(f"position_integration must be 'sap_euler' or 'midpoint', got {position_integration!r}.")
        self.collect_iteration_stats = bool(collect_iteration_stats)
        self.check_line_search_errors = bool(check_line_search_errors)
        tau = model.shape_material_tau.cpu().numpy() if model.shape_material_tau is not None else np.zeros(0)
        explicit = tau[np.isfinite(tau) & (tau >= 0.0)]
        shape_tau = (float(explicit[0]) if explicit.size else 0.0) if contact_tau_d is None else float(contact_tau_d)
        if contact_tau_d is None and shape_tau == 0.0:
            warnings.warn("No contact dissipation authored on the model and no contact_tau_d given: tau_d falls "
                          "back to 0.0.", stacklevel=2)
        self.contact_jacobian = SapContactJacobian(
            model, max_rigid_contact=self.max_rigid_contact, fallback_mu=fallback_mu,
            fallback_stiffness=fallback_stiffness, fallback_tau_d=shape_tau, contact_weight_mode=contact_weight_mode,
            contact_point_mode=contact_point_mode, tree_blocked=tree_blocked, _view=view)
        # the solve-side fallback is per pair: tau(shape0) + tau(shape1) (sim/solver_sap.py:945-955)
        self.contact_solve = SapContactSolve(
            model, max_rigid_contact=self.max_rigid_contact, contact_beta=contact_beta, contact_sigma=contact_sigma,
            contact_tau_d=2.0 * shape_tau, block_size=block_size, diag_shift=diag_shift,
            solve_precision=self.contact_solve_precision, linear_solve_precision=self.contact_linear_solve_precision,
            hessian_precision=hessian_precision, tree_blocked=tree_blocked, _view=view)
        self.view = view
        self.num_envs, self.dof_count, self.dof_per_env = view.W, int(model.joint_dof_count), view.n
        dev = view.device
        self._v_guess_active = torch.zeros(1, dtype=I32, device=dev)
        self._q_out_tmp = torch.zeros(int(model.joint_coord_count), dtype=F64, device=dev)
        self._tail = _abi.StepTail()
        # public-order boundary (sim/solver_sap.py:1198-1261): SAP-order copies of
        # public inputs, and FP64 staging of public outputs
        D, Bt = int(model.joint_dof_count), int(model.body_count)
        self._qd_sap_in = torch.zeros(D, dtype=F64, device=dev)
        self._f_sap_in = torch.zeros(D, dtype=F64, device=dev)
        self._bf_sap_in = torch.zeros(Bt, 6, dtype=F64, device=dev)
        self._qd_pub_out = torch.zeros(D, dtype=F64, device=dev)
        self._body_q_out = torch.zeros(Bt, 7, dtype=F64, device=dev)
        self._body_qd_out = torch.zeros(Bt, 6, dtype=F64, device=dev)
        self.stage_events = None  # list -> per-stage CUDA events (see _mark)
        self.warm_start = str(warm_start).strip().lower().replace("-", "_")
        if self.warm_start not in ("previous_velocity", "previous_impulses", "learned"):
            raise ValueError("warm_start must be 'previous_velocity', 'previous_impulses' or 'learned', "
                             f"got {warm_start!r}.")
        self.learned_candidates = str(learned_candidates).strip().lower().replace("-", "_")
        if self.learned_candidates not in ("new_contacts", "all_contacts"):
            raise ValueError(f"learned_candidates must be 'new_contacts' or 'all_contacts', got {learned_candidates!r}.")
        self.learned_warm_start = None
        if self.warm_start == "learned":
            from .warmstart import DEFAULT_WEIGHTS, LearnedWarmStart

            lw = learned_warm_start
            if lw is None or isinstance(lw, (str, os.PathLike)):
                lw = LearnedWarmStart.load(DEFAULT_WEIGHTS if lw is None else str(lw), dev)
            self.learned_warm_start = lw
        C = self.max_rigid_contact
        self.impulse_history = int(impulse_history)
        self.plain_start = bool(plain_start)
        if self.impulse_history not in (1, 2, 3):
            raise ValueError(f"impulse_history must be 1, 2 or 3, got {impulse_history!r}.")
        # candidate impulse sets: [0] the network's, [1] the history's start
        # impulses (evaluated last: it is the usual winner, and the last
        # candidate's evaluation seeds the first Newton iteration)
        self._gamma_cand = torch.zeros(2, view.W, max(C, 1), 3, dtype=F64, device=dev)
        # [1] holds the start impulses of this step's slots: the last solves'
        # impulses carried by contact identity (sapb_contact_history_update)
        # from the last solve's impulses by its own slots (the solve's
        # contact_gamma, read before this step's solve rewrites it) and
        # extrapolated over the impulses before them (_gamma_carried: the
        # last solve's by this step's slots, _gamma_older: the one before)
        self._gamma_prev = self._gamma_cand[1]
        self._gamma_carried = torch.zeros(view.W, max(C, 1), 3, dtype=F64, device=dev)
        self._gamma_older = torch.zeros(view.W, max(C, 1), 3, dtype=F64, device=dev)
        self._normal_up = torch.zeros(view.W, max(C, 1), dtype=F64, device=dev)
        self._v_start = None
        if self.warm_start != "previous_velocity":
            self._hist_key_shape = torch.zeros(view.W, max(C, 1), 2, dtype=I32, device=dev)
            self._hist_key_point = torch.zeros(view.W, max(C, 1), 3, dtype=F64, device=dev)
            self._hist_key_count = torch.zeros(view.W, dtype=I32, device=dev)
            self.has_history = torch.zeros(view.W, max(C, 1), dtype=I32, device=dev)
            # the contact history, run by the free-motion launch on its slots:
            # the last solve's impulses (contact_gamma, by its slots) carried by
            # contact identity and extrapolated into the start impulses
            H = _abi.ContactHistory()
            H.key_shape, H.key_point = _ptr(self._hist_key_shape), _ptr(self._hist_key_point)
            H.key_count = _ptr(self._hist_key_count)
            H.gamma_prev, H.gamma_hist, H.has_history = (_ptr(self.contact_solve.contact_gamma),
                                                         _ptr(self._gamma_carried),
                                                         _ptr(self.has_history))
            H.order, H.gamma_older, H.gamma_start = (self.impulse_history, _ptr(self._gamma_older),
                                                     _ptr(self._gamma_prev))
            if not self.contact_solve.tree_blocked:
                # the start velocity v* + A^-1 J^T gamma_start, formed by the
                # free motion with its own factor of A
                self._v_start = torch.zeros(view.W * view.n, dtype=F64, device=dev)
            self.contact_jacobian.set_history(
                H, v_start=self._v_start,
                factor_new_contacts_only=(self.warm_start == "learned" and self.learned_candidates == "new_contacts"
                                          and not self.contact_solve.tree_blocked))
        if self.learned_warm_start is not None:
            self.learned_warm_start.set_regularization(contact_beta, contact_sigma, 2.0 * shape_tau)
            # network inputs J_c v* and, for the network's impulses, the
            # factor of A (new contacts only in the new_contacts mode; the
            # tree-blocked solve factors A's tree blocks itself)
            if self.contact_solve.tree_blocked:
                self.contact_jacobian.keep_contact_velocities()
            else:
                self.contact_jacobian.keep_dynamics_factor()
            self._gamma_zero = torch.zeros(view.W, max(C, 1), 3, dtype=F64, device=dev)
        self.work_order = str(work_order).strip().lower().replace("-", "_")
        if self.work_order not in ("previous_iterations", "index"):
            raise ValueError(f"work_order must be 'previous_iterations' or 'index', got {work_order!r}.")
        if self.work_order == "previous_iterations" and view.W > 32768:
            self.work_order = "index"  # the device sort of the work order holds at most 32768 worlds
        self._world_order = torch.arange(view.W, dtype=I32, device=dev)
        if autotune:
            from .autotune import SolveAutotuner

            self.contact_solve.autotuner = SolveAutotuner(None if autotune is True else autotune)
        self.reset_runtime_state()

    @property
    def device(self):
        return self.view.device

    def get_max_contact_count(self) -> int:
        return int(self.max_rigid_contact) * max(int(self.num_envs), 1)

    def close(self) -> None:
        pass

    def notify_model_changed(self, flags: int) -> None:
        return

    def c_step_options(self) -> _abi.StepOptions:
        """This solver's configuration as the options of the C step handle
        (sapb_create / sapb_step): the same contact preparation, solve
        options, integrator, warm start (previous velocity or previous
        impulses, with the same impulse history) and work order, so a C host stepping the same model gets
        the same trajectory."""
        if self.warm_start == "learned" and self.learned_candidates != "new_contacts":
            raise NotImplementedError("the C step handle runs the learned start on new contacts only")
        if self.static_substep:
            iters, ls_iters = self.static_substep_iterations, self.static_substep_line_search_iterations
        else:
            iters, ls_iters = self.max_iterations, self.line_search_max_iterations
        _, solve = self.contact_solve.solve_options(
            self.line_search_variant, max_iterations=iters, optimality_abs_tol=self.optimality_abs_tol,
            optimality_rel_tol=self.optimality_rel_tol, cost_abs_tol=self.cost_abs_tol,
            cost_rel_tol=self.cost_rel_tol, line_search_max_iterations=ls_iters, armijo_c=self.armijo_c,
            rho=self.rho, line_search_relative_slop=self.line_search_relative_slop)
        o = _abi.StepOptions()
        o.prepare = _abi.PrepareOptions.from_buffer_copy(self.contact_jacobian.opts)
        o.solve = solve
        o.solve.skip_plain_start = 0 if self.plain_start else 1
        o.position_integration = (_abi.SAPB_INTEGRATE_MIDPOINT if self.position_integration == "midpoint"
                                  else _abi.SAPB_INTEGRATE_SAP_EULER)
        o.warm_start = {"previous_impulses": _abi.SAPB_WARM_START_PREVIOUS_IMPULSES,
                        "learned": _abi.SAPB_WARM_START_LEARNED}.get(self.warm_start,
                                                                     _abi.SAPB_WARM_START_PREVIOUS_VELOCITY)
        if self.warm_start == "learned":
            # the network by reference: its device weights stay with this solver
            lw = self.learned_warm_start
            net = _abi.StepNetwork()
            net.packed, net.bias = lw.mlp.packed.data_ptr(), lw.mlp.bias.data_ptr()
            net.norm = lw.norm_struct
            net.feature_tau_d = float(lw.tau_fallback)
            net.impulse_tau_d = float(lw.solve_options.contact_tau_d)
            self._c_network = net
            o.network = ctypes.pointer(net)
        o.work_order = (_abi.SAPB_WORK_ORDER_PREVIOUS_ITERATIONS if self.work_order == "previous_iterations"
                        else _abi.SAPB_WORK_ORDER_INDEX)
        o.impulse_history = self.impulse_history
        return o

    def capture_steps(self, state_a: SapState, state_b: SapState, control: SapControl | None, contacts, dt,
                      warmup: int = 1) -> "torch.cuda.CUDAGraph":
        """Capture two consecutive steps (state_a -> state_b -> state_a) in one
        CUDA graph; each replay advances the rollout by two steps with every
        launch of both steps (free motion, warm start, solve, integration)
        replayed without host work.  `warmup` eager step pairs run first (they
        advance the rollout too) so the capture sees no first-call setup."""
        if not isinstance(dt, (int, float)):
            raise TypeError("capture_steps needs a scalar dt (it is baked into the graph)")
        side = torch.cuda.Stream(self.view.device)
        side.wait_stream(torch.cuda.current_stream(self.view.device))
        with torch.cuda.stream(side):
            for _ in range(max(int(warmup), 1)):
                self.step(state_a, state_b, control, contacts, dt)
                self.step(state_b, state_a, control, contacts, dt)
        torch.cuda.current_stream(self.view.device).wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, capture_error_mode="thread_local"):
            self.step(state_a, state_b, control, contacts, dt)
            self.step(state_b, state_a, control, contacts, dt)
        return graph

    def capture_host_steps(self, host_state: dict, host_contacts: tuple, state_a: SapState, state_b: SapState,
                           control: SapControl | None, dt, warmup: int = 1) -> "HostStepGraph":
        """Two consecutive steps fed from and returned to pinned host memory,
        captured in one CUDA graph.  Every step copies its state
        (`host_state["joint_q"]`, `["joint_qd"]`) host -> device, steps, and
        copies the new state back into the same host tensors; step k of a
        pair takes its contacts from `host_contacts[k]` (SapContacts of
        pinned host tensors).  Each step's contacts are copied into one of
        two device buffers on a second stream while the step before it
        computes, so that copy overlaps the step; the graph joins the copy
        stream before it ends, so one replay holds all the copies of its two
        steps.  The host contacts of the first step of a pair are read
        during the second step of the previous replay.  `warmup` eager pairs
        (the same copies and steps) run first and advance the rollout."""
        if not isinstance(dt, (int, float)):
            raise TypeError("capture_host_steps needs a scalar dt (it is baked into the graph)")
        if len(host_contacts) != 2:
            raise ValueError("host_contacts holds the contacts of the two steps of a pair")
        for name in ("joint_q", "joint_qd"):
            if not host_state[name].is_pinned():
                raise ValueError(f"host_state[{name!r}] must be pinned host memory")
        fields = [k for k, v in vars(host_contacts[0]).items() if isinstance(v, torch.Tensor)]
        for hc in host_contacts:
            for k in fields:
                t = getattr(hc, k)
                if t is None or not t.is_pinned():
                    raise ValueError(f"host contacts {k!r} must be pinned host tensors in both sets")
        dev = self.view.device
        dev_contacts = tuple(SapContacts(**{k: getattr(hc, k).to(dev) for k in fields}) for hc in host_contacts)
        main = torch.cuda.current_stream(dev)
        copy = torch.cuda.Stream(dev)

        def put(dst: SapContacts, src: SapContacts):
            for k in fields:
                getattr(dst, k).copy_(getattr(src, k), non_blocking=True)

        def pair():
            cur = torch.cuda.current_stream(dev)
            for k, (a, b) in enumerate(((state_a, state_b), (state_b, state_a))):
                # the state first (the step waits for it), then the other
                # buffer's contacts on the copy stream while this step runs:
                # the second step's, then the next pair's first step's
                a.joint_q.copy_(host_state["joint_q"], non_blocking=True)
                a.joint_qd.copy_(host_state["joint_qd"], non_blocking=True)
                if k == 1:
                    cur.wait_stream(copy)  # this step's contacts (copied during the first step)
                copy.wait_stream(cur)  # the buffer is free once the step before this one ended
                with torch.cuda.stream(copy):
                    put(dev_contacts[1 - k], host_contacts[1 - k])
                self.step(a, b, control, dev_contacts[k], dt)
                host_state["joint_q"].copy_(b.joint_q, non_blocking=True)
                host_state["joint_qd"].copy_(b.joint_qd, non_blocking=True)
            cur.wait_stream(copy)

        side = torch.cuda.Stream(dev)
        side.wait_stream(main)
        with torch.cuda.stream(side):
            for _ in range(max(int(warmup), 1)):
                pair()
        main.wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, capture_error_mode="thread_local"):
            pair()
        return HostStepGraph(graph, dev_contacts, copy)

    def _mark(self, stage: str | None) -> None:
        """Stage timing: when `stage_events` is a list, record a CUDA event on
        the current stream at each stage boundary as (stage, event); the
        stage ends at the next record (None closes the step)."""
        if self.stage_events is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(torch.cuda.current_stream(self.view.device))
            self.stage_events.append((stage, ev))

    def stage_times(self) -> dict:
        """Milliseconds per stage summed over the recorded steps (syncs)."""
        out: dict = {}
        ev = self.stage_events or []
        if ev:
            ev[-1][1].synchronize()
        for (name, e0), (_, e1) in zip(ev[:-1], ev[1:]):
            if name is not None:
                out[name] = out.get(name, 0.0) + e0.elapsed_time(e1)
        return out

    def reset_runtime_state(self, state: SapState | None = None) -> None:
        """sim/solver_sap.py:1004-1017"""
        self.sim_time = 0.0
        self.frame_id = 0
        self.last_contact_count = 0
        self.last_truncated_contact_count = 0
        self.last_solve_iterations = 0
        self.last_line_search_iterations = 0
        self.last_converged = True
        self._v_guess_active.zero_()
        if hasattr(self, "_gamma_cand"):
            self._gamma_cand.zero_()
            self._gamma_carried.zero_()
            self._gamma_older.zero_()
        if hasattr(self, "_hist_key_count"):
            self._hist_key_count.zero_()
            self.has_history.zero_()
        if hasattr(self, "_world_order"):
            torch.arange(self.view.W, dtype=I32, device=self.view.device, out=self._world_order)
        self.last_contacts = None
        self.last_contact_jacobian_result = None
        self.last_contact_solve_result = None

    def step(self, state_in: SapState, state_out: SapState, control: SapControl | None, contacts, dt) -> SapState:
        """sim/solver_sap.py:1388-1494"""
        if getattr(state_in, "requires_grad", False):
            raise NotImplementedError("SolverSAP does not support grad states.")
        if not isinstance(state_in, SapState):
            raise TypeError("SolverSAP.step requires SapState input.")
        if not isinstance(state_out, SapState):
            raise TypeError("SolverSAP.step requires SapState output.")
        if control is not None and not isinstance(control, SapControl):
            raise TypeError("SolverSAP.step requires SapControl.")
        if contacts is None:
            contacts = SapContacts()
        if not isinstance(contacts, SapContacts):
            contacts = sap_contacts_from_newton(contacts)
        for s, name in ((state_in, "state_in"), (state_out, "state_out")):
            if getattr(s, "joint_qd_order", "sap") not in ("sap", "public"):
                raise ValueError(f"Unsupported SapState joint_qd_order={s.joint_qd_order!r}.")
        self.contact_jacobian.set_dt(dt)
        self.last_contacts = contacts
        mark = self._mark
        solve_state, solve_control, output_public = self._boundary_in(state_in, state_out, control)
        mark("free_motion")
        cr = self.contact_jacobian.compute(solve_state, contacts, control=solve_control)
        if self.static_substep:
            iters, ls_iters = self.static_substep_iterations, self.static_substep_line_search_iterations
        else:
            iters, ls_iters = self.max_iterations, self.line_search_max_iterations
        v0 = self.contact_jacobian._qd
        # the solve's start velocity in its own layout (uneven batches: slots
        # of the largest world's DOF count, written by the free motion)
        v0_solve = self.contact_jacobian.qd_slots if self.view.uneven else v0
        mark("warm_start")
        # the contact history ran inside the free-motion launch: _gamma_prev
        # holds the start impulses, _v_start the start velocity
        gamma0 = v_cands = gamma0_base = None
        if self.warm_start == "previous_impulses":
            if self._v_start is not None:
                v_cands = self._v_start
            else:
                gamma0 = self._gamma_prev  # tree-blocked: the solve maps them tree by tree
        elif self.warm_start == "learned" and self.contact_solve.tree_blocked:
            # one impulse set for the tree-blocked candidate: the history's
            # start impulses where a contact has them, the network's on new
            # contacts (the solve forms v* + A^-1 J^T gamma tree by tree)
            self._normal_up.copy_(cr.contact_env_R_WC[..., 2, 2])
            self.learned_warm_start.predict(
                num_envs=self.view.W, dof_per_env=int(cr.contact_env_jacobian.shape[-1]),
                max_contacts=self.max_rigid_contact, normal_up=self._normal_up, gamma_prev=self._gamma_prev,
                out=self._gamma_cand[0], vc_star=self.contact_jacobian.contact_env_vc_star,
                contact_count=cr.contact_env_count, dynamics_matrix=None, jacobian=cr.contact_env_jacobian,
                phi0=cr.contact_env_phi0, w_eff=cr.contact_env_w_eff, mu=cr.contact_env_mu,
                stiffness=cr.contact_env_stiffness, tau_d=cr.contact_env_tau_d, v_star=self.contact_jacobian.v_star,
                v0=self.contact_jacobian.v_star, dt=self.contact_jacobian.dt_world, has_history=self.has_history)
            gamma0 = self._gamma_cand[0]
        elif self.warm_start == "learned":
            self._normal_up.copy_(cr.contact_env_R_WC[..., 2, 2])
            # new_contacts: the network's impulses on new contacts only (zero
            # where the start velocity already holds the history's), added to
            # the start velocity through A^-1 J^T; all_contacts: the network
            # corrects the carried impulses, a set of its own beside the
            # start velocity
            new_only = self.learned_candidates == "new_contacts"
            self.learned_warm_start.predict(
                num_envs=self.view.W, dof_per_env=self.view.n, max_contacts=self.max_rigid_contact,
                normal_up=self._normal_up, gamma_prev=self._gamma_zero if new_only else self._gamma_carried,
                out=self._gamma_cand[0],
                vc_star=self.contact_jacobian.contact_env_vc_star,
                contact_count=cr.contact_env_count, dynamics_matrix=cr.dynamics_matrix_env,
                jacobian=cr.contact_env_jacobian, phi0=cr.contact_env_phi0, w_eff=cr.contact_env_w_eff,
                mu=cr.contact_env_mu, stiffness=cr.contact_env_stiffness, tau_d=cr.contact_env_tau_d,
                v_star=self.contact_jacobian.v_star, v0=self.contact_jacobian.v_star,
                dt=self.contact_jacobian.dt_world,
                has_history=self.has_history if self.learned_candidates == "new_contacts" else None)
            gamma0 = self._gamma_cand[0:1]
            if new_only:
                gamma0_base = self._v_start
            else:
                v_cands = self._v_start
        mark("contact_solve")
        sr = self.contact_solve.solve(
            cr, solve_state, solve_control, self.contact_jacobian.dt_world, self.contact_jacobian.v_star, v0=v0_solve,
            v_guess=self.contact_solve.v_flat, v_guess_active=self._v_guess_active, gamma0=gamma0,
            v_candidates=v_cands, gamma0_base=gamma0_base, skip_plain_start=not self.plain_start,
            max_iterations=iters,
            optimality_abs_tol=self.optimality_abs_tol, optimality_rel_tol=self.optimality_rel_tol,
            cost_abs_tol=self.cost_abs_tol, cost_rel_tol=self.cost_rel_tol, line_search_max_iterations=ls_iters,
            armijo_c=self.armijo_c, rho=self.rho, line_search_relative_slop=self.line_search_relative_slop,
            line_search_variant=self.line_search_variant,
            world_order=self._world_order if self.work_order == "previous_iterations" else None)
        if self.work_order == "previous_iterations":
            # next step's queue: most Newton iterations first (stable: ties keep index order)
            check(load().sapb_world_order(_ptr(sr.newton_iterations_env), self.view.W, _ptr(self._world_order),
                                          ctypes.c_void_p(torch.cuda.current_stream(self.view.device).cuda_stream)),
                  "sapb_world_order")
        mark("integrate")
        # the tail in one launch (sapb_step_tail_launch): position integration
        # (sim/solver_sap.py:1267-1386), the new velocities in the output's
        # order and, for a public-order output, the forward kinematics of the
        # new pose (:1467-1469); outputs written in place when they are
        # contiguous FP64, else staged and copied
        T = self._tail
        q_in = self.contact_jacobian._q
        direct = lambda t, n: (t is not None and t.dtype == F64 and t.is_contiguous() and t.numel() == n)
        q_out = state_out.joint_q if (direct(state_out.joint_q, q_in.numel())
                                      and state_out.joint_q.data_ptr() != q_in.data_ptr()) else self._q_out_tmp
        qd_out = state_out.joint_qd if direct(state_out.joint_qd, self._qd_pub_out.numel()) else self._qd_pub_out
        T.joint_q_in, T.v_prev, T.v_new = _ptr(q_in), _ptr(v0), _ptr(sr.v_flat)
        T.dt = _ptr(self.contact_jacobian.dt_world)
        T.mode = _abi.SAPB_INTEGRATE_MIDPOINT if self.position_integration == "midpoint" else _abi.SAPB_INTEGRATE_SAP_EULER
        T.qd_public = 1 if output_public else 0
        T.joint_q_out, T.joint_qd_out = _ptr(q_out), _ptr(qd_out)
        bq_out = bqd_out = None
        if output_public:
            nb = self._body_q_out.numel()
            bq_out = state_out.body_q if direct(state_out.body_q, nb) else self._body_q_out
            if getattr(state_out, "body_qd", None) is not None:
                bqd_out = state_out.body_qd if direct(state_out.body_qd, self._body_qd_out.numel()) \
                    else self._body_qd_out
        T.body_q_out, T.body_qd_out = _ptr(bq_out), _ptr(bqd_out)
        check(load().sapb_step_tail_launch(ctypes.byref(self.view.desc), ctypes.byref(T),
                                           ctypes.c_void_p(torch.cuda.current_stream(self.view.device).cuda_stream)),
              "sapb_step_tail_launch")
        if q_out is not state_out.joint_q:
            state_out.joint_q.copy_(q_out.reshape(state_out.joint_q.shape))
        if qd_out is not state_out.joint_qd:
            state_out.joint_qd.copy_(qd_out.reshape(state_out.joint_qd.shape))
        if bq_out is not None and bq_out is not state_out.body_q and state_out.body_q is not None:
            state_out.body_q.copy_(bq_out.reshape(state_out.body_q.shape))
        if bqd_out is not None and bqd_out is not state_out.body_qd:
            state_out.body_qd.copy_(bqd_out.reshape(state_out.body_qd.shape))
        if state_out.body_f is not None and state_in.body_f is not None and state_out.body_f is not state_in.body_f:
            state_out.body_f.copy_(state_in.body_f)
        mark(None)
        self._v_guess_active.fill_(1)  # warm start from this step's solution (sim/solver_sap.py:1441-1451)
        self.last_contact_jacobian_result = cr
        self.last_contact_solve_result = sr
        self.last_solve_iterations = -1
        self.last_line_search_iterations = -1
        self.last_converged = True
        if not isinstance(dt, torch.Tensor):
            self.sim_time += float(dt)
        self.frame_id += 1
        return state_out

    def _boundary_in(self, state_in: SapState, state_out: SapState, control: SapControl | None):
        """Public-order inputs -> SAP order (sim/solver_sap.py:1198-1261):
        returns the SAP-order state and control the step runs on, and whether
        the output is public."""
        lib, stream = load(), ctypes.c_void_p(torch.cuda.current_stream(self.view.device).cuda_stream)
        desc = ctypes.byref(self.view.desc)
        if getattr(state_in, "joint_qd_order", "sap") == "public":
            q = _f64(state_in.joint_q)
            bf_pub = None
            if state_in.body_f is not None and getattr(state_in, "body_f_order", "sap") == "public":
                bf_pub = _f64(state_in.body_f.reshape(-1, 6))
            bq = _f64(state_in.body_q.reshape(-1, 7)) if bf_pub is not None else None
            check(lib.sapb_public_to_sap(desc, _ptr(q), _ptr(bq), _ptr(_f64(state_in.joint_qd)), None,
                                         _ptr(bf_pub), _ptr(self._qd_sap_in), None, _ptr(self._bf_sap_in), stream),
                  "sapb_public_to_sap")
            state_in = SapState(joint_q=state_in.joint_q, joint_qd=self._qd_sap_in, body_q=state_in.body_q,
                                body_qd=getattr(state_in, "body_qd", None),
                                body_f=self._bf_sap_in if bf_pub is not None else state_in.body_f,
                                joint_qd_order="sap", body_f_order="sap")
        if control is not None and getattr(control, "joint_f_order", "sap") == "public" and control.joint_f is not None:
            q = _f64(state_in.joint_q)
            check(lib.sapb_public_to_sap(desc, _ptr(q), None, None, _ptr(_f64(control.joint_f)), None, None,
                                         _ptr(self._f_sap_in), None, stream), "sapb_public_to_sap")
            control = SapControl(joint_f=self._f_sap_in, joint_target_pos=control.joint_target_pos,
                                 joint_target_vel=control.joint_target_vel, joint_act=control.joint_act,
                                 joint_f_order="sap")
        return state_in, control, getattr(state_out, "joint_qd_order", "sap") == "public"

    def update_contacts(self, contacts: SapContacts) -> None:
        raise NotImplementedError("SolverSAP does not expose contact-force writeback yet.")


__all__ = ["SolverSAP", "SapFreeMotion", "SapContactJacobian", "SapContactSolve", "SapFreeMotionResult",
           "SapContactJacobianResult", "SapContactSolveResult", "SAP_CONTACT_PRESET_VARIANTS"]
