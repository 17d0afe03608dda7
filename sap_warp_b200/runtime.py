"""SAP runtime containers (drop-in for sim/sap_runtime.py:47-264), holding
torch tensors instead of Warp arrays.

Field names, shapes and meanings follow the reference so that code written
against SapModel / SapState / SapControl / SapContacts keeps working.  Real
model data is FP64 (the reference keeps FP64 mirrors of every field the SAP
step reads, `sap_debug_*`); joint types and indices are int32.  Joint
coordinates, velocities and forces are flat over all worlds, in SAP DOF
order (free joint: [angular, linear]).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Literal

import torch

SAP_JOINT_PRISMATIC = 0
SAP_JOINT_REVOLUTE = 1
SAP_JOINT_BALL = 2
SAP_JOINT_FIXED = 3
SAP_JOINT_FREE = 4
SAP_JOINT_DISTANCE = 5
SAP_JOINT_D6 = 6
SAP_JOINT_TARGET_NONE = 0

SapDofOrder = Literal["sap", "public"]


@dataclass(frozen=True)
class SapModel:
    """Immutable model arrays (sim/sap_runtime.py:47-174)."""

    device: Any
    joint_count: int
    joint_dof_count: int
    joint_coord_count: int
    body_count: int
    articulation_count: int
    world_count: int
    shape_count: int
    requires_grad: bool

    joint_type: torch.Tensor  # int32 [J]
    joint_articulation: torch.Tensor  # int32 [J]
    joint_parent: torch.Tensor  # int32 [J] parent body or -1
    joint_child: torch.Tensor  # int32 [J] child body
    joint_q_start: torch.Tensor  # int32 [J+1]
    joint_qd_start: torch.Tensor  # int32 [J+1]
    joint_dof_dim: torch.Tensor  # int32 [J, 2] (linear, angular) axis counts
    joint_axis: torch.Tensor  # f64 [dofs, 3]
    joint_X_p: torch.Tensor  # f64 [J, 7] (p, q xyzw) joint frame in the parent body
    joint_X_c: torch.Tensor  # f64 [J, 7] joint frame in the child body
    joint_ancestor: torch.Tensor  # int32 [J] parent joint or -1
    articulation_start: torch.Tensor  # int32 [A+1]
    joint_q: torch.Tensor  # f64 [coords]
    joint_qd: torch.Tensor  # f64 [dofs]

    body_q: torch.Tensor  # f64 [B, 7]
    body_qd: torch.Tensor  # f64 [B, 6]
    body_mass: torch.Tensor  # f64 [B]
    body_inertia: torch.Tensor  # f64 [B, 3, 3] about the COM, body axes
    body_com: torch.Tensor  # f64 [B, 3] in the body frame
    body_flags: torch.Tensor  # int32 [B]
    body_world: torch.Tensor  # int32 [B]
    gravity: torch.Tensor  # f64 [W, 3]
    joint_armature: torch.Tensor  # f64 [dofs]

    shape_body: torch.Tensor  # int32 [S] (-1: static)
    shape_material_mu: torch.Tensor | None
    shape_material_ke: torch.Tensor | None
    shape_material_tau: torch.Tensor | None

    joint_target_mode: torch.Tensor  # int32 [dofs]
    joint_target_ke: torch.Tensor  # f32 [dofs]
    joint_target_kd: torch.Tensor  # f32 [dofs]
    joint_target_pos: torch.Tensor  # f32 [dofs]
    joint_target_vel: torch.Tensor  # f32 [dofs]
    joint_f: torch.Tensor  # f64 [dofs]
    joint_act: torch.Tensor  # f32 [dofs]
    joint_effort_limit: torch.Tensor  # f32 [dofs]
    joint_limit_lower: torch.Tensor  # f64 [dofs]
    joint_limit_upper: torch.Tensor  # f64 [dofs]
    joint_limit_ke: torch.Tensor  # f64 [dofs]
    joint_limit_kd: torch.Tensor  # f64 [dofs]

    up_axis: int = 2
    body_label: tuple = ()
    joint_label: tuple = ()
    # uneven batches (an extension: worlds of different sizes in one model):
    # int32 [W+1] offsets of each world's joints, bodies, DOFs and
    # articulations in the arrays above; None: equal per-world blocks
    world_joint_start: torch.Tensor | None = None
    world_body_start: torch.Tensor | None = None
    world_dof_start: torch.Tensor | None = None
    world_articulation_start: torch.Tensor | None = None

    def state(self, requires_grad: bool | None = None) -> "SapState":
        """A SapState initialised from the model's joint and body arrays."""
        return SapState(
            joint_q=self.joint_q.clone(),
            joint_qd=self.joint_qd.clone(),
            body_q=self.body_q.clone(),
            body_qd=self.body_qd.clone(),
            body_f=torch.zeros_like(self.body_qd),
            joint_qd_order="sap",
            body_f_order="sap",
        )

    def control(self, requires_grad: bool | None = None, clone_variables: bool = True) -> "SapControl":
        """A SapControl initialised from the model's force, target and actuation arrays."""
        c = (lambda t: t.clone()) if clone_variables else (lambda t: t)
        return SapControl(
            joint_f=c(self.joint_f),
            joint_target_pos=c(self.joint_target_pos),
            joint_target_vel=c(self.joint_target_vel),
            joint_act=c(self.joint_act),
            joint_f_order="sap",
        )


@dataclass(frozen=True)
class SapState:
    """Mutable state (sim/sap_runtime.py:177-205)."""

    joint_q: torch.Tensor
    joint_qd: torch.Tensor
    body_q: torch.Tensor
    body_qd: torch.Tensor | None = None
    body_f: torch.Tensor | None = None  # f64 [B, 6]: the negated applied wrench at the body origin, SAP order
    joint_qd_order: SapDofOrder = "sap"
    body_f_order: SapDofOrder = "sap"
    requires_grad: bool = False

    def clear_forces(self) -> None:
        """Clear external body forces in place."""
        if self.body_f is not None:
            self.body_f.zero_()

    def assign(self, other: "SapState") -> None:
        """Copy every state array from `other` (matching optional buffers)."""
        for name in ("joint_q", "joint_qd", "body_q", "body_qd", "body_f"):
            dst, src = getattr(self, name, None), getattr(other, name, None)
            if dst is None and src is None:
                continue
            if dst is None or src is None:
                raise ValueError(f"SapState assign mismatch for {name}")
            dst.copy_(src)


@dataclass(frozen=True)
class SapControl:
    """Control inputs (sim/sap_runtime.py:208-227)."""

    joint_f: torch.Tensor
    joint_target_pos: torch.Tensor | None = None
    joint_target_vel: torch.Tensor | None = None
    joint_act: torch.Tensor | None = None
    joint_f_order: SapDofOrder = "sap"

    def clear(self) -> None:
        """Zero forces, targets and actuation in place."""
        for t in (self.joint_f, self.joint_target_pos, self.joint_target_vel, self.joint_act):
            if t is not None:
                t.zero_()


@dataclass(frozen=True)
class SapContacts:
    """Flat rigid-contact buffer produced by collision (sim/sap_runtime.py:230-264):
    witness points in the body frames of their shapes, normal in world
    pointing from shape0 to shape1, per-shape margins."""

    rigid_contact_count: torch.Tensor | None = None  # int32 [1]
    rigid_contact_shape0: torch.Tensor | None = None  # int32 [N]
    rigid_contact_shape1: torch.Tensor | None = None
    rigid_contact_point0: torch.Tensor | None = None  # f32 [N, 3]
    rigid_contact_point1: torch.Tensor | None = None
    rigid_contact_normal: torch.Tensor | None = None  # f32 [N, 3]
    rigid_contact_margin0: torch.Tensor | None = None  # f32 [N]
    rigid_contact_margin1: torch.Tensor | None = None
    rigid_contact_point0d: torch.Tensor | None = None  # optional f64 mirrors
    rigid_contact_point1d: torch.Tensor | None = None
    rigid_contact_normald: torch.Tensor | None = None
    rigid_contact_margin0d: torch.Tensor | None = None
    rigid_contact_margin1d: torch.Tensor | None = None
    hydro_contact_arrays: Any | None = None

    @property
    def has_rigid_contacts(self) -> bool:
        return self.rigid_contact_count is not None

    @property
    def has_f64_rigid_contacts(self) -> bool:
        return all(getattr(self, k) is not None for k in (
            "rigid_contact_point0d", "rigid_contact_point1d", "rigid_contact_normald",
            "rigid_contact_margin0d", "rigid_contact_margin1d"))


def _as_tensor(x, device=None):
    """Zero-copy view of a foreign array through DLPack or the CUDA array
    interface (Warp/Newton arrays provide both), else torch.as_tensor."""
    if x is None or isinstance(x, torch.Tensor):
        return x
    if hasattr(x, "__dlpack__"):
        return torch.from_dlpack(x)
    if hasattr(x, "__cuda_array_interface__"):
        return torch.as_tensor(x, device=device if device is not None else "cuda")
    return torch.as_tensor(x, device=device)


def sap_contacts_from_newton(contacts) -> SapContacts:
    """Wrap a Newton contact buffer (sim/sap_runtime.py:421-442)."""
    if isinstance(contacts, SapContacts):
        return contacts
    if contacts is None:
        return SapContacts()
    names = [f.name for f in SapContacts.__dataclass_fields__.values() if f.name != "hydro_contact_arrays"]
    return SapContacts(**{k: _as_tensor(getattr(contacts, k, None)) for k in names})


def sap_state_from_newton(state) -> SapState:
    """Wrap a Newton state (sim/sap_runtime.py:388-404); public DOF order."""
    if isinstance(state, SapState):
        return state
    return SapState(joint_q=_as_tensor(state.joint_q), joint_qd=_as_tensor(state.joint_qd),
                    body_q=_as_tensor(state.body_q), body_qd=_as_tensor(getattr(state, "body_qd", None)),
                    body_f=_as_tensor(getattr(state, "body_f", None)), joint_qd_order="public",
                    body_f_order="public")


def sap_control_from_newton(control) -> SapControl:
    """Wrap a Newton control (sim/sap_runtime.py:407-418); public DOF order."""
    if isinstance(control, SapControl):
        return control
    return SapControl(joint_f=_as_tensor(control.joint_f),
                      joint_target_pos=_as_tensor(getattr(control, "joint_target_pos", None)),
                      joint_target_vel=_as_tensor(getattr(control, "joint_target_vel", None)),
                      joint_act=_as_tensor(getattr(control, "joint_act", None)), joint_f_order="public")


Model = SapModel
State = SapState
Control = SapControl
