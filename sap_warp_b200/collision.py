"""Contact generation for primitive shapes on the GPU (sapb_generate_contacts):
planes, spheres and boxes into the flat SapContacts buffer the step reads.

The reference takes its contacts from its collision pipeline
(sim/collision/pipeline.py); this covers the primitive pairs of the
synthetic scenes (plane-sphere, plane-box, sphere-sphere, sphere-box,
box-box vertex-face) so that scenes of boxes and spheres can be stepped with
contacts that follow the bodies, without the reference's collision code.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _abi
from ._lib import check, load
from .runtime import SapContacts

F64, I32 = torch.float64, torch.int32


@dataclass
class ShapeSet:
    """Host description of the shapes: `shapes_per_world` local shapes per
    world (contiguous by world, global index w * shapes_per_world + i), then
    `num_global_shapes` static shapes met by every world."""

    num_worlds: int
    shapes_per_world: int
    num_global_shapes: int
    shape_type: np.ndarray  # int32 [S] SAPB_SHAPE_*
    shape_scale: np.ndarray  # [S, 3] sphere radius in [0], box half extents
    shape_X_bs: np.ndarray  # [S, 7] shape frame in its body frame (world frame if static)
    shape_body: np.ndarray  # int32 [S], -1 static
    shape_margin: np.ndarray | None = None  # [S]
    shape_collision_group: np.ndarray | None = None  # int32 [S] (sim/collision/broad_phase_common.py:133-150)


class ContactOverflowError(RuntimeError):
    """More contacts were found than the contact buffer holds."""


class ContactGenerator:
    """Owns the device buffers of contact generation for one ShapeSet and a
    model view; `generate(joint_q)` runs the forward kinematics of the
    coordinates (body poses) and the contact generation, and returns
    SapContacts views into its buffers (no host synchronisation)."""

    def __init__(self, shapes: ShapeSet, view, capacity: int, gap: float = 1.0e-3):
        self.view = view
        dev = view.device
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
        self._keep = dict(type=t(shapes.shape_type, I32), scale=t(shapes.shape_scale, F64),
                          X=t(shapes.shape_X_bs, F64), body=t(shapes.shape_body, I32),
                          margin=None if shapes.shape_margin is None else t(shapes.shape_margin, F64),
                          group=None if shapes.shape_collision_group is None
                          else t(shapes.shape_collision_group, I32))
        S = _abi.CollisionShapes()
        S.num_worlds, S.shapes_per_world, S.num_global_shapes = (shapes.num_worlds, shapes.shapes_per_world,
                                                                  shapes.num_global_shapes)
        S.shape_type, S.shape_scale = self._keep["type"].data_ptr(), self._keep["scale"].data_ptr()
        S.shape_X_bs, S.shape_body = self._keep["X"].data_ptr(), self._keep["body"].data_ptr()
        S.shape_margin = 0 if self._keep["margin"] is None else self._keep["margin"].data_ptr()
        S.gap = float(gap)
        S.shape_collision_group = 0 if self._keep["group"] is None else self._keep["group"].data_ptr()
        self.shapes = S
        lib = load()
        ws = int(lib.sapb_contacts_workspace_size(ctypes.byref(S)))
        self.workspace = torch.zeros(max(ws, 16), dtype=torch.uint8, device=dev)
        cap = int(capacity)
        z = lambda *s, dt=F64: torch.zeros(*s, dtype=dt, device=dev)
        self.count = z(1, dt=I32)
        self.shape0, self.shape1 = z(cap, dt=I32), z(cap, dt=I32)
        self.point0, self.point1, self.normal = z(cap, 3), z(cap, 3), z(cap, 3)
        self.margin0, self.margin1 = z(cap), z(cap)
        self.point0f, self.point1f, self.normalf = (z(cap, 3, dt=torch.float32), z(cap, 3, dt=torch.float32),
                                                    z(cap, 3, dt=torch.float32))
        self.margin0f, self.margin1f = z(cap, dt=torch.float32), z(cap, dt=torch.float32)
        self.body_q = z(int(view.W * view.Bw), 7)
        O = _abi.ContactOutputs()
        O.capacity, O.count = cap, self.count.data_ptr()
        O.shape0, O.shape1 = self.shape0.data_ptr(), self.shape1.data_ptr()
        O.point0, O.point1, O.normal = self.point0.data_ptr(), self.point1.data_ptr(), self.normal.data_ptr()
        O.margin0, O.margin1 = self.margin0.data_ptr(), self.margin1.data_ptr()
        self.outputs = O

    def generate(self, joint_q: torch.Tensor, *, check_capacity: bool = False) -> SapContacts:
        """Contacts at the coordinates joint_q.  The count buffer receives
        the number of contacts found, which exceeds the capacity when the
        buffer overflowed (only the first `capacity`, in pair order, are
        written; the step reads at most that many).  check_capacity=True reads
        the count back (a host synchronisation) and raises ContactOverflowError
        on overflow; otherwise call `overflowed()` when convenient."""
        lib = load()
        stream = ctypes.c_void_p(torch.cuda.current_stream(self.view.device).cuda_stream)
        q = joint_q if (joint_q.dtype == F64 and joint_q.is_contiguous()) else joint_q.to(F64).contiguous()
        check(lib.sapb_eval_fk(ctypes.byref(self.view.desc), q.data_ptr(), None, self.body_q.data_ptr(), None, stream),
              "sapb_eval_fk")
        check(lib.sapb_generate_contacts(ctypes.byref(self.shapes), self.body_q.data_ptr(), ctypes.byref(self.outputs),
                                         self.workspace.data_ptr(), self.workspace.numel(), stream),
              "sapb_generate_contacts")
        self.point0f.copy_(self.point0)
        self.point1f.copy_(self.point1)
        self.normalf.copy_(self.normal)
        self.margin0f.copy_(self.margin0)
        self.margin1f.copy_(self.margin1)
        if check_capacity and self.overflowed():
            raise ContactOverflowError(
                f"contact generation found {int(self.count.item())} contacts for {self.outputs.capacity} slots; "
                "the contacts past the capacity were dropped")
        return SapContacts(rigid_contact_count=self.count, rigid_contact_shape0=self.shape0,
                           rigid_contact_shape1=self.shape1, rigid_contact_point0=self.point0f,
                           rigid_contact_point1=self.point1f, rigid_contact_normal=self.normalf,
                           rigid_contact_margin0=self.margin0f, rigid_contact_margin1=self.margin1f,
                           rigid_contact_point0d=self.point0, rigid_contact_point1d=self.point1,
                           rigid_contact_normald=self.normal, rigid_contact_margin0d=self.margin0,
                           rigid_contact_margin1d=self.margin1)

    def found(self) -> int:
        """Contacts found by the last generate() (reads the device count)."""
        return int(self.count.item())

    def overflowed(self) -> bool:
        """Whether the last generate() found more contacts than the capacity."""
        return self.found() > int(self.outputs.capacity)
