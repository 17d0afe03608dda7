"""Foreign device arrays (the way Warp / Newton hand theirs over: DLPack or
the CUDA array interface) wrapped zero-copy by runtime.sap_state_from_newton
/ sap_control_from_newton / sap_contacts_from_newton and stepped by
SolverSAP: the step reads the caller's memory and writes its results there,
bit for bit the step on torch tensors with the same values."""

import pytest
import torch

from sap_warp_b200 import models
from sap_warp_b200.runtime import (SapControl, SapState, sap_contacts_from_newton, sap_control_from_newton,
                                   sap_state_from_newton)
from sap_warp_b200.solver import SolverSAP

pytestmark = pytest.mark.gpu


class _DLPack:
    """A device array that exposes only the DLPack protocol."""

    def __init__(self, t):
        self.t = t

    def __dlpack__(self, *args, **kwargs):
        return self.t.__dlpack__(*args, **kwargs)

    def __dlpack_device__(self):
        return self.t.__dlpack_device__()


class _CAI:
    """A device array that exposes only the CUDA array interface."""

    def __init__(self, t):
        self.t = t

    @property
    def __cuda_array_interface__(self):
        return self.t.__cuda_array_interface__


class _Obj:
    def __init__(self, **kw):
        self.__dict__.update(kw)


@pytest.mark.parametrize("wrap", [_DLPack, _CAI])
def test_foreign_arrays_step_in_place(cuda_device, wrap):
    W = 32
    model, state, control, con, _ = models.rollout_scene("humanoid", W, 7, cuda_device)
    D, B = int(model.joint_dof_count), int(model.body_count)
    g = torch.Generator(device="cpu").manual_seed(4)
    qd_pub = (0.3 * torch.randn(D, generator=g, dtype=torch.float64)).to(cuda_device)
    f_pub = (0.5 * torch.randn(D, generator=g, dtype=torch.float64)).to(cuda_device)
    zeros = lambda *s: torch.zeros(*s, dtype=torch.float64, device=cuda_device)
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake", hessian_precision="fp32",
              warm_start="previous_impulses")
    # the step on torch tensors (public orders), twice, for the warm start
    ref_in = SapState(joint_q=state.joint_q.clone(), joint_qd=qd_pub.clone(), body_q=zeros(B, 7),
                      body_qd=zeros(B, 6), joint_qd_order="public")
    ref_out = SapState(joint_q=zeros(*state.joint_q.shape), joint_qd=zeros(D), body_q=zeros(B, 7),
                       body_qd=zeros(B, 6), joint_qd_order="public")
    ref_ctl = SapControl(joint_f=f_pub.clone(), joint_f_order="public")
    solver = SolverSAP(model, **kw)
    solver.step(ref_in, ref_out, ref_ctl, con, 2e-3)
    solver.step(ref_out, ref_in, ref_ctl, con, 2e-3)
    # the same on foreign arrays the caller owns
    mem_in = dict(joint_q=state.joint_q.clone(), joint_qd=qd_pub.clone(), body_q=zeros(B, 7), body_qd=zeros(B, 6))
    mem_out = dict(joint_q=zeros(*state.joint_q.shape), joint_qd=zeros(D), body_q=zeros(B, 7), body_qd=zeros(B, 6))
    n_in = _Obj(**{k: wrap(v) for k, v in mem_in.items()}, body_f=None)
    n_out = _Obj(**{k: wrap(v) for k, v in mem_out.items()}, body_f=None)
    st_in, st_out = sap_state_from_newton(n_in), sap_state_from_newton(n_out)
    assert st_in.joint_q.data_ptr() == mem_in["joint_q"].data_ptr()  # zero-copy views
    assert st_out.body_qd.data_ptr() == mem_out["body_qd"].data_ptr()
    ctl = sap_control_from_newton(_Obj(joint_f=wrap(f_pub.clone())))
    names = [k for k in vars(con) if isinstance(getattr(con, k), torch.Tensor)]
    n_con = _Obj(**{k: wrap(getattr(con, k).clone()) for k in names})
    contacts = sap_contacts_from_newton(n_con)
    assert contacts.rigid_contact_count.data_ptr() == n_con.rigid_contact_count.t.data_ptr()
    solver = SolverSAP(model, **kw)
    solver.step(st_in, st_out, ctl, contacts, 2e-3)
    solver.step(st_out, st_in, ctl, contacts, 2e-3)
    torch.cuda.synchronize()
    for k in ("joint_q", "joint_qd", "body_q", "body_qd"):
        assert torch.equal(mem_in[k], getattr(ref_in, k)), k  # written in the caller's memory
        assert torch.equal(mem_out[k], getattr(ref_out, k)), k
