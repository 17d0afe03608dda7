"""The public-order boundary on the GPU (sapb_public_to_sap,
sapb_sap_to_public_velocity, sapb_eval_fk through the C ABI) against the
numpy restatement of the reference's kernels, and a SolverSAP step with
public-order input and output against the SAP-order step."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import boundary as ob
from sap_warp_b200 import models
from sap_warp_b200._lib import check, load
from sap_warp_b200.runtime import SapControl, SapState
from sap_warp_b200.solver import SolverSAP, _ModelView

pytestmark = pytest.mark.gpu


def _case(kind, seed, worlds=4):
    rng = np.random.default_rng(seed)
    tpl = models.world_template(kind, rng, random_child_frames=True)
    g = models.replicate(tpl, worlds, rng)
    q = models.random_joint_q(tpl, rng, worlds).reshape(-1)
    return rng, tpl, g, q


def _t(a, dev):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)


@pytest.mark.parametrize("kind", ["humanoid", "arm_box", "slider", "quadruped", "joints"])
def test_conversions_and_fk_match_oracle(cuda_device, kind):
    rng, tpl, g, q = _case(kind, 11)
    model = models.to_model(tpl, g, q.reshape(4, -1), cuda_device)
    view = _ModelView(model)
    D, B = g["counts"]["dofs"], g["counts"]["bodies"]
    qd, f = rng.normal(size=D), rng.normal(size=D)
    bq_ref, bqd_ref = ob.eval_fk(g, q, qd)
    bf = rng.normal(size=(B, 6))
    sap_ref, fs_ref, bfs_ref = ob.public_to_sap(g, q, body_q=bq_ref, qd_pub=qd, f_pub=f, bf_pub=bf)
    lib, s = load(), ctypes.c_void_p(torch.cuda.current_stream(cuda_device).cuda_stream)
    tq, tqd, tf, tbf, tbq = _t(q, cuda_device), _t(qd, cuda_device), _t(f, cuda_device), _t(bf, cuda_device), \
        _t(bq_ref, cuda_device)
    out_v, out_f, out_bf = (torch.zeros(D, dtype=torch.float64, device=cuda_device),
                            torch.zeros(D, dtype=torch.float64, device=cuda_device),
                            torch.zeros(B, 6, dtype=torch.float64, device=cuda_device))
    d = ctypes.byref(view.desc)
    check(lib.sapb_public_to_sap(d, tq.data_ptr(), tbq.data_ptr(), tqd.data_ptr(), tf.data_ptr(), tbf.data_ptr(),
                                 out_v.data_ptr(), out_f.data_ptr(), out_bf.data_ptr(), s), "public_to_sap")
    back = torch.zeros(D, dtype=torch.float64, device=cuda_device)
    check(lib.sapb_sap_to_public_velocity(d, tq.data_ptr(), out_v.data_ptr(), back.data_ptr(), s), "sap_to_public")
    bq = torch.zeros(B, 7, dtype=torch.float64, device=cuda_device)
    bqd = torch.zeros(B, 6, dtype=torch.float64, device=cuda_device)
    check(lib.sapb_eval_fk(d, tq.data_ptr(), tqd.data_ptr(), bq.data_ptr(), bqd.data_ptr(), s), "eval_fk")
    torch.cuda.synchronize()
    np.testing.assert_allclose(out_v.cpu().numpy(), sap_ref, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(out_f.cpu().numpy(), fs_ref, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(out_bf.cpu().numpy(), bfs_ref, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(back.cpu().numpy(), qd, rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(bq.cpu().numpy(), bq_ref, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(bqd.cpu().numpy(), bqd_ref, rtol=1e-12, atol=1e-12)


def test_public_order_step_matches_sap_order_step(cuda_device):
    """A humanoid batch stepped with public-order state, forces and body
    forces equals the SAP-order step on the converted inputs; the public
    output holds the converted velocities and the forward kinematics of the
    new coordinates."""
    W = 16
    model, state, control, con, _ = models.rollout_scene("humanoid", W, 5, cuda_device)
    rng = np.random.default_rng(3)
    tpl = None
    g = {k: getattr(model, k).cpu().numpy() for k in ("joint_type", "joint_q_start", "joint_qd_start",
                                                        "joint_child", "joint_parent", "joint_X_p", "joint_X_c",
                                                        "joint_axis", "articulation_start", "body_mass")}
    g["joint_dof_dim"] = model.joint_dof_dim.cpu().numpy().reshape(-1, 2)
    g["body_com"] = model.body_com.cpu().numpy().reshape(-1, 3)
    g["joint_X_p"] = g["joint_X_p"].reshape(-1, 7)
    g["joint_X_c"] = g["joint_X_c"].reshape(-1, 7)
    g["joint_axis"] = g["joint_axis"].reshape(-1, 3)
    del tpl
    q = state.joint_q.cpu().numpy()
    D, B = int(model.joint_dof_count), int(model.body_count)
    qd_pub = rng.normal(scale=0.3, size=D)
    f_pub = rng.normal(scale=0.5, size=D)
    bq0, _ = ob.eval_fk(g, q, qd_pub)
    bf_pub = rng.normal(scale=0.5, size=(B, 6))
    qd_sap, f_sap, bf_sap = ob.public_to_sap(g, q, body_q=bq0, qd_pub=qd_pub, f_pub=f_pub, bf_pub=bf_pub)
    dev = cuda_device
    kw = dict(max_rigid_contact=32, contact_preset_variant="drake")
    sap_in = SapState(joint_q=state.joint_q.clone(), joint_qd=_t(qd_sap, dev), body_q=_t(bq0, dev),
                      body_f=_t(bf_sap, dev))
    sap_out = SapState(joint_q=torch.zeros_like(state.joint_q), joint_qd=torch.zeros(D, dtype=torch.float64,
                                                                                     device=dev),
                       body_q=torch.zeros(B, 7, dtype=torch.float64, device=dev),
                       body_f=torch.zeros(B, 6, dtype=torch.float64, device=dev))
    SolverSAP(model, **kw).step(sap_in, sap_out, SapControl(joint_f=_t(f_sap, dev)), con, 2e-3)
    pub_in = SapState(joint_q=state.joint_q.clone(), joint_qd=_t(qd_pub, dev), body_q=_t(bq0, dev),
                      body_f=_t(bf_pub, dev), joint_qd_order="public", body_f_order="public")
    pub_out = SapState(joint_q=torch.zeros_like(state.joint_q), joint_qd=torch.zeros(D, dtype=torch.float64,
                                                                                     device=dev),
                       body_q=torch.zeros(B, 7, dtype=torch.float64, device=dev),
                       body_qd=torch.zeros(B, 6, dtype=torch.float64, device=dev), joint_qd_order="public")
    SolverSAP(model, **kw).step(pub_in, pub_out, SapControl(joint_f=_t(f_pub, dev), joint_f_order="public"), con,
                                2e-3)
    torch.cuda.synchronize()
    q_out = sap_out.joint_q.cpu().numpy()
    np.testing.assert_allclose(pub_out.joint_q.cpu().numpy(), q_out, rtol=0, atol=1e-12)
    v_pub_ref = ob.sap_to_public_velocity(g, q_out, sap_out.joint_qd.cpu().numpy())
    np.testing.assert_allclose(pub_out.joint_qd.cpu().numpy(), v_pub_ref, rtol=1e-10, atol=1e-10)
    bq_ref, bqd_ref = ob.eval_fk(g, q_out, v_pub_ref)
    np.testing.assert_allclose(pub_out.body_q.cpu().numpy(), bq_ref, rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(pub_out.body_qd.cpu().numpy(), bqd_ref, rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("kind", ["humanoid", "joints", "arm_box"])
@pytest.mark.parametrize("mode", [0, 1])
def test_fused_tail_equals_the_separate_launches(cuda_device, kind, mode):
    """sapb_step_tail_launch (integration, velocities in SAP or public order,
    forward kinematics of the new pose, one CTA per world) writes the same
    bits as sapb_integrate_positions after a copy of the coordinates, then
    sapb_sap_to_public_velocity and sapb_eval_fk."""
    from sap_warp_b200 import _abi

    rng, tpl, g, q = _case(kind, 17)
    model = models.to_model(tpl, g, q.reshape(4, -1), cuda_device)
    view = _ModelView(model)
    D, B = g["counts"]["dofs"], g["counts"]["bodies"]
    dev = cuda_device
    tq, v0, v1 = _t(q, dev), _t(rng.normal(size=D), dev), _t(rng.normal(size=D), dev)
    dt = torch.full((4,), 2.0e-3, dtype=torch.float64, device=dev)
    lib, s = load(), ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    d = ctypes.byref(view.desc)
    # separate launches
    q_sep = tq.clone()
    check(lib.sapb_integrate_positions(d, tq.data_ptr(), v0.data_ptr(), v1.data_ptr(), dt.data_ptr(), mode,
                                       q_sep.data_ptr(), s), "integrate")
    qd_pub = torch.zeros(D, dtype=torch.float64, device=dev)
    check(lib.sapb_sap_to_public_velocity(d, q_sep.data_ptr(), v1.data_ptr(), qd_pub.data_ptr(), s), "public")
    bq_sep = torch.zeros(B, 7, dtype=torch.float64, device=dev)
    bqd_sep = torch.zeros(B, 6, dtype=torch.float64, device=dev)
    check(lib.sapb_eval_fk(d, q_sep.data_ptr(), qd_pub.data_ptr(), bq_sep.data_ptr(), bqd_sep.data_ptr(), s), "fk")
    for public in (0, 1):
        q_out = torch.full_like(tq, float("nan"))
        qd_out = torch.full_like(v1, float("nan"))
        bq = torch.full((B, 7), float("nan"), dtype=torch.float64, device=dev)
        bqd = torch.full((B, 6), float("nan"), dtype=torch.float64, device=dev)
        T = _abi.StepTail()
        T.joint_q_in, T.v_prev, T.v_new, T.dt = tq.data_ptr(), v0.data_ptr(), v1.data_ptr(), dt.data_ptr()
        T.mode, T.qd_public = mode, public
        T.joint_q_out, T.joint_qd_out = q_out.data_ptr(), qd_out.data_ptr()
        T.body_q_out = bq.data_ptr()
        T.body_qd_out = bqd.data_ptr() if public else None
        check(lib.sapb_step_tail_launch(d, ctypes.byref(T), s), "sapb_step_tail_launch")
        torch.cuda.synchronize()
        assert torch.equal(q_out, q_sep)
        assert torch.equal(qd_out, qd_pub if public else v1)
        if public:
            assert torch.equal(bq, bq_sep) and torch.equal(bqd, bqd_sep)
        else:
            assert torch.equal(bq, bq_sep)  # poses do not depend on the velocities
    # aliasing the input coordinates is refused
    T.joint_q_out = tq.data_ptr()
    assert lib.sapb_step_tail_launch(d, ctypes.byref(T), s) == _abi.SAPB_ERR_INVALID_ARGUMENT
