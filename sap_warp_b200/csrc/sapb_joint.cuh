// sapb_joint.cuh -- per-joint and per-articulation pieces of the step's
// tail, shared by the separate entry points (sapb_integrate_positions,
// sapb_sap_to_public_velocity, sapb_eval_fk) and the fused tail launch
// (sapb_step_tail): the position integrators (sim/solver_sap.py:144-733),
// the SAP -> public velocity shift of free / distance joints
// (sim/sap_helpers.py:1711-1760) and the forward kinematics of public
// coordinates along an articulation (sim/sap_kinematics.py:85-229).  FP64.
#pragma once

#include <cstdint>

#include "sapb_internal.h"
#include "sapb_spatial.cuh"

namespace sapb {

// Quaternion product and transform composition as the reference's transform
// algebra (no renormalisation).
__device__ __forceinline__ Xf xf_mul(Xf a, Xf b) { return Xf{a.p + qrot(a.q, b.p), qmul(a.q, b.q)}; }
__device__ __forceinline__ Xf xf_inv(Xf x) {
  const Q4 qi = qconj(x.q);
  return Xf{-qrot(qi, x.p), qi};
}

// New coordinates of joint j (q_out) from q_in and the velocities, step h:
// sap_euler (v_new) or midpoint (the mean of v_prev and v_new); fixed joints
// write nothing.
__device__ inline void integrate_joint(const sapb_model_desc& m, int j, const double* q_in, const double* v_prev,
                                       const double* v_new, double h, int mode, double* q_out) {
  const int jt = m.joint_type[j];
  const int qs = m.joint_q_start[j], ds = m.joint_qd_start[j];
  const bool mid = mode == SAPB_INTEGRATE_MIDPOINT;
  auto vel = [&](int k) { return mid ? 0.5 * (v_prev[k] + v_new[k]) : v_new[k]; };
  if (jt == SAPB_JOINT_PRISMATIC || jt == SAPB_JOINT_REVOLUTE) {
    q_out[qs] = q_in[qs] + h * vel(ds);
    return;
  }
  if (jt == SAPB_JOINT_FIXED) return;
  if (jt == SAPB_JOINT_BALL || jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
    const int o = jt == SAPB_JOINT_BALL ? 0 : 3;
    if (o == 3)
      for (int k = 0; k < 3; ++k) q_out[qs + k] = q_in[qs + k] + h * vel(ds + 3 + k);
    const Q4 q{q_in[qs + o], q_in[qs + o + 1], q_in[qs + o + 2], q_in[qs + o + 3]};
    const V3 w = v3(vel(ds), vel(ds + 1), vel(ds + 2));
    Q4 qn = q;
    if (!mid) {
      // qdot = 0.5 [0, w] q (sim/solver_sap.py:158-178)
      const double hd = 0.5 * h;
      qn = Q4{q.x + hd * (q.w * w.x + w.y * q.z - w.z * q.y), q.y + hd * (q.w * w.y + w.z * q.x - w.x * q.z),
              q.z + hd * (q.w * w.z + w.x * q.y - w.y * q.x), q.w - hd * (w.x * q.x + w.y * q.y + w.z * q.z)};
      const double nn = sqrt(qn.x * qn.x + qn.y * qn.y + qn.z * qn.z + qn.w * qn.w);
      if (nn > 0.0) qn = Q4{qn.x / nn, qn.y / nn, qn.z / nn, qn.w / nn};
    } else {
      // exp map of the midpoint angular velocity (sim/solver_sap.py:243-262)
      const double wn = sqrt(dot(w, w));
      const double angle = wn * h;
      if (angle > 1.0e-12) {
        const V3 axis = (1.0 / wn) * w;
        const Q4 r = qaxis_angle(axis, angle);
        qn = qmul(r, q);
        const double nn = sqrt(qn.x * qn.x + qn.y * qn.y + qn.z * qn.z + qn.w * qn.w);
        if (nn > 0.0) qn = Q4{qn.x / nn, qn.y / nn, qn.z / nn, qn.w / nn};
      }
    }
    q_out[qs + o] = qn.x;
    q_out[qs + o + 1] = qn.y;
    q_out[qs + o + 2] = qn.z;
    q_out[qs + o + 3] = qn.w;
    return;
  }
  // D6 and other multi-axis scalar joints: q += h * qd per axis
  const int dim = m.joint_dof_dim[2 * j] + m.joint_dof_dim[2 * j + 1];
  for (int k = 0; k < dim; ++k) q_out[qs + k] = q_in[qs + k] + h * vel(ds + k);
}

// Public velocities of joint j at coordinates joint_q (free / distance: [v_com; w]
// from SAP's [w; v_origin]; other joints copy).
__device__ inline void public_velocity_joint(const sapb_model_desc& m, int j, const double* joint_q,
                                             const double* qd_sap, double* qd_pub) {
  const int jt = m.joint_type[j];
  const int ds = m.joint_qd_start[j];
  const int dim = m.joint_dof_dim[2 * j] + m.joint_dof_dim[2 * j + 1];
  if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
    const int qs = m.joint_q_start[j];
    const int child = m.joint_child[j];
    const Q4 q{joint_q[qs + 3], joint_q[qs + 4], joint_q[qs + 5], joint_q[qs + 6]};
    const V3 r = qrot(q, load3(m.body_com + 3 * (size_t)child));
    const V3 w = load3(qd_sap + ds), v_o = load3(qd_sap + ds + 3);
    store3(qd_pub + ds, v_o + cross(w, r));
    store3(qd_pub + ds + 3, w);
  } else {
    for (int a = 0; a < dim; ++a) qd_pub[ds + a] = qd_sap[ds + a];
  }
}

// Body poses and public body velocities [v; w] of articulation a, joint by
// joint (its joints are ordered parents first).
__device__ inline void fk_articulation(const sapb_model_desc& m, int a, int num_bodies, const double* joint_q,
                                       const double* qd_pub, double* body_q, double* body_qd) {
  const int j0 = m.articulation_start[a], j1 = m.articulation_start[a + 1];
  for (int i = j0; i < j1; ++i) {
    const int parent = m.joint_parent[i], child = m.joint_child[i];
    if (child < 0 || child >= num_bodies) continue;
    const int jt = m.joint_type[i];
    const Xf X_pj = xf_load(m.joint_X_p + 7 * (size_t)i);
    const Xf X_cj = xf_load(m.joint_X_c + 7 * (size_t)i);
    Xf X_wpj = X_pj;
    V3 v_wpj = v3(0, 0, 0), w_wpj = v3(0, 0, 0);
    if (parent >= 0 && parent < num_bodies) {
      const Xf X_wp = xf_load(body_q + 7 * (size_t)parent);
      X_wpj = xf_mul(X_wp, X_pj);
      const V3 com_w = X_wp.p + qrot(X_wp.q, load3(m.body_com + 3 * (size_t)parent));
      const V3 r_p = X_wpj.p - com_w;
      if (body_qd) {
        const V3 w_p = load3(body_qd + 6 * (size_t)parent + 3);
        v_wpj = load3(body_qd + 6 * (size_t)parent) + cross(w_p, r_p);
        w_wpj = w_p;
      }
    }
    const int qs = m.joint_q_start[i], ds = m.joint_qd_start[i];
    Xf X_j{v3(0, 0, 0), qident()};
    V3 vj = v3(0, 0, 0), wj = v3(0, 0, 0);
    auto qd = [&](int k) { return qd_pub ? qd_pub[k] : 0.0; };
    if (jt == SAPB_JOINT_PRISMATIC) {
      const V3 ax = load3(m.joint_axis + 3 * (size_t)ds);
      X_j.p = joint_q[qs] * ax;
      vj = qd(ds) * ax;
    } else if (jt == SAPB_JOINT_REVOLUTE) {
      const V3 ax = load3(m.joint_axis + 3 * (size_t)ds);
      X_j.q = qaxis_angle(ax, joint_q[qs]);
      wj = qd(ds) * ax;
    } else if (jt == SAPB_JOINT_BALL) {
      X_j.q = Q4{joint_q[qs], joint_q[qs + 1], joint_q[qs + 2], joint_q[qs + 3]};
      wj = v3(qd(ds), qd(ds + 1), qd(ds + 2));
    } else if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
      X_j = Xf{v3(joint_q[qs], joint_q[qs + 1], joint_q[qs + 2]),
               Q4{joint_q[qs + 3], joint_q[qs + 4], joint_q[qs + 5], joint_q[qs + 6]}};
      vj = v3(qd(ds), qd(ds + 1), qd(ds + 2));
      wj = v3(qd(ds + 3), qd(ds + 4), qd(ds + 5));
    } else if (jt == SAPB_JOINT_D6) {  // sim/sap_kinematics.py:170-215
      const int lin = m.joint_dof_dim[2 * i], ang = m.joint_dof_dim[2 * i + 1];
      V3 ax[3];
      d6_mobilizer(m.joint_axis + 3 * (size_t)ds, joint_q + qs, lin, ang, &X_j, ax);
      for (int k = 0; k < lin && k < 3; ++k) vj = vj + qd(ds + k) * load3(m.joint_axis + 3 * (size_t)(ds + k));
      for (int k = 0; k < ang && k < 3; ++k) wj = wj + qd(ds + lin + k) * ax[k];
    }
    const Xf X_wc = xf_mul(xf_mul(X_wpj, X_j), xf_inv(X_cj));
    const V3 lin = v_wpj + qrot(X_wpj.q, vj), ang = w_wpj + qrot(X_wpj.q, wj);
    double* bq = body_q + 7 * (size_t)child;
    store3(bq, X_wc.p);
    bq[3] = X_wc.q.x;
    bq[4] = X_wc.q.y;
    bq[5] = X_wc.q.z;
    bq[6] = X_wc.q.w;
    if (body_qd) {
      store3(body_qd + 6 * (size_t)child, lin);
      store3(body_qd + 6 * (size_t)child + 3, ang);
    }
  }
}

}  // namespace sapb
