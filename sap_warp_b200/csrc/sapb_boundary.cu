// sapb_boundary.cu -- the public-order boundary of the step: conversions
// between the public joint / body orders of Newton-style callers and the SAP
// order the step runs in, and the forward kinematics of the public output.
//
//  - public -> SAP (sim/sap_helpers.py:1481-1622, 1811-1925, 2058-2095;
//    driven by SolverSAP._prepare_step_boundary, sim/solver_sap.py:1198-1261):
//    free / distance joints carry [v_com; w] publicly and [w; v_origin] in
//    SAP order, v_origin = v_com - w x r_com with r_com the body's COM offset
//    rotated by the joint's own quaternion; joint forces [f; tau_com] become
//    [tau_com + r_com x f; f]; body forces [f; tau_com] (at the COM) become
//    the negated body-origin wrench [-(tau_com + c x f); -f] (the inverse
//    dynamics residual stores -F_applied), c the COM offset rotated by the
//    body pose.  Other joints copy.
//  - SAP -> public velocities (sim/sap_helpers.py:1711-1760): the inverse
//    shift with the output pose, v_com = v_origin + w x r_com.
//  - forward kinematics of public coordinates (sim/sap_kinematics.py:85-229):
//    body poses and public body velocities [v; w] joint by joint along each
//    articulation.
// Thread per joint / body for the conversions, thread per articulation for
// the forward kinematics (its joints are ordered parents first).  FP64.
#include <cuda_runtime.h>

#include <cstdint>

#include "sapb_internal.h"
#include "sapb_spatial.cuh"

namespace sapb {

namespace {

struct BoundaryParams {
  sapb_model_desc m;
  int32_t num_joints, num_bodies, num_articulations;
};

// Quaternion product and transform composition as the reference's transform
// algebra (no renormalisation).
__device__ __forceinline__ Xf xf_mul(Xf a, Xf b) { return Xf{a.p + qrot(a.q, b.p), qmul(a.q, b.q)}; }
__device__ __forceinline__ Xf xf_inv(Xf x) {
  const Q4 qi = qconj(x.q);
  return Xf{-qrot(qi, x.p), qi};
}

__global__ void public_to_sap_kernel(const BoundaryParams P, const double* joint_q, const double* body_q,
                                     const double* qd_pub, const double* f_pub, const double* bf_pub,
                                     double* qd_sap, double* f_sap, double* bf_sap) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < P.num_joints) {
    const int j = t;
    const int jt = P.m.joint_type[j];
    const int ds = P.m.joint_qd_start[j];
    const int dim = P.m.joint_dof_dim[2 * j] + P.m.joint_dof_dim[2 * j + 1];
    if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
      const int qs = P.m.joint_q_start[j];
      const int child = P.m.joint_child[j];
      const Q4 q{joint_q[qs + 3], joint_q[qs + 4], joint_q[qs + 5], joint_q[qs + 6]};
      const V3 r = qrot(q, load3(P.m.body_com + 3 * (size_t)child));
      if (qd_pub) {
        const V3 v_com = load3(qd_pub + ds), w = load3(qd_pub + ds + 3);
        store3(qd_sap + ds, w);
        store3(qd_sap + ds + 3, v_com - cross(w, r));
      }
      if (f_pub) {
        const V3 f = load3(f_pub + ds), tau = load3(f_pub + ds + 3);
        store3(f_sap + ds, tau + cross(r, f));
        store3(f_sap + ds + 3, f);
      }
    } else {
      for (int a = 0; a < dim; ++a) {
        if (qd_pub) qd_sap[ds + a] = qd_pub[ds + a];
        if (f_pub) f_sap[ds + a] = f_pub[ds + a];
      }
    }
  }
  if (bf_pub && t < P.num_bodies) {
    const int b = t;
    const V3 f = load3(bf_pub + 6 * (size_t)b), tau = load3(bf_pub + 6 * (size_t)b + 3);
    const Q4 q{body_q[7 * (size_t)b + 3], body_q[7 * (size_t)b + 4], body_q[7 * (size_t)b + 5],
               body_q[7 * (size_t)b + 6]};
    const V3 c = qrot(q, load3(P.m.body_com + 3 * (size_t)b));
    store3(bf_sap + 6 * (size_t)b, -(tau + cross(c, f)));
    store3(bf_sap + 6 * (size_t)b + 3, -f);
  }
}

__global__ void sap_to_public_velocity_kernel(const BoundaryParams P, const double* joint_q, const double* qd_sap,
                                              double* qd_pub) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= P.num_joints) return;
  const int jt = P.m.joint_type[j];
  const int ds = P.m.joint_qd_start[j];
  const int dim = P.m.joint_dof_dim[2 * j] + P.m.joint_dof_dim[2 * j + 1];
  if (jt == SAPB_JOINT_FREE || jt == SAPB_JOINT_DISTANCE) {
    const int qs = P.m.joint_q_start[j];
    const int child = P.m.joint_child[j];
    const Q4 q{joint_q[qs + 3], joint_q[qs + 4], joint_q[qs + 5], joint_q[qs + 6]};
    const V3 r = qrot(q, load3(P.m.body_com + 3 * (size_t)child));
    const V3 w = load3(qd_sap + ds), v_o = load3(qd_sap + ds + 3);
    store3(qd_pub + ds, v_o + cross(w, r));
    store3(qd_pub + ds + 3, w);
  } else {
    for (int a = 0; a < dim; ++a) qd_pub[ds + a] = qd_sap[ds + a];
  }
}

__global__ void eval_fk_kernel(const BoundaryParams P, const double* joint_q, const double* qd_pub, double* body_q,
                               double* body_qd) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.num_articulations) return;
  const int j0 = P.m.articulation_start[a], j1 = P.m.articulation_start[a + 1];
  for (int i = j0; i < j1; ++i) {
    const int parent = P.m.joint_parent[i], child = P.m.joint_child[i];
    if (child < 0 || child >= P.num_bodies) continue;
    const int jt = P.m.joint_type[i];
    const Xf X_pj = xf_load(P.m.joint_X_p + 7 * (size_t)i);
    const Xf X_cj = xf_load(P.m.joint_X_c + 7 * (size_t)i);
    Xf X_wpj = X_pj;
    V3 v_wpj = v3(0, 0, 0), w_wpj = v3(0, 0, 0);
    if (parent >= 0 && parent < P.num_bodies) {
      const Xf X_wp = xf_load(body_q + 7 * (size_t)parent);
      X_wpj = xf_mul(X_wp, X_pj);
      const V3 com_w = X_wp.p + qrot(X_wp.q, load3(P.m.body_com + 3 * (size_t)parent));
      const V3 r_p = X_wpj.p - com_w;
      if (body_qd) {
        const V3 w_p = load3(body_qd + 6 * (size_t)parent + 3);
        v_wpj = load3(body_qd + 6 * (size_t)parent) + cross(w_p, r_p);
        w_wpj = w_p;
      }
    }
    const int qs = P.m.joint_q_start[i], ds = P.m.joint_qd_start[i];
    Xf X_j{v3(0, 0, 0), qident()};
    V3 vj = v3(0, 0, 0), wj = v3(0, 0, 0);
    auto qd = [&](int k) { return qd_pub ? qd_pub[k] : 0.0; };
    if (jt == SAPB_JOINT_PRISMATIC) {
      const V3 ax = load3(P.m.joint_axis + 3 * (size_t)ds);
      X_j.p = joint_q[qs] * ax;
      vj = qd(ds) * ax;
    } else if (jt == SAPB_JOINT_REVOLUTE) {
      const V3 ax = load3(P.m.joint_axis + 3 * (size_t)ds);
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
      const int lin = P.m.joint_dof_dim[2 * i], ang = P.m.joint_dof_dim[2 * i + 1];
      V3 ax[3];
      d6_mobilizer(P.m.joint_axis + 3 * (size_t)ds, joint_q + qs, lin, ang, &X_j, ax);
      for (int k = 0; k < lin && k < 3; ++k) vj = vj + qd(ds + k) * load3(P.m.joint_axis + 3 * (size_t)(ds + k));
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

BoundaryParams make_params(const sapb_model_desc* m) {
  BoundaryParams P;
  P.m = *m;
  P.num_joints = m->num_worlds * m->joints_per_world;
  P.num_bodies = m->num_worlds * m->bodies_per_world;
  P.num_articulations = m->num_worlds * m->articulations_per_world;
  return P;
}

int32_t finish(const char* where) {
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_last_error("%s: %s", where, cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

}  // namespace

int32_t public_to_sap_launch(const sapb_model_desc* m, const double* joint_q, const double* body_q,
                             const double* qd_pub, const double* f_pub, const double* bf_pub, double* qd_sap,
                             double* f_sap, double* bf_sap, cudaStream_t stream) {
  const BoundaryParams P = make_params(m);
  const int n = P.num_joints > P.num_bodies ? P.num_joints : P.num_bodies;
  if (n == 0) return SAPB_OK;
  public_to_sap_kernel<<<(n + 127) / 128, 128, 0, stream>>>(P, joint_q, body_q, qd_pub, f_pub, bf_pub, qd_sap,
                                                             f_sap, bf_sap);
  return finish("public to SAP conversion");
}

int32_t sap_to_public_launch(const sapb_model_desc* m, const double* joint_q, const double* qd_sap, double* qd_pub,
                             cudaStream_t stream) {
  const BoundaryParams P = make_params(m);
  if (P.num_joints == 0) return SAPB_OK;
  sap_to_public_velocity_kernel<<<(P.num_joints + 127) / 128, 128, 0, stream>>>(P, joint_q, qd_sap, qd_pub);
  return finish("SAP to public conversion");
}

int32_t eval_fk_launch(const sapb_model_desc* m, const double* joint_q, const double* qd_pub, double* body_q,
                       double* body_qd, cudaStream_t stream) {
  const BoundaryParams P = make_params(m);
  if (P.num_articulations == 0) return SAPB_OK;
  eval_fk_kernel<<<(P.num_articulations + 127) / 128, 128, 0, stream>>>(P, joint_q, qd_pub, body_q, body_qd);
  return finish("forward kinematics");
}

}  // namespace sapb
