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
#include "sapb_joint.cuh"
#include "sapb_spatial.cuh"

namespace sapb {

namespace {

struct BoundaryParams {
  sapb_model_desc m;
  int32_t num_joints, num_bodies, num_articulations;
};

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
  public_velocity_joint(P.m, j, joint_q, qd_sap, qd_pub);
}

__global__ void eval_fk_kernel(const BoundaryParams P, const double* joint_q, const double* qd_pub, double* body_q,
                               double* body_qd) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= P.num_articulations) return;
  fk_articulation(P.m, a, P.num_bodies, joint_q, qd_pub, body_q, body_qd);
}

BoundaryParams make_params(const sapb_model_desc* m) {
  BoundaryParams P;
  P.m = *m;
  P.num_joints = model_joints(*m);
  P.num_bodies = model_bodies(*m);
  P.num_articulations = model_articulations(*m);
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
