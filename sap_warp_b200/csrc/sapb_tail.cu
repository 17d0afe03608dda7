// sapb_tail.cu -- the step's tail in one launch: per world (one CTA), the
// threads take the world's joints for the new coordinates and velocities
// (the integrators of sim/solver_sap.py:144-733; the public velocity shift
// of sim/sap_helpers.py:1711-1760 at the new coordinates), then, after the
// block's barrier, one thread per articulation runs the forward kinematics
// of the new public coordinates (sim/sap_kinematics.py:85-229).  The
// arithmetic is the separate entry points' (sapb_joint.cuh), so the fused
// launch writes the same bits.
#include <cuda_runtime.h>

#include <cstdint>

#include "sapb_internal.h"
#include "sapb_joint.cuh"

namespace sapb {
namespace {

__global__ void step_tail_kernel(const sapb_model_desc m, const sapb_step_tail T) {
  const int e = blockIdx.x;
  const WorldSpan ws = world_span(m, e);
  const double h = T.dt[e];
  // the solve's velocities by global DOF index: its slots of dofs_per_world
  // per world (an offset of zero when the blocks are equal)
  const double* v_new = T.v_new + ((long long)e * m.dofs_per_world - ws.d0);
  for (int jl = threadIdx.x; jl < ws.nj; jl += blockDim.x) {
    const int j = ws.j0 + jl;
    if (m.joint_type[j] == SAPB_JOINT_FIXED) {
      for (int k = m.joint_q_start[j]; k < m.joint_q_start[j + 1]; ++k) T.joint_q_out[k] = T.joint_q_in[k];
    } else {
      integrate_joint(m, j, T.joint_q_in, T.v_prev, v_new, h, T.mode, T.joint_q_out);
    }
    if (T.joint_qd_out) {
      if (T.qd_public) {
        public_velocity_joint(m, j, T.joint_q_out, v_new, T.joint_qd_out);
      } else {
        const int ds = m.joint_qd_start[j];
        const int dim = m.joint_dof_dim[2 * j] + m.joint_dof_dim[2 * j + 1];
        for (int k = 0; k < dim; ++k) T.joint_qd_out[ds + k] = v_new[ds + k];
      }
    }
  }
  if (!T.body_q_out) return;  // uniform over the block
  __syncthreads();            // this world's new coordinates and velocities
  for (int al = threadIdx.x; al < ws.na; al += blockDim.x)
    fk_articulation(m, ws.a0 + al, model_bodies(m), T.joint_q_out,
                    T.qd_public ? T.joint_qd_out : nullptr, T.body_q_out, T.body_qd_out);
}

}  // namespace
}  // namespace sapb

using namespace sapb;

extern "C" int32_t sapb_step_tail_launch(const sapb_model_desc* m, const sapb_step_tail* t, void* stream) {
  if (!m || !t || m->num_worlds < 0 || m->joints_per_world < 0 || !t->joint_q_in || !t->v_new || !t->dt ||
      !t->joint_q_out || t->joint_q_out == t->joint_q_in || (t->mode == SAPB_INTEGRATE_MIDPOINT && !t->v_prev) ||
      (t->mode != SAPB_INTEGRATE_SAP_EULER && t->mode != SAPB_INTEGRATE_MIDPOINT) ||
      (t->body_qd_out && (!t->body_q_out || !t->qd_public || !t->joint_qd_out)) || !m->joint_type ||
      !m->joint_q_start || !m->joint_qd_start || !m->joint_dof_dim ||
      (t->body_q_out && (!m->articulation_start || !m->joint_parent || !m->joint_child || !m->joint_X_p ||
                         !m->joint_X_c || !m->body_com))) {
    set_last_error("sapb_step_tail_launch: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (m->num_worlds == 0 || m->joints_per_world == 0) return SAPB_OK;
  int threads = m->joints_per_world > m->articulations_per_world ? m->joints_per_world : m->articulations_per_world;
  threads = (threads + 31) / 32 * 32;
  if (threads > 256) threads = 256;
  step_tail_kernel<<<m->num_worlds, threads, 0, static_cast<cudaStream_t>(stream)>>>(*m, *t);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_last_error("sapb_step_tail_launch: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}
