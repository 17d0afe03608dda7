// sapb_internal.h -- declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/sapb.h"

namespace sapb {

// Dynamic shared memory a block may opt into on sm_100 (227 KB) minus the
// kernels' static shared memory.
constexpr size_t kMaxSmemPerBlock = 227 * 1024 - 1024;

void set_last_error(const char* fmt, ...);

// A world's block of joints, bodies, DOFs and articulations in the global
// model arrays: equal blocks, or the offsets of an uneven batch.
struct WorldSpan {
  int j0, nj, b0, nb, d0, nd, a0, na;
};
__host__ __device__ inline WorldSpan world_span(const sapb_model_desc& m, int e) {
  WorldSpan w;
  if (m.world_joint_start) {
    w.j0 = m.world_joint_start[e];
    w.nj = m.world_joint_start[e + 1] - w.j0;
    w.b0 = m.world_body_start[e];
    w.nb = m.world_body_start[e + 1] - w.b0;
    w.d0 = m.world_dof_start[e];
    w.nd = m.world_dof_start[e + 1] - w.d0;
    w.a0 = m.world_articulation_start[e];
    w.na = m.world_articulation_start[e + 1] - w.a0;
  } else {
    w.j0 = e * m.joints_per_world;
    w.nj = m.joints_per_world;
    w.b0 = e * m.bodies_per_world;
    w.nb = m.bodies_per_world;
    w.d0 = e * m.dofs_per_world;
    w.nd = m.dofs_per_world;
    w.a0 = e * m.articulations_per_world;
    w.na = m.articulations_per_world;
  }
  return w;
}
__host__ __device__ inline int model_joints(const sapb_model_desc& m) {
  return m.world_joint_start ? m.total_joints : m.num_worlds * m.joints_per_world;
}
__host__ __device__ inline int model_bodies(const sapb_model_desc& m) {
  return m.world_joint_start ? m.total_bodies : m.num_worlds * m.bodies_per_world;
}
__host__ __device__ inline int model_articulations(const sapb_model_desc& m) {
  return m.world_joint_start ? m.total_articulations : m.num_worlds * m.articulations_per_world;
}
// The world of body b (-1 outside the model).
__host__ __device__ inline int body_world_of(const sapb_model_desc& m, int b) {
  if (b < 0 || b >= model_bodies(m)) return -1;
  return m.body_world ? m.body_world[b] : b / m.bodies_per_world;
}

size_t contact_solve_smem_bytes(int n, int C, int hessian_precision, int threads = 128);
int32_t contact_solve_occupancy(int n, int C, int hessian_precision, int variant, int threads = 128);
int ldlt_block_widths(int n, int32_t* out, int capacity);
int32_t contact_solve_launch(const sapb_contact_problem* p, const sapb_solve_options* o, const sapb_solve_outputs* out,
                             void* workspace, size_t workspace_bytes, cudaStream_t stream);

int32_t blocked_tree_block(int tree_dofs);
int32_t blocked_fill_capacity(int T, int NB, int C, bool fp32);
int32_t blocked_solve_launch(const sapb_blocked_problem* p, const sapb_solve_options* o,
                             const sapb_solve_outputs* out, void* workspace, cudaStream_t stream);
int32_t dense_to_blocked_launch(const sapb_contact_problem* d, int T, int NB, const int32_t* tree_dof_start,
                                double* tree_mass, double* jac, int32_t* contact_tree, cudaStream_t stream);

int32_t public_to_sap_launch(const sapb_model_desc* m, const double* joint_q, const double* body_q,
                             const double* qd_pub, const double* f_pub, const double* bf_pub, double* qd_sap,
                             double* f_sap, double* bf_sap, cudaStream_t stream);
int32_t sap_to_public_launch(const sapb_model_desc* m, const double* joint_q, const double* qd_sap, double* qd_pub,
                             cudaStream_t stream);
int32_t eval_fk_launch(const sapb_model_desc* m, const double* joint_q, const double* qd_pub, double* body_q,
                       double* body_qd, cudaStream_t stream);

size_t contacts_workspace_bytes(const sapb_collision_shapes* s);
int32_t contacts_launch(const sapb_collision_shapes* s, const double* body_q, const sapb_contact_outputs* out,
                        void* workspace, cudaStream_t stream);

// tree_block: 0 for the dense layout, else the block size of the tree-blocked outputs
size_t prepare_smem_bytes(int B, int n, int C, int tree_block);
// The contact history; rank_src non-NULL: the free-motion launch's slot
// list, ranked in place and used as the slots' sources (sapb_history.cu).
int32_t history_launch(const sapb_contact_history* h, int32_t* rank_src, cudaStream_t stream);
int32_t prepare_launch(const sapb_model_desc* m, const sapb_step_inputs* in, const sapb_prepare_options* o,
                       const sapb_prepare_outputs* out, void* workspace, size_t workspace_bytes,
                       cudaStream_t stream);
int32_t integrate_launch(const sapb_model_desc* m, const double* q_in, const double* v_prev, const double* v_new,
                         const double* dt, int mode, double* q_out, cudaStream_t stream);

}  // namespace sapb
