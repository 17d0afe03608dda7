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

size_t contact_solve_smem_bytes(int n, int C, int hessian_precision);
int32_t contact_solve_occupancy(int n, int C, int hessian_precision, int variant);
int ldlt_block_widths(int n, int32_t* out, int capacity);
int32_t contact_solve_launch(const sapb_contact_problem* p, const sapb_solve_options* o, const sapb_solve_outputs* out,
                             void* workspace, size_t workspace_bytes, cudaStream_t stream);

int32_t blocked_fill_capacity(int T, int NB, int C, bool fp32);
int32_t blocked_solve_launch(const sapb_blocked_problem* p, const sapb_solve_options* o,
                             const sapb_solve_outputs* out, void* workspace, cudaStream_t stream);
int32_t dense_to_blocked_launch(const sapb_contact_problem* d, int T, int NB, double* tree_mass, double* jac,
                                int32_t* contact_tree, cudaStream_t stream);

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

size_t prepare_smem_bytes(int B, int n, int C, bool tree_blocked);
// The contact history; rank_src non-NULL: the free-motion launch's slot
// list, ranked in place and used as the slots' sources (sapb_history.cu).
int32_t history_launch(const sapb_contact_history* h, int32_t* rank_src, cudaStream_t stream);
int32_t prepare_launch(const sapb_model_desc* m, const sapb_step_inputs* in, const sapb_prepare_options* o,
                       const sapb_prepare_outputs* out, void* workspace, size_t workspace_bytes,
                       cudaStream_t stream);
int32_t integrate_launch(const sapb_model_desc* m, const double* q_in, const double* v_prev, const double* v_new,
                         const double* dt, int mode, double* q_out, cudaStream_t stream);

}  // namespace sapb
