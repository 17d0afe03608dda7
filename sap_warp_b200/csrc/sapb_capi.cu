// sapb_capi.cu -- the extern "C" entry points declared in include/sapb.h.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "sapb_internal.h"

namespace sapb {

static thread_local char g_last_error[512] = {0};

void set_last_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

}  // namespace sapb

extern "C" {

int32_t sapb_abi_version(void) { return SAPB_ABI_VERSION; }

const char* sapb_last_error(void) { return sapb::g_last_error; }

int32_t sapb_contact_solve_occupancy(int32_t dof_per_env, int32_t max_contacts, int32_t hessian_precision,
                                     int32_t line_search_variant) {
  if (line_search_variant < SAPB_LS_MONOTONE_DECAY || line_search_variant > SAPB_LS_EXACT_ROOT) {
    sapb::set_last_error("sapb_contact_solve_occupancy: unknown line search variant %d", line_search_variant);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::contact_solve_occupancy(dof_per_env, max_contacts, hessian_precision, line_search_variant);
}

int32_t sapb_contact_solve_occupancy_threads(int32_t dof_per_env, int32_t max_contacts, int32_t hessian_precision,
                                             int32_t line_search_variant, int32_t threads_per_cta) {
  if (line_search_variant < SAPB_LS_MONOTONE_DECAY || line_search_variant > SAPB_LS_EXACT_ROOT ||
      !(threads_per_cta == 0 || threads_per_cta == 128 || threads_per_cta == 256)) {
    sapb::set_last_error("sapb_contact_solve_occupancy_threads: unknown line search variant %d or thread count %d",
                         line_search_variant, threads_per_cta);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::contact_solve_occupancy(dof_per_env, max_contacts, hessian_precision, line_search_variant,
                                       threads_per_cta);
}

int32_t sapb_contact_solve_ldlt_blocks(int32_t dof_per_env, int32_t* widths, int32_t capacity) {
  if (dof_per_env < 1 || capacity < 0 || (capacity > 0 && !widths)) {
    sapb::set_last_error("sapb_contact_solve_ldlt_blocks: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::ldlt_block_widths(dof_per_env, widths, capacity);
}

void sapb_solve_options_default(sapb_solve_options* o, int32_t variant) {
  // SapContactSolve defaults: sim/contact_solve.py:3299-3316 and 6129-6182.
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->contact_beta = 1.0;
  o->contact_sigma = 1.0e-3;
  o->contact_tau_d = 0.1;
  o->diag_shift = 0.0;
  o->max_iterations = 100;
  o->optimality_abs_tol = 1.0e-14;
  o->optimality_rel_tol = 1.0e-6;
  o->line_search_variant = variant;
  o->cost_abs_tol = variant == SAPB_LS_MONOTONE_DECAY ? 0.0 : 1.0e-30;
  o->cost_rel_tol = variant == SAPB_LS_MONOTONE_DECAY ? 5.0e-3 : 1.0e-15;
  o->line_search_max_iterations = variant == SAPB_LS_EXACT_ROOT ? 100 : 40;
  o->armijo_c = 1.0e-4;
  o->rho = 0.8;
  o->line_search_relative_slop = 1000.0 * 2.220446049250313e-16;
  o->linear_solve_precision = SAPB_FP64;
  o->hessian_precision = SAPB_FP64;
  o->cubic_init = 1;
}

size_t sapb_contact_solve_workspace_size(int32_t num_envs, int32_t dof_per_env, int32_t max_contacts) {
  (void)num_envs;
  (void)dof_per_env;
  (void)max_contacts;
  return 256;  // the persistent kernel's work counter, padded
}

int32_t sapb_contact_solve(const sapb_contact_problem* p, const sapb_solve_options* o, const sapb_solve_outputs* out,
                           void* workspace, size_t workspace_bytes, void* stream) {
  if (!p || !o || !out || !out->v) {
    sapb::set_last_error("sapb_contact_solve: null problem, options or output velocity");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->num_envs < 0 || p->dof_per_env <= 0 || p->max_contacts < 0) {
    sapb::set_last_error("sapb_contact_solve: bad sizes num_envs=%d dof_per_env=%d max_contacts=%d", p->num_envs,
                         p->dof_per_env, p->max_contacts);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->gamma0_count < 0 || p->v_candidate_count < 0) {
    sapb::set_last_error("sapb_contact_solve: negative candidate count");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->dof_per_env > 60) {
    sapb::set_last_error("sapb_contact_solve: dof_per_env=%d > 60 is not supported by the on-chip solve",
                         p->dof_per_env);
    return SAPB_ERR_UNSUPPORTED;
  }
  if (!p->contact_count || !p->dynamics_matrix || !p->v_star || !p->v0 || !p->dt) {
    sapb::set_last_error("sapb_contact_solve: missing required input array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->max_contacts > 0 && (!p->jacobian || !p->phi0 || !p->w_eff || !p->mu || !p->stiffness)) {
    sapb::set_last_error("sapb_contact_solve: missing contact array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->dof && (p->dof->has_pd || p->dof->has_limits) && (!p->dof->dof_coord_index || !p->dof->joint_q)) {
    sapb::set_last_error("sapb_contact_solve: PD/limit terms requested without dof maps");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->dof && p->dof->has_pd &&
      (!p->dof->dof_target_index || !p->dof->joint_target_mode || !p->dof->joint_target_ke ||
       !p->dof->joint_target_kd || !p->dof->joint_effort_limit)) {
    sapb::set_last_error("sapb_contact_solve: PD terms requested without drive arrays");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->dof && p->dof->has_limits &&
      (!p->dof->limit_supported || !p->dof->joint_limit_lower || !p->dof->joint_limit_upper ||
       !p->dof->joint_limit_ke || !p->dof->joint_limit_kd)) {
    sapb::set_last_error("sapb_contact_solve: limit terms requested without limit arrays");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (o->line_search_variant < SAPB_LS_MONOTONE_DECAY || o->line_search_variant > SAPB_LS_EXACT_ROOT) {
    sapb::set_last_error("sapb_contact_solve: unknown line search variant %d", o->line_search_variant);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (!(o->threads_per_cta == 0 || o->threads_per_cta == 128 || o->threads_per_cta == 256)) {
    sapb::set_last_error("sapb_contact_solve: threads_per_cta must be 0, 128 or 256 (got %d)", o->threads_per_cta);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (o->line_search_variant == SAPB_LS_ARMIJO_DECAY && !(o->rho > 0.0 && o->rho < 1.0)) {
    sapb::set_last_error("sapb_contact_solve: rho must lie in (0, 1), got %g", o->rho);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (!workspace || workspace_bytes < sapb_contact_solve_workspace_size(p->num_envs, p->dof_per_env, p->max_contacts)) {
    sapb::set_last_error("sapb_contact_solve: workspace missing or smaller than sapb_contact_solve_workspace_size");
    return SAPB_ERR_WORKSPACE_TOO_SMALL;
  }
  return sapb::contact_solve_launch(p, o, out, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

int32_t sapb_blocked_tree_block(int32_t tree_dofs) { return sapb::blocked_tree_block(tree_dofs); }

int32_t sapb_blocked_fill_capacity(int32_t trees_per_env, int32_t tree_dofs, int32_t max_contacts,
                                   int32_t hessian_precision) {
  return sapb::blocked_fill_capacity(trees_per_env, tree_dofs, max_contacts, hessian_precision == SAPB_FP32);
}

size_t sapb_blocked_solve_workspace_size(int32_t num_envs, int32_t trees_per_env, int32_t max_contacts) {
  (void)num_envs;
  (void)trees_per_env;
  (void)max_contacts;
  return 256;  // the persistent kernel's work counter, padded
}

int32_t sapb_blocked_contact_solve(const sapb_blocked_problem* p, const sapb_solve_options* o,
                                   const sapb_solve_outputs* out, void* workspace, size_t workspace_bytes,
                                   void* stream) {
  if (!p || !o || !out || !out->v) {
    sapb::set_last_error("sapb_blocked_contact_solve: null problem, options or output velocity");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->num_envs < 0 || p->trees_per_env < 1 || p->max_contacts < 0) {
    sapb::set_last_error("sapb_blocked_contact_solve: bad sizes num_envs=%d trees_per_env=%d max_contacts=%d",
                         p->num_envs, p->trees_per_env, p->max_contacts);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->trees_per_env > 64 || p->tree_dofs < 1 || sapb::blocked_tree_block(p->tree_dofs) != p->tree_dofs) {
    sapb::set_last_error("sapb_blocked_contact_solve: supported are <= 64 trees in blocks of 6, 7 or 12 DOFs "
                         "(got %d trees, tree_dofs %d)", p->trees_per_env, p->tree_dofs);
    return SAPB_ERR_UNSUPPORTED;
  }
  if (p->dofs_per_world < 0 || p->dofs_per_world > p->trees_per_env * p->tree_dofs ||
      (!p->tree_dof_start && p->dofs_per_world != 0 && p->dofs_per_world != p->trees_per_env * p->tree_dofs)) {
    sapb::set_last_error("sapb_blocked_contact_solve: dofs_per_world=%d does not fit %d trees of at most %d DOFs",
                         p->dofs_per_world, p->trees_per_env, p->tree_dofs);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->max_contacts > 32767) {
    sapb::set_last_error("sapb_blocked_contact_solve: max_contacts=%d > 32767", p->max_contacts);
    return SAPB_ERR_UNSUPPORTED;
  }
  if (!p->contact_count || !p->tree_mass || !p->v_star || !p->v0 || !p->dt) {
    sapb::set_last_error("sapb_blocked_contact_solve: missing required input array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->max_contacts > 0 && (!p->jacobian || !p->contact_tree || !p->phi0 || !p->w_eff || !p->mu ||
                              !p->stiffness)) {
    sapb::set_last_error("sapb_blocked_contact_solve: missing contact array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->gamma0 && p->gamma0_count > 1) {
    sapb::set_last_error("sapb_blocked_contact_solve: one candidate impulse set at most (gamma0_count=%d)",
                         p->gamma0_count);
    return SAPB_ERR_UNSUPPORTED;
  }
  if (p->dof && (p->dof->has_pd || p->dof->has_limits) && (!p->dof->dof_coord_index || !p->dof->joint_q)) {
    sapb::set_last_error("sapb_blocked_contact_solve: drive / limit terms need dof_coord_index and joint_q");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->dof && p->dof->has_pd &&
      (!p->dof->dof_target_index || !p->dof->joint_target_mode || !p->dof->joint_target_ke ||
       !p->dof->joint_target_kd || !p->dof->joint_effort_limit)) {
    sapb::set_last_error("sapb_blocked_contact_solve: drive terms need their target and gain arrays");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (p->dof && p->dof->has_limits &&
      (!p->dof->limit_supported || !p->dof->joint_limit_lower || !p->dof->joint_limit_upper ||
       !p->dof->joint_limit_ke || !p->dof->joint_limit_kd)) {
    sapb::set_last_error("sapb_blocked_contact_solve: limit terms need their limit arrays");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (o->line_search_variant < SAPB_LS_MONOTONE_DECAY || o->line_search_variant > SAPB_LS_EXACT_ROOT) {
    sapb::set_last_error("sapb_blocked_contact_solve: unknown line search variant %d", o->line_search_variant);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (o->line_search_variant == SAPB_LS_ARMIJO_DECAY && !(o->rho > 0.0 && o->rho < 1.0)) {
    sapb::set_last_error("sapb_blocked_contact_solve: rho must lie in (0, 1), got %g", o->rho);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (!workspace ||
      workspace_bytes < sapb_blocked_solve_workspace_size(p->num_envs, p->trees_per_env, p->max_contacts)) {
    sapb::set_last_error("sapb_blocked_contact_solve: workspace missing or too small");
    return SAPB_ERR_WORKSPACE_TOO_SMALL;
  }
  return sapb::blocked_solve_launch(p, o, out, workspace, static_cast<cudaStream_t>(stream));
}

int32_t sapb_dense_to_blocked(const sapb_contact_problem* d, int32_t trees_per_env, int32_t tree_dofs,
                              const int32_t* tree_dof_start, double* tree_mass, double* jacobian,
                              int32_t* contact_tree, void* stream) {
  if (!d || !tree_mass || !jacobian || !contact_tree || !d->dynamics_matrix || !d->body_dof_start ||
      (d->max_contacts > 0 && !d->jacobian)) {
    sapb::set_last_error("sapb_dense_to_blocked: missing array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const int64_t cover = (int64_t)trees_per_env * tree_dofs;
  if (trees_per_env < 1 || trees_per_env > 64 || tree_dofs < 1 || d->num_envs < 0 || d->max_contacts < 0 ||
      (tree_dof_start ? cover < d->dof_per_env : cover != d->dof_per_env)) {
    sapb::set_last_error("sapb_dense_to_blocked: %d trees of %s%d DOFs do not make dof_per_env=%d", trees_per_env,
                         tree_dof_start ? "at most " : "", tree_dofs, d->dof_per_env);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::dense_to_blocked_launch(d, trees_per_env, tree_dofs, tree_dof_start, tree_mass, jacobian,
                                       contact_tree, static_cast<cudaStream_t>(stream));
}

size_t sapb_prepare_workspace_size(const sapb_model_desc* m, int32_t max_contacts) {
  if (!m || max_contacts < 0) return 0;
  return sizeof(int32_t) * ((size_t)m->num_worlds * (size_t)(max_contacts + 1) + 1) + 256;
}

static int32_t check_model(const sapb_model_desc* m, const char* where) {
  if (!m || m->num_worlds < 0 || m->joints_per_world <= 0 || m->bodies_per_world <= 0 || m->dofs_per_world <= 0 ||
      m->articulations_per_world <= 0) {
    sapb::set_last_error("%s: bad model sizes", where);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (!m->joint_type || !m->joint_parent || !m->joint_child || !m->joint_ancestor || !m->joint_q_start ||
      !m->joint_qd_start || !m->joint_dof_dim || !m->articulation_start || !m->joint_axis || !m->joint_X_p ||
      !m->joint_X_c || !m->joint_armature || !m->body_mass || !m->body_inertia || !m->body_com || !m->gravity) {
    sapb::set_last_error("%s: missing model array", where);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const bool uneven = m->world_joint_start || m->world_body_start || m->world_dof_start ||
                      m->world_articulation_start || m->body_world;
  if (uneven && (!m->world_joint_start || !m->world_body_start || !m->world_dof_start ||
                 !m->world_articulation_start || !m->body_world || m->total_joints <= 0 || m->total_bodies <= 0 ||
                 m->total_dofs <= 0 || m->total_articulations <= 0)) {
    sapb::set_last_error("%s: an uneven batch needs all four world offset arrays, body_world and the totals", where);
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return SAPB_OK;
}

int32_t sapb_free_motion_contacts(const sapb_model_desc* m, const sapb_step_inputs* in,
                                  const sapb_prepare_options* o, const sapb_prepare_outputs* out,
                                  void* workspace, size_t workspace_bytes, void* stream) {
  const int32_t st = check_model(m, "sapb_free_motion_contacts");
  if (st != SAPB_OK) return st;
  const bool blk = o && o->tree_blocked;
  if (!in || !o || !out || !in->joint_q || !in->joint_qd || !in->dt || !out->v_star ||
      (blk ? (!out->tree_mass || !out->contact_tree) : !out->dynamics_matrix)) {
    sapb::set_last_error("sapb_free_motion_contacts: missing input or output array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (o->max_contacts < 0 || in->contact_capacity < 0) {
    sapb::set_last_error("sapb_free_motion_contacts: negative contact sizes");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (in->contact_capacity > 0 &&
      (!in->contact_count || !in->contact_shape0 || !in->contact_shape1 || !in->contact_point0 ||
       !in->contact_point1 || !in->contact_normal || !m->shape_body)) {
    sapb::set_last_error("sapb_free_motion_contacts: missing contact array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (o->max_contacts > 0 && (!out->jacobian || !out->phi0 || !out->w_eff || !out->mu || !out->stiffness ||
                              !out->tau_d || !out->body0 || !out->body1)) {
    sapb::set_last_error("sapb_free_motion_contacts: missing contact output array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (blk && m->world_joint_start) {
    sapb::set_last_error("sapb_free_motion_contacts: tree-blocked outputs need equal per-world blocks");
    return SAPB_ERR_UNSUPPORTED;
  }
  const int tree_block = blk ? (o->tree_dofs > 0 ? o->tree_dofs : 6) : 0;
  if (blk && (m->bodies_per_world > 64 || m->articulations_per_world < 1 ||
              sapb::blocked_tree_block(tree_block) != tree_block ||
              (int64_t)m->articulations_per_world * tree_block < m->dofs_per_world || out->dynamics_factor)) {
    sapb::set_last_error("sapb_free_motion_contacts: tree-blocked outputs need worlds of <= 64 bodies whose "
                         "articulations fit blocks of tree_dofs in {6, 7, 12} (got %d bodies, %d articulations, "
                         "%d DOFs, tree_dofs %d) and no dynamics_factor output",
                         m->bodies_per_world, m->articulations_per_world, m->dofs_per_world, tree_block);
    return SAPB_ERR_UNSUPPORTED;
  }
  if (!blk && (m->bodies_per_world > 64 || m->dofs_per_world > 128)) {
    sapb::set_last_error("sapb_free_motion_contacts: at most 64 bodies and 128 DOFs per world (got %d, %d)",
                         m->bodies_per_world, m->dofs_per_world);
    return SAPB_ERR_UNSUPPORTED;
  }
  const size_t smem = sapb::prepare_smem_bytes(m->bodies_per_world, m->dofs_per_world, o->max_contacts, tree_block);
  if (smem > sapb::kMaxSmemPerBlock) {
    sapb::set_last_error("sapb_free_motion_contacts: world too large for one block (%zu bytes of shared memory)",
                         smem);
    return SAPB_ERR_UNSUPPORTED;
  }
  if (!workspace || workspace_bytes < sapb_prepare_workspace_size(m, o->max_contacts)) {
    sapb::set_last_error("sapb_free_motion_contacts: workspace missing or too small");
    return SAPB_ERR_WORKSPACE_TOO_SMALL;
  }
  return sapb::prepare_launch(m, in, o, out, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

int32_t sapb_public_to_sap(const sapb_model_desc* m, const double* joint_q, const double* body_q,
                           const double* joint_qd_public, const double* joint_f_public,
                           const double* body_f_public, double* joint_qd_sap, double* joint_f_sap,
                           double* body_f_sap, void* stream) {
  const int32_t st = check_model(m, "sapb_public_to_sap");
  if (st != SAPB_OK) return st;
  if ((joint_qd_public && !joint_qd_sap) || (joint_f_public && !joint_f_sap) || (body_f_public && !body_f_sap) ||
      ((joint_qd_public || joint_f_public) && !joint_q) || (body_f_public && !body_q)) {
    sapb::set_last_error("sapb_public_to_sap: an input without its output or pose array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::public_to_sap_launch(m, joint_q, body_q, joint_qd_public, joint_f_public, body_f_public, joint_qd_sap,
                                    joint_f_sap, body_f_sap, static_cast<cudaStream_t>(stream));
}

int32_t sapb_sap_to_public_velocity(const sapb_model_desc* m, const double* joint_q, const double* joint_qd_sap,
                                    double* joint_qd_public, void* stream) {
  const int32_t st = check_model(m, "sapb_sap_to_public_velocity");
  if (st != SAPB_OK) return st;
  if (!joint_q || !joint_qd_sap || !joint_qd_public) {
    sapb::set_last_error("sapb_sap_to_public_velocity: missing array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::sap_to_public_launch(m, joint_q, joint_qd_sap, joint_qd_public, static_cast<cudaStream_t>(stream));
}

int32_t sapb_eval_fk(const sapb_model_desc* m, const double* joint_q, const double* joint_qd_public, double* body_q,
                     double* body_qd, void* stream) {
  const int32_t st = check_model(m, "sapb_eval_fk");
  if (st != SAPB_OK) return st;
  if (!joint_q || !body_q || (body_qd && !joint_qd_public)) {
    sapb::set_last_error("sapb_eval_fk: missing array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::eval_fk_launch(m, joint_q, joint_qd_public, body_q, body_qd, static_cast<cudaStream_t>(stream));
}

size_t sapb_contacts_workspace_size(const sapb_collision_shapes* shapes) {
  if (!shapes || shapes->num_worlds < 0 || shapes->shapes_per_world < 0 || shapes->num_global_shapes < 0) return 0;
  return sapb::contacts_workspace_bytes(shapes);
}

int32_t sapb_generate_contacts(const sapb_collision_shapes* sh, const double* body_q, const sapb_contact_outputs* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  if (!sh || !out || !out->count || sh->num_worlds < 0 || sh->shapes_per_world < 0 || sh->num_global_shapes < 0 ||
      out->capacity < 0) {
    sapb::set_last_error("sapb_generate_contacts: bad arguments");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (sh->shapes_per_world > 4096) {
    sapb::set_last_error("sapb_generate_contacts: shapes_per_world=%d > 4096", sh->shapes_per_world);
    return SAPB_ERR_UNSUPPORTED;
  }
  if ((sh->num_worlds * sh->shapes_per_world + sh->num_global_shapes) > 0 &&
      (!sh->shape_type || !sh->shape_scale || !sh->shape_X_bs || !sh->shape_body || !body_q)) {
    sapb::set_last_error("sapb_generate_contacts: missing shape array or body poses");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (out->capacity > 0 && (!out->shape0 || !out->shape1 || !out->point0 || !out->point1 || !out->normal ||
                            !out->margin0 || !out->margin1)) {
    sapb::set_last_error("sapb_generate_contacts: missing output array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (!workspace || workspace_bytes < sapb::contacts_workspace_bytes(sh)) {
    sapb::set_last_error("sapb_generate_contacts: workspace missing or smaller than sapb_contacts_workspace_size");
    return SAPB_ERR_WORKSPACE_TOO_SMALL;
  }
  return sapb::contacts_launch(sh, body_q, out, workspace, static_cast<cudaStream_t>(stream));
}

int32_t sapb_integrate_positions(const sapb_model_desc* m, const double* q_in, const double* v_prev,
                                 const double* v_new, const double* dt, int32_t mode, double* q_out, void* stream) {
  const int32_t st = check_model(m, "sapb_integrate_positions");
  if (st != SAPB_OK) return st;
  if (m->world_joint_start) {
    sapb::set_last_error("sapb_integrate_positions: equal per-world blocks only (sapb_step_tail_launch takes uneven "
                         "batches)");
    return SAPB_ERR_UNSUPPORTED;
  }
  if (!q_in || !v_new || !dt || !q_out || (mode == SAPB_INTEGRATE_MIDPOINT && !v_prev) ||
      (mode != SAPB_INTEGRATE_MIDPOINT && mode != SAPB_INTEGRATE_SAP_EULER)) {
    sapb::set_last_error("sapb_integrate_positions: bad arguments");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  return sapb::integrate_launch(m, q_in, v_prev, v_new, dt, mode, q_out, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
