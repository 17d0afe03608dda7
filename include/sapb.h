/*
 * sapb.h -- C ABI of the B200-native SAP contact step.
 *
 * Every array argument is a raw pointer plus the sizes carried in the
 * descriptor structs below; no torch or CUDA C++ types appear in a signature.
 * Device entry points (sapb_*) take DEVICE pointers and a cudaStream_t passed
 * as `void*`; they never synchronise the host and never allocate, so a caller
 * may capture them in a CUDA graph.  The same descriptor structs are used by
 * the CPU oracle (oracle/sap_oracle.h) with HOST pointers.
 *
 * Index conventions follow the reference (mardigiorgio/sap_warp):
 *   E = num_envs (worlds), n = dof_per_env, C = max_contacts (per-world slots),
 *   all worlds have the same n (sim/contact_solve.py:3327-3335),
 *   generalized velocities are in SAP order, flat [E*n]
 *   (sim/contact_solve.py:299-338),
 *   per-world dense dynamics matrix A [E,n,n] (sim/contact_jacobian.py:110-150),
 *   per-contact Jacobian rows J [E,C,3,n], rows = (t1, t2, n) of the contact
 *   frame (sim/contact_jacobian.py:404-562).
 */
#ifndef SAPB_H
#define SAPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SAPB_ABI_VERSION 1

/* ---- return / status codes ------------------------------------------------ */
#define SAPB_OK 0
/* host-side argument errors (returned by the entry points) */
#define SAPB_ERR_INVALID_ARGUMENT (-100)
#define SAPB_ERR_UNSUPPORTED (-101)
#define SAPB_ERR_CUDA (-102)
#define SAPB_ERR_WORKSPACE_TOO_SMALL (-103)
/* per-world line-search status, the reference's device codes
 * (sim/contact_solve.py:2703-2705, 2873, 2904, 2989, 3026, 3099) */
#define SAPB_LS_ASCENT_DIRECTION (-1)
#define SAPB_LS_ALPHA_UNDERFLOW (-2)
#define SAPB_LS_BAD_BRACKET (-3)
#define SAPB_LS_BAD_GUESS (-4)
#define SAPB_LS_ROOT_ITERATION_CAP (-5)

/* contact modes (sim/contact_solve.py:60-63) */
#define SAPB_CONTACT_MODE_NONE 0
#define SAPB_CONTACT_MODE_STICTION 1
#define SAPB_CONTACT_MODE_SLIDING 2
#define SAPB_CONTACT_MODE_FRICTIONLESS 3

/* line-search variants (sim/contact_solve.py:69-81) */
#define SAPB_LS_MONOTONE_DECAY 0
#define SAPB_LS_ARMIJO_DECAY 1
#define SAPB_LS_EXACT_ROOT 2

/* precisions (sim/solver_sap.py:62-70) */
#define SAPB_FP64 0
#define SAPB_FP32 1

/* ---- contact solve ---------------------------------------------------------
 * Options of SapContactSolve.__init__ / .solve
 * (sim/contact_solve.py:3299-3316 and 6129-6154).  sapb_solve_options_default
 * fills the reference's SapContactSolve defaults. */
typedef struct sapb_solve_options {
  double contact_beta;            /* 1.0 */
  double contact_sigma;           /* 1e-3 */
  double contact_tau_d;           /* per-pair fallback when tau_d == NULL: 0.1 */
  double diag_shift;              /* 0.0 */
  int32_t max_iterations;         /* 100 */
  double optimality_abs_tol;      /* 1e-14 */
  double optimality_rel_tol;      /* 1e-6 */
  double cost_abs_tol;            /* variant dependent, sim/contact_solve.py:6178-6181 */
  double cost_rel_tol;            /* variant dependent */
  int32_t line_search_max_iterations; /* 40 (100 for exact_root) */
  double armijo_c;                /* 1e-4 */
  double rho;                     /* 0.8 */
  double line_search_relative_slop; /* 1000 * eps(fp64) */
  int32_t line_search_variant;    /* SAPB_LS_* ; solve() default monotone_decay */
  int32_t linear_solve_precision; /* SAPB_FP64 / SAPB_FP32: Newton-direction Cholesky */
  int32_t hessian_precision;      /* SAPB_FP64 / SAPB_FP32: J^T G J assembly */
  int32_t cubic_init;             /* exact_root cubic seed, sim/contact_solve.py:55-58 (1) */
} sapb_solve_options;

/* Per-DOF drive and limit model (the arrays SapContactSolve.prepare reads,
 * sim/contact_solve.py:4336-4429, with the maps of _build_dof_maps
 * sim/contact_solve.py:3681-3722 and _build_body_dof_maps :3724-3758).
 * Pointers may be NULL when has_pd / has_limits is 0.  Indices are global
 * (flat over all worlds) like the reference's model arrays. */
typedef struct sapb_dof_terms {
  int32_t has_pd;                 /* _detect_model_pd_terms, :3760-3770 */
  int32_t has_limits;             /* _detect_model_limit_terms, :3772-3785 */
  int32_t joint_coord_count;      /* length of joint_q; coordinates beyond it are ignored */
  const int32_t* dof_coord_index; /* [E*n] coordinate of each DOF or -1 */
  const int32_t* dof_target_index;/* [E*n] */
  const int32_t* limit_supported; /* [E*n] */
  const int32_t* joint_target_mode; /* [E*n] */
  const float* joint_target_ke;   /* [E*n] */
  const float* joint_target_kd;   /* [E*n] */
  const float* joint_effort_limit;/* [E*n] */
  const double* joint_limit_lower;/* [E*n] */
  const double* joint_limit_upper;/* [E*n] */
  const double* joint_limit_ke;   /* [E*n] */
  const double* joint_limit_kd;   /* [E*n] */
  const double* joint_q;          /* [coords] generalized positions */
  const float* joint_target_pos;  /* [E*n] or NULL (zeros) */
  const float* joint_target_vel;  /* [E*n] or NULL (zeros) */
  const float* joint_act;         /* [E*n] or NULL (zeros) */
} sapb_dof_terms;

/* The stage-2 problem of one step: SapContactJacobianResult fields
 * (sim/contact_jacobian.py:51-84) plus the velocities of solve().
 * Device pointers for sapb_contact_solve, host pointers for the oracle. */
typedef struct sapb_contact_problem {
  int32_t num_envs;
  int32_t dof_per_env;
  int32_t max_contacts;           /* C: per-world slot capacity */
  int32_t num_bodies;             /* length of body_dof_start / body_dof_count */
  const int32_t* contact_count;   /* [E] contacts per world (clamped to C) */
  const double* dynamics_matrix;  /* [E,n,n] */
  const double* jacobian;         /* [E,C,3,n] */
  const double* phi0;             /* [E,C] */
  const double* w_eff;            /* [E,C] */
  const double* mu;               /* [E,C] */
  const double* stiffness;        /* [E,C] */
  const double* tau_d;            /* [E,C] or NULL -> options.contact_tau_d */
  const int32_t* body0;           /* [E,C] global body of shape0 or -1 (NULL: none) */
  const int32_t* body1;           /* [E,C] */
  const int32_t* body_dof_start;  /* [bodies] env-local first DOF of a body's articulation, -1 */
  const int32_t* body_dof_count;  /* [bodies] */
  const double* v_star;           /* [E*n] free-motion velocity */
  const double* v0;               /* [E*n] start-of-step velocity */
  double* v_guess;                /* [E*n] warm start in / seeded velocity out, or NULL */
  const int32_t* v_guess_active;  /* [1] nonzero: start from v_guess; NULL: never */
  const double* dt;               /* [E] per-world time step */
  const sapb_dof_terms* dof;      /* NULL: no PD / limit terms */
} sapb_contact_problem;

/* Outputs: the SapContactSolveResult fields a caller reads
 * (sim/contact_solve.py:188-232).  Any pointer except v may be NULL. */
typedef struct sapb_solve_outputs {
  double* v;                      /* [E*n] solved velocity (v_flat) */
  double* contact_gamma;          /* [E,C,3] impulses at the solution */
  int32_t* contact_mode;          /* [E,C] projection mode at the returned velocity */
  double* cost;                   /* [E] */
  int32_t* newton_iterations;     /* [E] */
  int32_t* line_search_iterations;/* [E] accumulated accepted trials */
  int32_t* converged;             /* [E] 1 if optimality or cost test met */
  int32_t* status;                /* [E] last line-search status (0 or SAPB_LS_*) */
  double* grad_norm;              /* [E] ||D^-1/2 grad|| over participating DOFs */
} sapb_solve_outputs;

/* Fill the reference defaults of SapContactSolve for a line-search variant.
 * Replaces the Python defaults of solve(), sim/contact_solve.py:6129-6182. */
void sapb_solve_options_default(sapb_solve_options* opts, int32_t line_search_variant);

/* ABI version of the loaded library (SAPB_ABI_VERSION). */
int32_t sapb_abi_version(void);

/* Bytes of device workspace sapb_contact_solve needs for this shape.
 * Replaces the work buffers allocated in SapContactSolve.__init__
 * (sim/contact_solve.py:3454-3652). */
size_t sapb_contact_solve_workspace_size(int32_t num_envs, int32_t dof_per_env, int32_t max_contacts);

/* Solve the SAP stage-2 problem of every world in one launch.
 * Replaces SapContactSolve.solve (sim/contact_solve.py:6129-6285), including
 * prepare() (:4285-4429) and the conditional Newton loop (:5474-5655).
 * workspace: device buffer of sapb_contact_solve_workspace_size bytes.
 * stream: cudaStream_t.  Returns SAPB_OK or a host-side SAPB_ERR_*. */
int32_t sapb_contact_solve(const sapb_contact_problem* problem, const sapb_solve_options* opts,
                           const sapb_solve_outputs* out, void* workspace, size_t workspace_bytes,
                           void* stream);

/* The same solve as sapb_contact_solve for callers that cannot allocate device
 * memory (for example a plugin whose host runtime owns every device
 * allocation, or a binding with no device allocator): no workspace argument,
 * and no cudaMalloc / cudaFree or allocating library call.  No counterpart in
 * the reference.  Its scratch is a fixed 4 KiB array compiled into the
 * library, held by every GPU that loads the library until exit; problems
 * whose sapb_contact_solve_workspace_size exceeds it are rejected with
 * SAPB_ERR_WORKSPACE_TOO_SMALL.  The first call on a device looks up the
 * array's device address (once per device, with that device current); make
 * that first call before any stream capture.  All calls share the array and
 * the solve clears what must start at zero, so calls that overlap on the GPU
 * (concurrent streams) race: serialize them. */
int32_t sapb_contact_solve_noalloc(const sapb_contact_problem* problem, const sapb_solve_options* opts,
                                   const sapb_solve_outputs* out, void* stream);

/* Last CUDA error string seen by the library on this thread ("" if none). */
const char* sapb_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* SAPB_H */
