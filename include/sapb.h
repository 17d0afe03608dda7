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

#define SAPB_ABI_VERSION 20

/* ---- return / status codes ------------------------------------------------ */
#define SAPB_OK 0
/* host-side argument errors (returned by the entry points) */
#define SAPB_ERR_INVALID_ARGUMENT (-100)
#define SAPB_ERR_UNSUPPORTED (-101)
#define SAPB_ERR_CUDA (-102)
#define SAPB_ERR_WORKSPACE_TOO_SMALL (-103)
#define SAPB_ERR_TIMEOUT (-104)          /* a bounded device-side wait gave up */
/* per-world line-search status, the reference's device codes
 * (sim/contact_solve.py:2703-2705, 2873, 2904, 2989, 3026, 3099) */
#define SAPB_LS_ASCENT_DIRECTION (-1)
#define SAPB_LS_ALPHA_UNDERFLOW (-2)
#define SAPB_LS_BAD_BRACKET (-3)
#define SAPB_LS_BAD_GUESS (-4)
#define SAPB_LS_ROOT_ITERATION_CAP (-5)
/* Per-world status of sapb_blocked_contact_solve: the world's block factor
 * needs more off-diagonal blocks than sapb_blocked_fill_capacity; v = v*. */
#define SAPB_WORLD_FACTOR_CAPACITY (-10)
/* Per-world statuses of sapb_contact_solve (no counterpart in the reference,
 * whose solve carries NaNs to the iteration cap): a NaN / Inf in the world's
 * inputs (A, J, phi0, w_eff, mu, stiffness, tau_d, v*, start velocity) --
 * the world is not solved, v = its start velocity, no iterations; a Newton
 * factorization met a pivot that is not positive and finite (H not SPD) --
 * the solve stops there, v = the last accepted iterate. */
#define SAPB_WORLD_NOT_FINITE (-11)
#define SAPB_WORLD_NOT_SPD (-12)

/* contact modes (sim/contact_solve.py:60-63) */
#define SAPB_CONTACT_MODE_NONE 0
#define SAPB_CONTACT_MODE_STICTION 1
#define SAPB_CONTACT_MODE_SLIDING 2
#define SAPB_CONTACT_MODE_FRICTIONLESS 3

/* joint types (sim/sap_runtime.py:21-27) */
#define SAPB_JOINT_PRISMATIC 0
#define SAPB_JOINT_REVOLUTE 1
#define SAPB_JOINT_BALL 2
#define SAPB_JOINT_FIXED 3
#define SAPB_JOINT_FREE 4
#define SAPB_JOINT_DISTANCE 5
#define SAPB_JOINT_D6 6

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
  int32_t ctas_per_sm;            /* resident CTAs per SM of the persistent dense solve: 0 as many as fit
                                   * (sapb_contact_solve_occupancy), k at most k; results do not depend on it */
  int32_t ldlt_block;             /* column-block width of the dense solve's LDL^T: 0 the default for the DOF
                                   * count, else one of sapb_contact_solve_ldlt_blocks (others: the default);
                                   * the width changes the factorization's rounding, not the tolerance */
  int32_t skip_plain_start;       /* nonzero, with candidate starts: start from the best candidate without
                                   * evaluating the plain start (v_guess or v0), which is kept only as the
                                   * fallback when no candidate's cost is finite; 0: the plain start competes */
  int32_t threads_per_cta;        /* threads of one world's CTA in the dense solve: 0 or 128 the default (the
                                   * kernel specialised on the DOF count), 256 the runtime-size kernel with
                                   * eight warps per world (for worlds whose shared memory leaves one or two
                                   * CTAs per SM); in the tree-blocked solve 128 or 256, 0 picking 128 for
                                   * worlds of up to 128 padded DOFs (T * tree_dofs) and 256 beyond; results
                                   * do not depend on it beyond rounding */
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
  /* Uneven batches (the solve's dof_count): [E+1] offsets of each world's
   * DOFs in the model's global DOF order, in which the per-DOF arrays above
   * and dof_target_index then are (world e's DOF i is world_dof_start[e] +
   * i); NULL: the per-DOF arrays are in the solve's [E*n] layout. */
  const int32_t* world_dof_start;
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
  /* Candidate starts (no counterpart in the reference): gamma0_count sets of
   * starting impulses [K][E,C,3] back to back, or NULL.  For each set the
   * solve forms v_c = v* + A^-1 J^T gamma_c on the participating DOFs and
   * starts Newton from the lowest-cost start among the plain one (v_guess or
   * v0) and the candidates.  gamma0_count <= 1 means one set. */
  const double* gamma0;
  int32_t gamma0_count;
  /* Optional [E,n,n] LDL^T factor of dynamics_matrix as written by
   * sapb_free_motion_contacts (dynamics_factor output): the candidate starts
   * solve with it instead of factoring A again.  NULL: factor in the solve. */
  const double* dynamics_factor;
  /* Optional [E] order in which the persistent kernel takes the worlds (a
   * permutation of 0..E-1, e.g. by descending estimated work for uneven
   * batches); entries outside [0, E) are skipped.  NULL: index order. */
  const int32_t* world_order;
  /* Candidate start velocities [K][E*n] back to back (v_candidate_count <= 1
   * means one), or NULL: each is taken on the participating DOFs (v* on the
   * others) and tried like the impulse candidates, before them -- e.g. the
   * v_start output of sapb_free_motion_contacts.  Chosen-start numbering:
   * 0 plain, 1..K the velocity candidates, K+1.. the impulse sets. */
  const double* v_candidates;
  int32_t v_candidate_count;
  /* Optional [E*n] base velocity of the impulse candidates: v_c = base +
   * A^-1 J^T gamma_c (NULL: base = v*).  A world whose candidate impulses are
   * all zero then starts at the base without reading dynamics_factor. */
  const double* gamma0_base;
  /* Optional [E] DOF count of each world (uneven batches without padding,
   * 1..dof_per_env): world e uses the first dof_count[e] of its dof_per_env
   * DOF slots.  Its A block is stored compact at the start of its slot
   * (dof_count[e]^2 values, row stride dof_count[e]), its Jacobian rows
   * likewise (stride dof_count[e]), its per-DOF arrays (v*, v0, v_guess, v,
   * dof terms, candidates, factor) at e * dof_per_env + [0, dof_count[e]);
   * the rest of its v slots are written as zero.  Runs the runtime-size
   * kernel.  NULL: every world has dof_per_env DOFs. */
  const int32_t* dof_count;
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
  int32_t* warm_start_accepted;   /* [E] chosen start: 0 plain, then the velocity candidates, then the impulse
                                   * sets, counted from 1 (NULL: not written) */
} sapb_solve_outputs;

/* ---- free motion + contact Jacobian ---------------------------------------
 * Model of W replicated worlds with equal contiguous per-world blocks of
 * joints, bodies, DOFs and coordinates (the layout the reference requires,
 * sim/contact_solve.py:3327-3335).  Arrays are global (all worlds), indices
 * global, as in SapModel (sim/sap_runtime.py:47-174).  Joints are ordered
 * parents before children within each articulation. */
typedef struct sapb_model_desc {
  int32_t num_worlds;
  int32_t joints_per_world;
  int32_t bodies_per_world;
  int32_t dofs_per_world;
  int32_t coords_per_world;
  int32_t articulations_per_world;
  int32_t num_shapes;
  const int32_t* joint_type;        /* [J] SAP_JOINT_* of sim/sap_runtime.py:21-27 */
  const int32_t* joint_parent;      /* [J] parent body or -1 */
  const int32_t* joint_child;       /* [J] child body */
  const int32_t* joint_ancestor;    /* [J] parent joint or -1 */
  const int32_t* joint_q_start;     /* [J+1] */
  const int32_t* joint_qd_start;    /* [J+1] */
  const int32_t* joint_dof_dim;     /* [J][2] linear, angular axis counts */
  const int32_t* articulation_start;/* [A+1] */
  const double* joint_axis;         /* [dofs][3] */
  const double* joint_X_p;          /* [J][7] p, q(xyzw): joint frame F in the parent */
  const double* joint_X_c;          /* [J][7] joint frame M in the child */
  const double* joint_armature;     /* [dofs] */
  const double* body_mass;          /* [B] */
  const double* body_inertia;       /* [B][3][3] about the COM, body axes */
  const double* body_com;           /* [B][3] body frame */
  const double* gravity;            /* [W][3] */
  const int32_t* shape_body;        /* [S] (-1: static) */
  const double* shape_material_mu;  /* [S] or NULL -> fallback */
  const double* shape_material_ke;  /* [S] or NULL -> fallback */
  const double* shape_material_tau; /* [S] or NULL -> fallback */
  /* Uneven batches (no counterpart in the reference, whose per-world blocks
   * are equal, sim/contact_solve.py:3327-3335).  NULL: every world has the
   * *_per_world counts.  Else [W+1] prefix offsets of each world's joints,
   * bodies, DOFs and articulations in the global arrays, the world of each
   * body [B], and the totals; the *_per_world counts are then the largest
   * world's (coordinates follow joint_q_start).  The free motion then writes
   * the solve's per-DOF arrays (v*, vdot, v_start, qd_slots) in slots of
   * dofs_per_world per world, A and the Jacobian rows compact in their
   * slots -- the layout of sapb_contact_problem.dof_count -- and the step's
   * tail reads the solve's velocities from those slots.  The dense layout
   * only (the C handle included); sapb_integrate_positions takes equal
   * blocks. */
  const int32_t* world_joint_start;
  const int32_t* world_body_start;
  const int32_t* world_dof_start;
  const int32_t* world_articulation_start;
  const int32_t* body_world;
  int32_t total_joints, total_bodies, total_dofs, total_articulations;
} sapb_model_desc;

/* Start-of-step state, control and the flat contact buffer of collision
 * (SapState / SapControl / SapContacts, sim/sap_runtime.py:177-264), SAP DOF
 * order, FP64 mirrors of the contact arrays. */
typedef struct sapb_step_inputs {
  const double* joint_q;            /* [coords] */
  const double* joint_qd;           /* [dofs] */
  const double* joint_f;            /* [dofs] or NULL */
  const double* body_f;             /* [B][6] negated applied wrench at the body origin, or NULL */
  const double* dt;                 /* [W] */
  int32_t contact_capacity;         /* length of the flat contact arrays */
  const int32_t* contact_count;     /* [1] live contacts */
  const int32_t* contact_shape0;    /* [N] */
  const int32_t* contact_shape1;    /* [N] */
  const double* contact_point0;     /* [N][3] in the body frame of shape0's body (world if static) */
  const double* contact_point1;     /* [N][3] */
  const double* contact_normal;     /* [N][3] world, from shape0 to shape1 */
  const double* contact_margin0;    /* [N] */
  const double* contact_margin1;    /* [N] */
} sapb_step_inputs;

#define SAPB_WEIGHT_BODY_INERTIA 0
#define SAPB_WEIGHT_DIAG_DELASSUS 1
#define SAPB_POINT_WITNESS 0
#define SAPB_POINT_MIDPOINT 1

typedef struct sapb_prepare_options {
  int32_t max_contacts;             /* per-world slots (max_rigid_contact) */
  int32_t contact_weight_mode;      /* SAPB_WEIGHT_* (sim/contact_jacobian.py:153-401) */
  int32_t contact_point_mode;       /* SAPB_POINT_* */
  double fallback_mu;
  double fallback_stiffness;
  double fallback_tau_d;
  /* Nonzero: tree-blocked outputs.  The trees are the world's articulations
   * (a free body is one tree of 6 DOFs; an arm another), each holding at
   * most tree_dofs DOFs, contiguous in the world's DOF order.  tree_mass
   * [W][T][NB][NB] (T articulations per world, NB = tree_dofs: a tree's
   * block of A, padded with the identity beyond its own DOFs) and
   * contact_tree are written, jacobian is [W][C][3][2 NB] in the layout of
   * sapb_blocked_problem (zero in padded columns), and dynamics_matrix /
   * dynamics_factor are not written (may be NULL).  A world with a tree of
   * more than tree_dofs DOFs gets NaN in v_star, so the solve reports it
   * SAPB_WORLD_NOT_FINITE.  No counterpart in the reference, which keeps
   * every world dense: A_env with the zero blocks between trees and rows
   * over all DOFs (sim/contact_jacobian.py:110-150, 404-562).  At most 64
   * bodies per world. */
  int32_t tree_blocked;
  /* Nonzero (with a history whose has_history marks new contacts): write
   * dynamics_factor only for worlds with a new contact in a live slot, the
   * only worlds whose network-predicted impulses need it; other worlds'
   * factors are left unwritten. */
  int32_t factor_new_contacts_only;
  int32_t tree_dofs;                /* NB of the tree-blocked outputs (0: 6, worlds of free bodies) */
} sapb_prepare_options;

/* Outputs: SapFreeMotionResult (sim/free_motion.py:63-68) and the
 * SapContactJacobianResult arrays the contact solve reads
 * (sim/contact_jacobian.py:51-84).  Any pointer but v_star,
 * dynamics_matrix, jacobian and the contact arrays may be NULL. */
struct sapb_contact_history;

typedef struct sapb_prepare_outputs {
  double* v_star;                   /* [dofs] */
  double* vdot;                     /* [dofs] */
  double* dynamics_matrix;          /* [W][n][n]  A = M + diag(armature) */
  double* jacobian;                 /* [W][C][3][n] */
  int32_t* contact_count;           /* [W] contacts in each world (before clamping to C) */
  double* phi0;                     /* [W][C] */
  double* w_eff;                    /* [W][C] */
  double* mu;                       /* [W][C] */
  double* stiffness;                /* [W][C] */
  double* tau_d;                    /* [W][C] */
  int32_t* body0;                   /* [W][C] global bodies */
  int32_t* body1;                   /* [W][C] */
  double* point;                    /* [W][C][3] stiffness-weighted contact point, or NULL */
  double* frame;                    /* [W][C][9] rows t1, t2, n, or NULL */
  int32_t* truncated_count;         /* [1] contacts beyond max_contacts, or NULL */
  double* body_q;                   /* [B][7] start-of-step body poses, or NULL */
  double* dynamics_factor;          /* [W][n][n] LDL^T of A (below the diagonal L_ik d_k, on it d_k;
                                       above it unspecified), or NULL */
  double* vc_star;                  /* [W][C][3] free-motion contact velocities J_c v*, or NULL */
  double* tree_mass;                /* [W][T][NB][NB] diagonal blocks of A (tree_blocked only) */
  int32_t* contact_tree;            /* [W][C][2] tree of each contact side, -1 static (tree_blocked only) */
  int32_t* contact_source;          /* [W][C] flat contact index of each slot, -1 past the world's count, or NULL */
  /* The contact history (sapb_contact_history_update), run by this launch
   * between the contact scatter and the free motion, on this launch's slots
   * and contact buffer: its num_envs, max_contacts, num_flat, contact_count,
   * contact_source and flat_* fields are ignored (filled here), the others
   * are as sapb_contact_history documents.  NULL: no history. */
  const struct sapb_contact_history* history;
  /* [W][n] the candidate start v* + A^-1 J^T gamma_start of each world
   * (gamma_start of the history by this launch's slots; FP64, through the
   * free motion's own LDL^T), or NULL.  Dense layout; needs history with
   * gamma_start. */
  double* v_start;
  /* [W][dofs_per_world] the start-of-step velocities in the solve's slots
   * (uneven batches: the solve's v0), or NULL */
  double* qd_slots;
} sapb_prepare_outputs;

/* Device workspace bytes of sapb_free_motion_contacts. */
size_t sapb_prepare_workspace_size(const sapb_model_desc* model, int32_t max_contacts);

/* Free motion and contact Jacobian of every world: FK, bias forces, RNEA,
 * the mass matrix and v* (SapFreeMotion.compute, sim/free_motion.py:2180-2208
 * with _compute_sap_core :2094-2178), then the per-world contact slots, frames,
 * phi0, combined materials, Jacobian rows and weights
 * (SapContactJacobian.compute, sim/contact_jacobian.py:1649-1985).  Slots are
 * claimed atomically like the reference's scatter (:470), then ordered by
 * flat contact index within each world, so an untruncated world's slot order
 * is the flat buffer's.  At most 64 bodies and 128 DOFs per world
 * (SAPB_ERR_UNSUPPORTED otherwise); with opts->tree_blocked, worlds of up
 * to 64 free bodies (384 DOFs) in the tree-blocked layout. */
int32_t sapb_free_motion_contacts(const sapb_model_desc* model, const sapb_step_inputs* in,
                                  const sapb_prepare_options* opts, const sapb_prepare_outputs* out,
                                  void* workspace, size_t workspace_bytes, void* stream);

#define SAPB_INTEGRATE_SAP_EULER 0
#define SAPB_INTEGRATE_MIDPOINT 1

/* Position integration q_{n+1} from SAP-order velocities (FP64 state),
 * replaces _integrate_generalized_positions_{sap_euler,midpoint}_f64
 * (sim/solver_sap.py:288-733, driven by :1267-1386).  v_prev is the
 * start-of-step velocity (midpoint only). */
int32_t sapb_integrate_positions(const sapb_model_desc* model, const double* joint_q_in, const double* v_prev,
                                 const double* v_new, const double* dt, int32_t mode, double* joint_q_out,
                                 void* stream);

/* The step's tail in one launch (the integrators above, the public output
 * of sim/solver_sap.py:1467-1469 with sim/sap_helpers.py:1711-1760 and the
 * forward kinematics of sim/sap_kinematics.py:85-229): one CTA per world
 * writes every joint's new coordinates (fixed joints copy theirs), the new
 * velocities in SAP or public order, and optionally the body poses and
 * public body velocities of the new public coordinates.  Replaces
 * sapb_integrate_positions + copies + sapb_sap_to_public_velocity +
 * sapb_eval_fk, with the same arithmetic. */
typedef struct sapb_step_tail {
  const double* joint_q_in;         /* [coords] start-of-step coordinates */
  const double* v_prev;             /* [dofs] start-of-step velocity (midpoint only; SAP order) */
  const double* v_new;              /* [dofs] the solve's velocity (SAP order) */
  const double* dt;                 /* [W] */
  int32_t mode;                     /* SAPB_INTEGRATE_SAP_EULER / _MIDPOINT */
  int32_t qd_public;                /* nonzero: joint_qd_out in public order (at the new coordinates) */
  double* joint_q_out;              /* [coords], must not alias joint_q_in */
  double* joint_qd_out;             /* [dofs] or NULL */
  double* body_q_out;               /* [B][7] or NULL: forward kinematics of the new coordinates */
  double* body_qd_out;              /* [B][6] or NULL: public body velocities [v; w] (needs qd_public
                                     * and joint_qd_out) */
} sapb_step_tail;

int32_t sapb_step_tail_launch(const sapb_model_desc* model, const sapb_step_tail* tail, void* stream);

/* ---- contact history ------------------------------------------------------
 * Impulses carried from one step's contact slots to the next step's by
 * contact identity (no counterpart in the reference, which warm-starts from
 * the previous velocity only): a contact is the same if its shape pair
 * matches and its shape1 witness point in shape1's body frame (the stable
 * feature of every primitive pair: sphere centre, box corner) is the mutually
 * nearest among the pair's contacts, looked for within 64 slots of its own.
 * Slots shift when contacts appear or vanish; with an unchanged contact
 * buffer every slot maps to itself.  One CTA per world; the keys are
 * updated in place (this step's replace the previous step's).
 *
 * Start impulses (`order` 2 or 3): along each contact's identity the
 * history keeps the impulses of up to `order` past steps, and the start is
 * their polynomial extrapolation to this step -- 2 g1 - g2 from two,
 * 3 g1 - 3 g2 + g3 from three (g1 the last solve's impulse, g2 the one
 * before, g3 the one before that), the carried g1 from one, zero for a new
 * contact.  Impulses of a persistent contact change smoothly from step to
 * step, so the extrapolation lands nearer this step's solution than g1;
 * the solve compares the start's cost with the plain start's anyway.  With
 * order 2 or 3, gamma_hist and has_history are in/out (the previous call's
 * outputs, by the previous slots) and must persist between calls. */
typedef struct sapb_contact_history {
  int32_t num_envs;
  int32_t max_contacts;             /* C */
  int32_t num_flat;                 /* length of the flat contact arrays */
  const int32_t* contact_count;     /* [W] this step's contacts per world (clamped to C) */
  const int32_t* contact_source;    /* [W][C] flat index of each slot (sapb_prepare_outputs) */
  const int32_t* flat_shape0;       /* [N] */
  const int32_t* flat_shape1;       /* [N] */
  const double* flat_point1;        /* [N][3] shape1 witness in its body frame */
  int32_t* key_shape;               /* [W][C][2] in: the previous step's keys; out: this step's */
  double* key_point;                /* [W][C][3] */
  int32_t* key_count;               /* [W] in: previous counts (0 before the first step); out: this step's */
  const double* gamma_prev;         /* [W][C][3] the previous step's impulses by its slots */
  double* gamma_hist;               /* [W][C][3] out: carried impulses g1 (0 for new contacts); order >= 2: in */
  int32_t* has_history;             /* [W][C] out: past impulses known for the slot's contact, 1..order (1 with
                                     * order <= 1), 0 new or empty slot; order >= 2: in */
  int32_t order;                    /* 0 or 1: carried impulses; 2: linear extrapolation; 3: quadratic */
  double* gamma_older;              /* [W][C][3] order 3: in/out g2 by slot (the impulses two solves back) */
  double* gamma_start;              /* [W][C][3] out: the start impulses (NULL: not written) */
} sapb_contact_history;

int32_t sapb_contact_history_update(const sapb_contact_history* hist, void* stream);

/* ---- the whole step behind a handle -----------------------------------------
 * SolverSAP (sim/solver_sap.py:736-1512) as a C API: sapb_create allocates
 * every work buffer (SolverSAP.__init__, :749-968); sapb_step runs one step
 * (SolverSAP.step, :1388-1494) -- free motion and contact rows, the contact
 * solve warm-started from the previous solution, position integration --
 * on `stream`, without host synchronisation and without allocating, so a
 * caller may capture it in a CUDA graph; sapb_get_status reads the per-world
 * solve status; sapb_destroy frees the buffers.  SAP-order state (the public
 * boundary is sapb_public_to_sap / sapb_sap_to_public_velocity / sapb_eval_fk). */
typedef struct sapb_handle sapb_handle;

#define SAPB_WARM_START_PREVIOUS_VELOCITY 0  /* the reference's: start from the last solution */
#define SAPB_WARM_START_PREVIOUS_IMPULSES 1  /* also try v* + A^-1 J^T gamma0, gamma0 the start impulses
                                               * of the contact history (candidate start) */
#define SAPB_WARM_START_LEARNED 2  /* the history's start, plus the network's impulses on new contacts
                                    * (sapb_step_options.network; SolverSAP(warm_start="learned")) */

struct sapb_step_network;
#define SAPB_WORK_ORDER_INDEX 0
#define SAPB_WORK_ORDER_PREVIOUS_ITERATIONS 1  /* most Newton iterations of the last step first */

typedef struct sapb_step_options {
  sapb_prepare_options prepare;     /* max_contacts, weight / point modes, fallbacks; tree_blocked: the
                                     * tree-blocked layout and solve (the trees are world 0's articulations,
                                     * tree_dofs 0: the smallest block holding them) */
  sapb_solve_options solve;         /* the contact solve's options (line search, precisions, tolerances) */
  int32_t position_integration;     /* SAPB_INTEGRATE_SAP_EULER / SAPB_INTEGRATE_MIDPOINT */
  int32_t warm_start;               /* SAPB_WARM_START_* */
  int32_t work_order;               /* SAPB_WORK_ORDER_* */
  int32_t impulse_history;          /* previous impulses: the contact history's order (1 carried, 2 linear,
                                     * 3 quadratic extrapolation; 0 = 3) */
  const struct sapb_step_network* network;  /* SAPB_WARM_START_LEARNED: the network (kept alive by the caller
                                             * for the handle's life), else NULL */
} sapb_step_options;

/* One step's device arrays: the start-of-step state, control and contacts
 * (in), the drive / limit model (NULL: none; its joint_q is replaced by
 * in.joint_q) and the new state (out; q_out must not alias in.joint_q). */
typedef struct sapb_step_io {
  sapb_step_inputs in;
  const sapb_dof_terms* dof;
  double* joint_q_out;              /* [coords] */
  double* joint_qd_out;             /* [dofs] SAP order */
} sapb_step_io;

/* Fill the defaults of SolverSAP's keywords for a drake-preset step
 * (sim/solver_sap.py:749-791): 128 contact slots, armijo_decay, FP64,
 * sap_euler, previous-velocity warm start, work order by previous iterations,
 * impulse history of order 3. */
void sapb_step_options_default(sapb_step_options* opts);
/* Allocate the step's buffers for `model` (device arrays the caller keeps
 * alive while the handle lives); reads the model's index arrays once
 * (synchronous).  SAPB_ERR_UNSUPPORTED for shapes the on-chip solve cannot
 * hold. */
int32_t sapb_create(const sapb_model_desc* model, const sapb_step_options* opts, sapb_handle** out);
/* One step on `stream` (see above). */
int32_t sapb_step(sapb_handle* handle, const sapb_step_io* io, void* stream);
/* Copy the last step's per-world solve status (0, SAPB_LS_* or SAPB_WORLD_*),
 * convergence flags and Newton iterations into [W] arrays (host or device;
 * any may be NULL), asynchronously on `stream`. */
int32_t sapb_get_status(const sapb_handle* handle, int32_t* status, int32_t* converged, int32_t* newton_iterations,
                        void* stream);
/* Device pointers of the handle's solve outputs (SapContactSolveResult views,
 * sim/contact_solve.py:188-232): valid until sapb_destroy. */
int32_t sapb_step_solve_outputs(const sapb_handle* handle, sapb_solve_outputs* out);
void sapb_destroy(sapb_handle* handle);

/* The order in which the persistent solve should take the worlds next step:
 * by the last Newton iterations, most first, ties in index order (stable),
 * sorted on the device by one CTA (at most 32768 worlds).  No counterpart in
 * the reference (its solve has no work queue). */
int32_t sapb_world_order(const int32_t* newton_iterations, int32_t num_envs, int32_t* order, void* stream);

/* ---- public-order boundary ------------------------------------------------
 * Newton-style callers hold joint velocities / forces in the public order
 * (free and distance joints: [v_com; w] and [f; tau_com]) and body forces as
 * [f; tau] at the COM; the step runs in SAP order ([w; v_origin], body-origin
 * wrenches).  These restate the boundary of SolverSAP.step
 * (sim/solver_sap.py:1198-1261, 1467-1469).  All arrays FP64, device. */

/* Public -> SAP order (copy_public_to_sap_velocity_f64_from_joint_pose,
 * _copy_public_to_sap_force_kernel_f64_from_joint_pose and
 * _copy_public_body_force_to_sap_body_origin_kernel, sim/sap_helpers.py:
 * 1481-1622, 1811-2095).  joint_q [coords] gives the free joints' rotation;
 * body_q [B][7] the bodies' (for body forces).  Any of the three public
 * inputs may be NULL (its output is then not written). */
int32_t sapb_public_to_sap(const sapb_model_desc* model, const double* joint_q, const double* body_q,
                           const double* joint_qd_public, const double* joint_f_public,
                           const double* body_f_public, double* joint_qd_sap, double* joint_f_sap,
                           double* body_f_sap, void* stream);

/* SAP -> public joint velocities with the pose joint_q
 * (_copy_sap_to_public_velocity_f64_from_joint_pose, sim/sap_helpers.py:1711-1760). */
int32_t sapb_sap_to_public_velocity(const sapb_model_desc* model, const double* joint_q,
                                    const double* joint_qd_sap, double* joint_qd_public, void* stream);

/* Forward kinematics of public coordinates: body poses [B][7] and public body
 * velocities [B][6] ([v; w], may be NULL) articulation by articulation
 * (sap_eval_fk, sim/sap_kinematics.py:85-341; FP64 here, FP32 there). */
int32_t sapb_eval_fk(const sapb_model_desc* model, const double* joint_q, const double* joint_qd_public,
                     double* body_q, double* body_qd, void* stream);

/* ---- contact generation for primitive shapes ------------------------------
 * Planes, spheres and boxes: plane-sphere, plane-box (corners), sphere-sphere,
 * sphere-box (closest point), box-box (corners against faces, both ways; no
 * edge-edge).  Writes the flat contact buffer as the reference's
 * sap_write_contact does (sim/collision/pipeline.py:52-118): shape pair,
 * witness points in the body frames of their shapes (world frame for static
 * shapes), unit normal from shape0 to shape1, margins (a sphere's radius is
 * in its margin, its witness point the centre).  A covering of the synthetic
 * scenes' pairs, not the reference's general narrow phase (GJK / MPR,
 * meshes, SDFs, contact reduction).  Deterministic order: pairs by world,
 * then shape index, contacts of a pair in a fixed order. */
#define SAPB_SHAPE_PLANE 0
#define SAPB_SHAPE_SPHERE 1
#define SAPB_SHAPE_BOX 2

typedef struct sapb_collision_shapes {
  int32_t num_worlds;
  int32_t shapes_per_world;         /* local shapes, contiguous per world */
  int32_t num_global_shapes;        /* static shapes after all worlds' shapes, met by every world (the ground) */
  const int32_t* shape_type;        /* [S] SAPB_SHAPE_* */
  const double* shape_scale;        /* [S][3] sphere radius in [0]; box half extents */
  const double* shape_X_bs;         /* [S][7] shape frame in its body frame (world frame for static shapes);
                                       a plane is z = 0 of its frame with normal +z */
  const int32_t* shape_body;        /* [S] body, -1 static */
  const double* shape_margin;       /* [S] or NULL */
  double gap;                       /* emit contacts whose signed distance is below gap */
  /* [S] collision groups or NULL (every pair is tested): the rule of
   * sap_test_group_pair (sim/collision/broad_phase_common.py:133-150) --
   * 0 meets nothing, a positive group meets itself and negative groups, a
   * negative group meets every group but itself. */
  const int32_t* shape_collision_group;
} sapb_collision_shapes;

typedef struct sapb_contact_outputs {
  int32_t capacity;
  int32_t* count;                   /* [1] contacts found (may exceed capacity: then only the first
                                       capacity, in pair order, are written; INT32_MAX saturates) */
  int32_t* shape0;                  /* [capacity] */
  int32_t* shape1;
  double* point0;                   /* [capacity][3] */
  double* point1;
  double* normal;
  double* margin0;                  /* [capacity] */
  double* margin1;
} sapb_contact_outputs;

/* Device workspace bytes of sapb_generate_contacts. */
size_t sapb_contacts_workspace_size(const sapb_collision_shapes* shapes);

/* Contacts of every world at the body poses body_q [B][7] (device), in the
 * format the reference's collision pipeline writes with sap_write_contact
 * (sim/collision/pipeline.py:52-118); the primitive pairs of
 * sim/collision/primitive.py (plane-sphere :89-97, sphere-sphere :99-130,
 * plane-box :354-428, sphere-box :1150-1205; box-box as vertex-face). */
int32_t sapb_generate_contacts(const sapb_collision_shapes* shapes, const double* body_q,
                               const sapb_contact_outputs* out, void* workspace, size_t workspace_bytes,
                               void* stream);

/* Resident CTAs per SM the dense contact solve can hold for this world shape
 * (the upper end of sapb_solve_options.ctas_per_sm), or a negative status. */
int32_t sapb_contact_solve_occupancy(int32_t dof_per_env, int32_t max_contacts, int32_t hessian_precision,
                                     int32_t line_search_variant);

/* The same for a threads_per_cta choice of sapb_solve_options (0, 128 or
 * 256), or a negative status. */
int32_t sapb_contact_solve_occupancy_threads(int32_t dof_per_env, int32_t max_contacts, int32_t hessian_precision,
                                             int32_t line_search_variant, int32_t threads_per_cta);

/* The LDL^T column-block widths the dense solve is built with for worlds of
 * dof_per_env DOFs (the first is the default), written to widths (at most
 * capacity); returns their count.  The autotuner's compile-time variants. */
int32_t sapb_contact_solve_ldlt_blocks(int32_t dof_per_env, int32_t* widths, int32_t capacity);

/* Fill the reference defaults of SapContactSolve for a line-search variant.
 * Replaces the Python defaults of solve(), sim/contact_solve.py:6129-6182. */
void sapb_solve_options_default(sapb_solve_options* opts, int32_t line_search_variant);

/* Measured fused multiply-add rate of the current GPU in the given precision
 * (SAPB_FP64 / SAPB_FP32), in FLOP/s: eight independent FMA chains per
 * thread, 2048 threads per SM, `iters` steps each, timed with CUDA events on
 * `stream` after a warm-up launch (synchronises the stream).  The FP64 figure
 * is the denominator of the contact solve's FP64-pipe fraction.  No
 * counterpart in the reference (a measurement of this build's roofline). */
int32_t sapb_measure_fma_rate(int32_t precision, int32_t iters, double* flops_per_s, void* stream);

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

/* ---- worlds of many small trees ---------------------------------------------
 * The stage-2 problem in a tree-blocked layout, for worlds made of up to 64
 * trees of at most tree_dofs DOFs each (for example 64 free bodies: 384
 * DOFs; or a 7-DOF arm among free boxes).  The reference keeps such worlds
 * dense: A_env with its zero blocks between trees
 * (sim/contact_jacobian.py:110-150) and J rows over all n DOFs (:404-562).
 * Here A is its diagonal tree blocks and each contact row holds the columns
 * of the (at most two) trees the contact touches.  Trees are contiguous in
 * the world's DOF order: tree t holds DOFs tree_dof_start[t] ..
 * tree_dof_start[t+1]-1 (NULL: DOFs t * tree_dofs .. , every tree full).
 * A tree's block and row columns are NB = tree_dofs wide; a tree with fewer
 * DOFs is padded with the identity in its block and zero columns, padding
 * the solve keeps to itself (the per-DOF vectors are the world's own DOFs).
 * A contact whose two sides lie on one tree is given as one side with the
 * summed columns.  Drive and limit terms through `dof` (optional). */
typedef struct sapb_blocked_problem {
  int32_t num_envs;
  int32_t trees_per_env;          /* T <= 64 */
  int32_t tree_dofs;              /* NB: a block size sapb_blocked_tree_block returns (6: a free body) */
  int32_t max_contacts;           /* C: per-world slot capacity */
  const int32_t* contact_count;   /* [E] contacts per world (clamped to C) */
  const double* tree_mass;        /* [E,T,NB,NB] diagonal blocks of A */
  const double* jacobian;         /* [E,C,3,2*NB]: columns [0,NB) on contact_tree[..,0], [NB,2NB) on [..,1] */
  const int32_t* contact_tree;    /* [E,C,2] tree of each side, -1: none (static) */
  const double* phi0;             /* [E,C] */
  const double* w_eff;            /* [E,C] */
  const double* mu;               /* [E,C] */
  const double* stiffness;        /* [E,C] */
  const double* tau_d;            /* [E,C] or NULL -> options.contact_tau_d */
  const double* v_star;           /* [E*n] free-motion velocity (n = dofs_per_world) */
  const double* v0;               /* [E*n] start-of-step velocity */
  double* v_guess;                /* [E*n] warm start in / seeded velocity out, or NULL */
  const int32_t* v_guess_active;  /* [1] nonzero: start from v_guess; NULL: never */
  const double* dt;               /* [E] */
  const int32_t* world_order;     /* [E] order of the persistent queue, or NULL */
  /* A candidate start (no counterpart in the reference): starting impulses
   * [E,C,3] (for example the previous step's), or NULL.  The solve forms
   * v_c = v* + A^-1 J^T gamma0 tree by tree (A is block diagonal) and starts
   * Newton from v_c when its cost is below the plain start's (v_guess or
   * v0); warm_start_accepted reports 1 then.  gamma0_count must be <= 1. */
  const double* gamma0;
  int32_t gamma0_count;
  /* Trees of different sizes: [T+1] first DOF of each tree in the world
   * (device, the same for every world; increasing, each tree at most
   * tree_dofs DOFs, tree_dof_start[T] = dofs_per_world), or NULL. */
  const int32_t* tree_dof_start;
  int32_t dofs_per_world;         /* n; 0: T * tree_dofs */
  /* Drive and limit terms (sim/contact_solve.py:490-683), the per-DOF arrays
   * in the [E*n] layout of the world's own DOFs, or NULL: none. */
  const sapb_dof_terms* dof;
} sapb_blocked_problem;

/* The block size NB the blocked solve is built with for trees of up to
 * tree_dofs DOFs: the smallest of 6, 7 and 12 that holds them (0: none). */
int32_t sapb_blocked_tree_block(int32_t tree_dofs);

/* Off-diagonal factor blocks one world of this shape can hold on chip
 * without drive / limit terms (with them, their 11 vectors per DOF take
 * room first; 0: the shape does not fit or tree_dofs is not a built block
 * size).  A world whose
 * elimination (rounds of independent minimum-degree trees, with fill) needs
 * more gets the per-world status SAPB_WORLD_FACTOR_CAPACITY. */
int32_t sapb_blocked_fill_capacity(int32_t trees_per_env, int32_t tree_dofs, int32_t max_contacts,
                                   int32_t hessian_precision);

/* Bytes of device workspace sapb_blocked_contact_solve needs. */
size_t sapb_blocked_solve_workspace_size(int32_t num_envs, int32_t trees_per_env, int32_t max_contacts);

/* The solve of sapb_contact_solve on the tree-blocked layout: the same
 * Newton loop, line searches and convergence test (sim/contact_solve.py:
 * 6129-6285), the Newton Hessian block sparse (a block per tree and per
 * pair of trees in contact) and factored by a block LDL^T in
 * hessian_precision.  Outputs as sapb_contact_solve (v in the tree-by-tree
 * DOF order; warm_start_accepted 0 plain start, 1 the gamma0 candidate). */
int32_t sapb_blocked_contact_solve(const sapb_blocked_problem* problem, const sapb_solve_options* opts,
                                   const sapb_solve_outputs* out, void* workspace, size_t workspace_bytes,
                                   void* stream);

/* Gather a dense problem whose worlds are trees_per_env trees into the
 * blocked layout: tree_mass [E,T,NB,NB], jacobian [E,C,3,2NB], contact_tree
 * [E,C,2] (device pointers).  tree_dof_start (device [T+1], or NULL: trees of
 * tree_dofs DOFs each) as in sapb_blocked_problem; a body's tree is the one
 * holding body_dof_start of the body.  The other blocked fields alias the
 * dense ones. */
int32_t sapb_dense_to_blocked(const sapb_contact_problem* dense, int32_t trees_per_env, int32_t tree_dofs,
                              const int32_t* tree_dof_start, double* tree_mass, double* jacobian,
                              int32_t* contact_tree, void* stream);

/* Last CUDA error string seen by the library on this thread ("" if none). */
const char* sapb_last_error(void);

/* ---- learned warm start -----------------------------------------------------
 * A per-contact MLP 12 -> 128 -> 128 -> 128 -> 3 (GELU, tanh form), BF16
 * weights and activations, FP32 accumulation, run and trained on the tensor
 * cores (tcgen05) by the kernels below.  No counterpart in the reference,
 * whose only warm start is the previous step's velocity
 * (sim/solver_sap.py:1441-1451).
 *
 * Inputs of a contact slot (raw, before normalisation): phi0; J_c v* in the
 * contact frame (t1, t2, n); the world-up component of the contact normal;
 * mu; log10(stiffness); tau_d; dt; w_eff * gamma_prev (t1, t2, n).  The
 * output y maps to a correction u = y * output_scale + output_shift
 * (velocity units) of SAP's unprojected impulse y0 = gamma_prev + u / w_eff
 * (gamma_prev = 0 when not given); gamma0 is the regularized projection of
 * y0 (the impulse SAP assigns to the contact velocity vhat - R y0). */
#define SAPB_MLP_INPUTS 12
#define SAPB_MLP_INPUTS_PADDED 16
#define SAPB_MLP_HIDDEN 128
#define SAPB_MLP_OUTPUTS 3
/* FP32 master parameters W1[128][12] b1[128] W2[128][128] b2 W3[128][128] b3
 * W4[3][128] b4[3]; the forward reads BF16 operand images (packed) and FP32
 * biases made from them by sapb_mlp_pack / sapb_mlp_adam. */
#define SAPB_MLP_PARAM_COUNT 35075
#define SAPB_MLP_PACKED_COUNT 35200
#define SAPB_MLP_BIAS_COUNT 387

typedef struct sapb_warmstart_norm {
  float feature_mean[SAPB_MLP_INPUTS];
  float feature_inv_std[SAPB_MLP_INPUTS];
  float output_scale[SAPB_MLP_OUTPUTS];
  float output_shift[SAPB_MLP_OUTPUTS];
} sapb_warmstart_norm;

/* The warm-start network of the C step handle (SAPB_WARM_START_LEARNED):
 * its device weights, the normalisation, and the two tau_d fallbacks the
 * Python LearnedWarmStart uses (features: its tau_fallback; the impulse
 * map's regularization: contact_tau_d, with contact_beta / contact_sigma
 * those of the step's solve options). */
typedef struct sapb_step_network {
  const uint16_t* packed;           /* SAPB_MLP_PACKED_COUNT BF16 weights, the forward's layout (device) */
  const float* bias;                /* SAPB_MLP_BIAS_COUNT (device) */
  sapb_warmstart_norm norm;
  double feature_tau_d;
  double impulse_tau_d;
} sapb_step_network;

/* Saved forward state of one training batch of `rows` rows. */
typedef struct sapb_mlp_train_buffers {
  uint16_t* act;  /* BF16 [act_elems] hidden activations (tile images) */
  float* pre;     /* FP32 [pre_elems] pre-activations */
  float* dy;      /* FP32 [rows,3] dL/dy of the mean squared error */
  float* loss;    /* FP32 [1] sum of squared errors, accumulated */
} sapb_mlp_train_buffers;

typedef struct sapb_adam_options {
  float lr, beta1, beta2, eps, weight_decay;  /* decoupled weight decay */
} sapb_adam_options;

int32_t sapb_mlp_param_count(void);
int32_t sapb_mlp_packed_count(void);
int32_t sapb_mlp_bias_count(void);
int32_t sapb_mlp_train_buffer_sizes(int32_t rows, int64_t* act_elems, int64_t* pre_elems);
/* params [PARAM_COUNT] -> packed [PACKED_COUNT] (BF16 bits), bias [BIAS_COUNT]. */
int32_t sapb_mlp_pack(const float* params, uint16_t* packed, float* bias, void* stream);
/* y[rows,3] = MLP(x), x [rows,16] BF16 (16-byte aligned, columns 12..15 zero). */
int32_t sapb_mlp_forward(const uint16_t* packed, const float* bias, const uint16_t* x, int32_t rows, float* y,
                         void* stream);
/* sapb_mlp_forward over the 128-row tiles whose tile_active[tile] is nonzero
 * only (the other tiles' rows of y are not written). */
int32_t sapb_mlp_forward_tiles(const uint16_t* packed, const float* bias, const uint16_t* x, int32_t rows, float* y,
                               const int32_t* tile_active, void* stream);
/* Training forward: saves buf->act / buf->pre, writes buf->dy and adds the
 * squared error to buf->loss; y optional. */
int32_t sapb_mlp_forward_train(const uint16_t* packed, const float* bias, const uint16_t* x, const float* target,
                               int32_t rows, const sapb_mlp_train_buffers* buf, float* y, void* stream);
/* Adds dL/dparams (master layout) of the batch to grad. */
int32_t sapb_mlp_backward(const uint16_t* packed, const uint16_t* x, int32_t rows, const sapb_mlp_train_buffers* buf,
                          float* grad, void* stream);
/* One Adam step (step >= 1) on params with moments m, v; refreshes packed/bias. */
int32_t sapb_mlp_adam(float* params, const float* grad, float* m, float* v, const sapb_adam_options* opt,
                      int32_t step, uint16_t* packed, float* bias, void* stream);
/* Reads and clears the MLP kernels' timeout flag (synchronises `stream`):
 * SAPB_OK or SAPB_ERR_TIMEOUT. */
int32_t sapb_mlp_error(void* stream);
/* Failure-detection hooks of the MLP kernels (no counterpart in the
 * reference): every mbarrier wait of the forward / backward kernels gives up
 * after wait_polls polls (0: the default bound of 2^22 polls), after which
 * the kernel sets the timeout flag, waits (bounded) for any commit still in
 * flight, frees its tensor memory and exits; with drop_first_commit each
 * forward CTA issues no MMA commit for its first layer, so that wait cannot
 * complete (a deterministic timeout for tests).  Applies to later launches. */
int32_t sapb_mlp_test_hooks(int32_t wait_polls, int32_t drop_first_commit);
/* Per-slot network inputs of a stage-2 problem: normalised BF16 rows
 * features [E*C,16] and/or raw FP32 rows raw [E*C,12]; dead slots are zero.
 * normal_up [E,C] (NULL: 1), gamma_prev [E,C,3] (NULL: 0), vc_star [E,C,3]
 * the free-motion contact velocities J_c v* (NULL: formed from J and v*). */
int32_t sapb_warmstart_features(const sapb_contact_problem* problem, const double* normal_up,
                                const double* gamma_prev, const double* vc_star,
                                const sapb_warmstart_norm* norm, double tau_fallback, uint16_t* features,
                                float* raw, void* stream);
/* Per tile of 128 slot rows (E*C rows, world-major): 1 if a live slot has no
 * history (has_history [E,C] zero or NULL), i.e. the network has a row to
 * predict there; for sapb_mlp_forward_tiles. */
int32_t sapb_warmstart_active_tiles(const sapb_contact_problem* problem, const int32_t* has_history,
                                    int32_t* tile_active, void* stream);
/* gamma0 [E,C,3] from the network output mlp_out [E*C,3] and the previous
 * step's impulses gamma_prev [E,C,3] (NULL: 0); opts supplies the
 * regularization (contact_beta, contact_sigma, contact_tau_d fallback).
 * With has_history [E,C] (NULL: none), slots whose contact has history keep
 * gamma_prev and the network's prediction serves the others. */
int32_t sapb_warmstart_impulses(const sapb_contact_problem* problem, const float* mlp_out,
                                const double* gamma_prev, const int32_t* has_history,
                                const sapb_warmstart_norm* norm, const sapb_solve_options* opts, double* gamma0,
                                void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SAPB_H */
