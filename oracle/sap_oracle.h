/*
 * sap_oracle.h -- CPU FP64 restatement of the reference's SAP contact solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA path: it
 * may be called only by tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg / reference arm of bench.py.  The product never links or calls it.
 *
 * Parity status: the reference (mardigiorgio/sap_warp) is Python + NVIDIA
 * Warp and ships no tests, fixtures or golden vectors, and Warp cannot be
 * imported in this environment, so no output of the reference itself pins this
 * restatement.  It is pinned only to analytic known-answer cases derived from
 * the reference's formulas (tests/golden/known_answers.json), so parity is
 * "partially pinned".
 *
 * Each function cites the reference file:line it restates.
 */
#ifndef SAP_ORACLE_H
#define SAP_ORACLE_H

#include "../include/sapb.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Per-contact projection result (sim/contact_solve.py:743-921). */
typedef struct sapo_projection {
  double gamma[3];
  double g[9];      /* row-major 3x3 */
  double y[3];
  double rt, rn, cost;
  int32_t mode;
} sapo_projection;

/* Project one contact given its contact velocity vc. */
void sapo_project_contact(const double vc[3], double phi0, double w_eff, double mu, double k, double tau_d,
                          double beta, double sigma, double dt, int want_hessian, sapo_projection* out);

/* Effective PD gains (sim/sap_helpers.py:2305-2341). out = {kp_eff, kd_eff}. */
void sapo_effective_pd_gains(double kp, double kd, double dt, double delassus, double out[2]);

/* Clamp helpers (sim/sap_helpers.py:2251-2276). */
double sapo_clamp(double x, double limit);
double sapo_clamp_derivative(double x, double limit);
double sapo_clamp_antiderivative(double x, double limit);

/* Whole contact solve over all worlds with OpenMP (host pointers).
 * Restates SapContactSolve.solve (sim/contact_solve.py:6129-6285).
 * num_threads <= 0: OpenMP default.  Returns SAPB_OK or SAPB_ERR_INVALID_ARGUMENT. */
int32_t sapo_contact_solve(const sapb_contact_problem* problem, const sapb_solve_options* opts,
                           const sapb_solve_outputs* out, int32_t num_threads);

/* Dense FP64 Cholesky in place (lower), returns 0 or the failing column + 1.
 * Stands in for BlockCholeskySolverBatched (sim/blocked_cholesky.py:725-901). */
int32_t sapo_cholesky(double* a, int32_t n);

void sapo_solve_options_default(sapb_solve_options* opts, int32_t line_search_variant);

/* Free motion, contact rows and weights of every world (host pointers; the
 * same structs as sapb_free_motion_contacts), contacts in flat order per
 * world.  Restates SapFreeMotion.compute and SapContactJacobian.compute
 * (sim/free_motion.py:1804-2178, sim/contact_jacobian.py:153-562,
 * 1649-1985) with the reference's body-origin recursions.  OpenMP over
 * worlds; num_threads <= 0: OpenMP default. */
int32_t sapo_free_motion_contacts(const sapb_model_desc* model, const sapb_step_inputs* in,
                                  const sapb_prepare_options* opts, const sapb_prepare_outputs* out,
                                  int32_t num_threads);

/* Position integration (sim/solver_sap.py:144-733), host pointers. */
int32_t sapo_integrate_positions(const sapb_model_desc* model, const double* q_in, const double* v_prev,
                                 const double* v_new, const double* dt, int32_t mode, double* q_out);

#ifdef __cplusplus
}
#endif

#endif
