/*
 * sap_oracle.c -- CPU FP64 restatement of the reference's SAP contact solve.
 *
 * TEST INFRASTRUCTURE ONLY (see sap_oracle.h): the checker for the CUDA path,
 * never part of the product.  Parity partially pinned: analytic known-answer
 * cases only, no reference-run vectors exist (the reference needs Warp).
 *
 * The control flow restates the reference's batched Warp kernels world by
 * world.  The reference runs every world in lock-step through a device-side
 * conditional CUDA graph, but every kernel is indexed by world and the loop
 * counters it shares are equal for all active worlds, so a per-world loop
 * gives the same arithmetic.
 */
#include "sap_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Constants of sim/contact_solve.py:46-58. */
#define SAPO_PI 3.141592653589793
#define SAPO_SOFT_NORM_TOL 1.0e-7
#define SAPO_PD_BETA 0.1
#define SAPO_LIMIT_BETA 0.1
#define SAPO_LIMIT_WINDOW_FACTOR 2.0
#define SAPO_EXACT_ALPHA_MAX 1.5
#define SAPO_EXACT_F_TOL 1.0e-8

static inline double dmax(double a, double b) { return a > b ? a : b; }
static inline double dmin(double a, double b) { return a < b ? a : b; }

void sapo_solve_options_default(sapb_solve_options* o, int32_t variant) {
  /* SapContactSolve.__init__ / solve defaults, sim/contact_solve.py:3299-3316, 6129-6182. */
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

/* sim/sap_helpers.py:2251-2276 */
double sapo_clamp(double x, double limit) {
  if (limit <= 0.0 || !isfinite(limit)) return x;
  return dmax(-limit, dmin(limit, x));
}
double sapo_clamp_derivative(double x, double limit) {
  if (limit <= 0.0 || !isfinite(limit)) return 1.0;
  if (-limit <= x && x <= limit) return 1.0;
  return 0.0;
}
double sapo_clamp_antiderivative(double x, double limit) {
  if (limit <= 0.0 || !isfinite(limit)) return 0.5 * x * x;
  if (x < -limit) return -limit * (x + 0.5 * limit);
  if (x <= limit) return 0.5 * x * x;
  return limit * (x - 0.5 * limit);
}

/* sim/sap_helpers.py:2305-2341 */
void sapo_effective_pd_gains(double kp, double kd, double dt, double delassus, double out[2]) {
  out[0] = 0.0;
  out[1] = 0.0;
  if (kp <= 0.0 && kd <= 0.0) return;
  const double beta = SAPO_PD_BETA;
  const double beta_factor = beta * beta / (4.0 * SAPO_PI * SAPO_PI);
  const double r_nr = beta_factor * dmax(delassus, 1.0e-12);
  const double common = dt * kp + kd;
  if (common <= 0.0) return;
  const double r = 1.0 / (dt * common);
  if (r >= r_nr) {
    out[0] = kp;
    out[1] = kd;
    return;
  }
  double kp_eff = kp, kd_eff = kd;
  if (dt * kp > kd && kp > 0.0) {
    const double tau = kd / kp;
    kp_eff = 1.0 / (dt * (dt + tau) * r_nr);
    kd_eff = tau * kp_eff;
  } else if (kd > 0.0) {
    const double tau_inv = kp / kd;
    kd_eff = 1.0 / (dt * (1.0 + dt * tau_inv) * r_nr);
    kp_eff = tau_inv * kd_eff;
  } else {
    kp_eff = 1.0 / (dt * dt * r_nr);
    kd_eff = 0.0;
  }
  out[0] = kp_eff;
  out[1] = kd_eff;
}

/* Projection onto the regularized friction cone:
 * _projection_eval_contact_sap_batched sim/contact_solve.py:743-921 (gamma, G,
 * mode, cost) and its cost-only twin sim/sap_helpers.py:2381-2448. */
void sapo_project_contact(const double vc[3], double phi0, double w_eff, double mu, double k, double tau_d,
                          double beta, double sigma, double dt, int want_hessian, sapo_projection* p) {
  double wi = w_eff;
  if (wi < 1.0e-12 || !isfinite(wi)) wi = 1.0e-12;
  const double beta_factor = beta * beta / (4.0 * SAPO_PI * SAPO_PI);
  const double rn_hard = beta_factor * wi;
  double k_c = k;
  if (k_c <= 0.0 || !isfinite(k_c)) k_c = 1.0;
  const double tau_c = dmax(tau_d, 0.0);
  const double rn_soft = 1.0 / (dt * k_c * (dt + tau_c));
  double rn = dmax(rn_hard, rn_soft);
  double rt = sigma * wi;
  if (rt < 1.0e-30) rt = 1.0e-30;
  if (rn < 1.0e-30) rn = 1.0e-30;
  const double rt_inv = 1.0 / rt;
  const double rn_inv = 1.0 / rn;
  const double vhat_n = -phi0 / (dt + tau_c);
  const double y0 = -rt_inv * vc[0];
  const double y1 = -rt_inv * vc[1];
  const double y2 = rn_inv * (vhat_n - vc[2]);
  double m = mu;
  if (m < 0.0 || !isfinite(m)) m = 0.0;
  const double yr = sqrt(y0 * y0 + y1 * y1 + SAPO_SOFT_NORM_TOL * SAPO_SOFT_NORM_TOL);
  double tx = 0.0, ty = 0.0;
  if (yr > 0.0) {
    tx = y0 / yr;
    ty = y1 / yr;
  }
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  double G[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int32_t mode = SAPB_CONTACT_MODE_NONE;
  if (m <= 1.0e-12) {
    if (y2 > 0.0) {
      g2 = y2;
      G[8] = rn_inv;
      mode = SAPB_CONTACT_MODE_FRICTIONLESS;
    }
  } else {
    const double mu_tilde = m * sqrt(rt / rn);
    const double mu_hat = m * rt / rn;
    const double factor = 1.0 / (1.0 + mu_tilde * mu_tilde);
    if (yr <= m * y2) {
      g0 = y0;
      g1 = y1;
      g2 = y2;
      G[0] = rt_inv;
      G[4] = rt_inv;
      G[8] = rn_inv;
      mode = SAPB_CONTACT_MODE_STICTION;
    } else if ((-mu_hat * yr < y2) && (y2 < yr / m)) {
      const double gn = (y2 + mu_hat * yr) * factor;
      g0 = m * gn * tx;
      g1 = m * gn * ty;
      g2 = gn;
      if (want_hessian) {
        const double p00 = tx * tx, p01 = tx * ty, p10 = ty * tx, p11 = ty * ty;
        const double pp00 = 1.0 - p00, pp01 = -p01, pp10 = -p10, pp11 = 1.0 - p11;
        double gn_over_yr = 0.0;
        if (yr > 0.0) gn_over_yr = gn / yr;
        const double d00 = m * (gn_over_yr * pp00 + mu_hat * factor * p00);
        const double d01 = m * (gn_over_yr * pp01 + mu_hat * factor * p01);
        const double d10 = m * (gn_over_yr * pp10 + mu_hat * factor * p10);
        const double d11 = m * (gn_over_yr * pp11 + mu_hat * factor * p11);
        const double dn0 = m * factor * tx;
        const double dn1 = m * factor * ty;
        const double nd0 = mu_hat * factor * tx;
        const double nd1 = mu_hat * factor * ty;
        G[0] = d00 * rt_inv;
        G[1] = d01 * rt_inv;
        G[2] = dn0 * rn_inv;
        G[3] = d10 * rt_inv;
        G[4] = d11 * rt_inv;
        G[5] = dn1 * rn_inv;
        G[6] = nd0 * rt_inv;
        G[7] = nd1 * rt_inv;
        G[8] = factor * rn_inv;
      }
      mode = SAPB_CONTACT_MODE_SLIDING;
    }
  }
  p->gamma[0] = g0;
  p->gamma[1] = g1;
  p->gamma[2] = g2;
  memcpy(p->g, G, sizeof(G));
  p->y[0] = y0;
  p->y[1] = y1;
  p->y[2] = y2;
  p->rt = rt;
  p->rn = rn;
  p->cost = 0.5 * (rt * (g0 * g0 + g1 * g1) + rn * g2 * g2);
  p->mode = mode;
}

int32_t sapo_cholesky(double* a, int32_t n) {
  for (int32_t j = 0; j < n; ++j) {
    double d = a[j * n + j];
    for (int32_t k = 0; k < j; ++k) d -= a[j * n + k] * a[j * n + k];
    const double ljj = sqrt(d);
    a[j * n + j] = ljj;
    for (int32_t i = j + 1; i < n; ++i) {
      double s = a[i * n + j];
      for (int32_t k = 0; k < j; ++k) s -= a[i * n + k] * a[j * n + k];
      a[i * n + j] = s / ljj;
    }
    for (int32_t i = 0; i < j; ++i) a[i * n + j] = 0.0;
  }
  for (int32_t j = 0; j < n; ++j)
    if (!(a[j * n + j] > 0.0)) return j + 1;
  return 0;
}

static int32_t sapo_cholesky_f32(float* a, int32_t n) {
  for (int32_t j = 0; j < n; ++j) {
    float d = a[j * n + j];
    for (int32_t k = 0; k < j; ++k) d -= a[j * n + k] * a[j * n + k];
    const float ljj = sqrtf(d);
    a[j * n + j] = ljj;
    for (int32_t i = j + 1; i < n; ++i) {
      float s = a[i * n + j];
      for (int32_t k = 0; k < j; ++k) s -= a[i * n + k] * a[j * n + k];
      a[i * n + j] = s / ljj;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------- */
/* Per-world solver state.                                                   */

typedef struct world_ctx {
  int32_t n, count, C;
  const double* A;    /* n*n */
  const double* J;    /* C*3*n */
  const double *phi0, *w, *mu, *k, *tau; /* count */
  double tau_fallback;
  double dt, beta, sigma;
  int has_pd, has_lim;
  /* prepared per-DOF terms */
  double *v_star, *v, *a_inv_diag, *d_scale;
  int32_t* pd_active;
  double *pd_a, *pd_gain, *pd_limit;
  int32_t *lo_act, *up_act;
  double *lo_vhat, *up_vhat, *lo_r, *up_r, *lo_rinv, *up_rinv;
  int32_t* part;
  /* evaluation buffers at the current iterate */
  double *vc, *gamma, *ccost, *impulse, *grad, *dyn;
  double *pd_gamma, *pd_hdiag, *lim_grad, *lim_hdiag;
  double cost;
  /* scratch */
  double *H, *dv, *dp, *vt, *tmp_vc, *tmp_gamma, *tmp_imp, *G;
  double *t_pd_hdiag, *t_lim_hdiag, *t_G;
} world_ctx;

static double ctx_tau(const world_ctx* w, int32_t c) { return w->tau ? w->tau[c] : w->tau_fallback; }

/* vc = J_c v for every contact (the serial n-loop of :784-791). */
static void contact_velocities(const world_ctx* w, const double* v, double* vc) {
  const int32_t n = w->n;
  for (int32_t c = 0; c < w->count; ++c) {
    for (int32_t r = 0; r < 3; ++r) {
      const double* row = w->J + ((size_t)c * 3 + r) * n;
      double s = 0.0;
      for (int32_t j = 0; j < n; ++j) s += row[j] * v[j];
      vc[c * 3 + r] = s;
    }
  }
}

/* Evaluate the objective at v: contact gamma, costs, PD and limit terms, the
 * constraint impulse J^T gamma + PD + limits, grad = A(v-v*) - impulse and the
 * dynamics impulse A v.  Restates _evaluate_problem(defer_constraint_terms)
 * sim/contact_solve.py:4751-4966 with _projection_eval_contact_gamma (:973-1069),
 * the contact impulse tile kernel (:1245-1280) and the model-terms kernel
 * (:1493-1627).  If want_g != NULL also returns the contact G (the Hessian
 * variant :743-921). Outputs go to the given buffers; returns the total cost. */
static double evaluate(const world_ctx* w, const double* v, double* vc, double* gamma, double* ccost,
                       double* impulse, double* grad, double* dyn, double* pd_gamma, double* pd_hdiag,
                       double* lim_grad, double* lim_hdiag, double* want_g) {
  const int32_t n = w->n;
  double total = 0.0;
  contact_velocities(w, v, vc);
  for (int32_t c = 0; c < w->count; ++c) {
    sapo_projection p;
    sapo_project_contact(vc + 3 * c, w->phi0[c], w->w[c], w->mu[c], w->k[c], ctx_tau(w, c), w->beta, w->sigma,
                         w->dt, want_g != NULL, &p);
    gamma[3 * c + 0] = p.gamma[0];
    gamma[3 * c + 1] = p.gamma[1];
    gamma[3 * c + 2] = p.gamma[2];
    if (ccost) ccost[c] = p.cost;
    if (want_g) memcpy(want_g + 9 * c, p.g, sizeof(p.g));
    total += p.cost;
  }
  for (int32_t i = 0; i < n; ++i) {
    double s = 0.0;
    for (int32_t c = 0; c < w->count; ++c)
      for (int32_t r = 0; r < 3; ++r) s += w->J[((size_t)c * 3 + r) * n + i] * gamma[3 * c + r];
    impulse[i] = s;
  }
  for (int32_t i = 0; i < n; ++i) {
    const double* arow = w->A + (size_t)i * n;
    double a_res = 0.0, a_v = 0.0;
    for (int32_t j = 0; j < n; ++j) {
      a_res += arow[j] * (v[j] - w->v_star[j]);
      a_v += arow[j] * v[j];
    }
    const double vi = v[i];
    double model_cost = 0.5 * (vi - w->v_star[i]) * a_res;
    double pdg = 0.0, pdh = 0.0;
    if (w->has_pd && w->pd_active[i]) {
      const double gain = w->pd_gain[i];
      const double y = w->pd_a[i] - gain * vi;
      pdg = w->dt * sapo_clamp(y, w->pd_limit[i]);
      pdh = w->dt * gain * sapo_clamp_derivative(y, w->pd_limit[i]);
      double pdc = 0.0;
      if (gain > 0.0) pdc = (w->dt / gain) * sapo_clamp_antiderivative(y, w->pd_limit[i]);
      model_cost += pdc;
    }
    double lg = 0.0, lh = 0.0, lc = 0.0;
    if (w->has_lim) {
      if (w->lo_act[i]) {
        const double g = w->lo_rinv[i] * (w->lo_vhat[i] - vi);
        if (g > 0.0) {
          lg += g;
          lh += w->lo_rinv[i];
          lc += 0.5 * w->lo_r[i] * g * g;
        }
      }
      if (w->up_act[i]) {
        const double g = w->up_rinv[i] * (w->up_vhat[i] + vi);
        if (g > 0.0) {
          lg -= g;
          lh += w->up_rinv[i];
          lc += 0.5 * w->up_r[i] * g * g;
        }
      }
      model_cost += lc;
    }
    impulse[i] += pdg + lg;
    if (grad) grad[i] = a_res - impulse[i];
    if (dyn) dyn[i] = a_v;
    if (pd_gamma) pd_gamma[i] = pdg;
    if (pd_hdiag) pd_hdiag[i] = pdh;
    if (lim_grad) lim_grad[i] = lg;
    if (lim_hdiag) lim_hdiag[i] = lh;
    total += model_cost;
  }
  return total;
}

/* Regularizer (contact + PD + limit) cost at a trial velocity; the momentum
 * term comes from the line coefficients.  _replace_trial_cost_with_sap_line_search_cost
 * sim/contact_solve.py:2379-2420. */
static double trial_regularizer(const world_ctx* w, const double* vt, const double* vc_trial, double* gamma,
                                double* impulse, double* pd_hdiag, double* lim_hdiag, double* g_out) {
  const int32_t n = w->n;
  double reg = 0.0;
  for (int32_t c = 0; c < w->count; ++c) {
    sapo_projection p;
    sapo_project_contact(vc_trial + 3 * c, w->phi0[c], w->w[c], w->mu[c], w->k[c], ctx_tau(w, c), w->beta,
                         w->sigma, w->dt, g_out != NULL, &p);
    if (gamma) {
      gamma[3 * c + 0] = p.gamma[0];
      gamma[3 * c + 1] = p.gamma[1];
      gamma[3 * c + 2] = p.gamma[2];
    }
    if (g_out) memcpy(g_out + 9 * c, p.g, sizeof(p.g));
    reg += p.cost;
  }
  for (int32_t i = 0; i < n; ++i) {
    const double vi = vt[i];
    double pdg = 0.0, pdh = 0.0, lg = 0.0, lh = 0.0;
    if (w->has_pd && w->pd_active[i]) {
      const double gain = w->pd_gain[i];
      const double y = w->pd_a[i] - gain * vi;
      pdg = w->dt * sapo_clamp(y, w->pd_limit[i]);
      pdh = w->dt * gain * sapo_clamp_derivative(y, w->pd_limit[i]);
      if (gain > 0.0) reg += (w->dt / gain) * sapo_clamp_antiderivative(y, w->pd_limit[i]);
    }
    if (w->has_lim) {
      if (w->lo_act[i]) {
        const double g = w->lo_rinv[i] * (w->lo_vhat[i] - vi);
        if (g > 0.0) {
          lg += g;
          lh += w->lo_rinv[i];
          reg += 0.5 * w->lo_r[i] * g * g;
        }
      }
      if (w->up_act[i]) {
        const double g = w->up_rinv[i] * (w->up_vhat[i] + vi);
        if (g > 0.0) {
          lg -= g;
          lh += w->up_rinv[i];
          reg += 0.5 * w->up_r[i] * g * g;
        }
      }
    }
    if (impulse) {
      double s = 0.0;
      for (int32_t c = 0; c < w->count; ++c)
        for (int32_t r = 0; r < 3; ++r) s += w->J[((size_t)c * 3 + r) * n + i] * gamma[3 * c + r];
      impulse[i] = s + pdg + lg;
    }
    if (pd_hdiag) pd_hdiag[i] = pdh;
    if (lim_hdiag) lim_hdiag[i] = lh;
  }
  return reg;
}

/* Newton direction H dv = -grad with H = A + J^T G J + diag(PD + limit)
 * (_assemble_hessian_from_terms :4968-5009, contact GEMM :1334-1432, total
 * :1630-1654) and the padded masked Cholesky (:5069-5106). */
static void newton_direction(world_ctx* w, const sapb_solve_options* o) {
  const int32_t n = w->n;
  double* H = w->H;
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = 0; j < n; ++j) H[i * n + j] = w->A[i * n + j];
  /* contact part: sum_c J_c^T G_c J_c */
  for (int32_t c = 0; c < w->count; ++c) {
    const double* G = w->G + 9 * c;
    const double* J0 = w->J + ((size_t)c * 3 + 0) * n;
    const double* J1 = w->J + ((size_t)c * 3 + 1) * n;
    const double* J2 = w->J + ((size_t)c * 3 + 2) * n;
    for (int32_t j = 0; j < n; ++j) {
      const double gj0 = G[0] * J0[j] + G[1] * J1[j] + G[2] * J2[j];
      const double gj1 = G[3] * J0[j] + G[4] * J1[j] + G[5] * J2[j];
      const double gj2 = G[6] * J0[j] + G[7] * J1[j] + G[8] * J2[j];
      for (int32_t i = j; i < n; ++i) H[i * n + j] += J0[i] * gj0 + J1[i] * gj1 + J2[i] * gj2;
    }
  }
  for (int32_t j = 0; j < n; ++j)
    for (int32_t i = j + 1; i < n; ++i) H[j * n + i] = H[i * n + j];
  for (int32_t i = 0; i < n; ++i) {
    double d = 0.0;
    if (w->has_pd) d += w->pd_hdiag[i];
    if (w->has_lim) d += w->lim_hdiag[i];
    H[i * n + i] += d + o->diag_shift;
  }
  if (o->linear_solve_precision == SAPB_FP32) {
    float* Hf = (float*)malloc(sizeof(float) * (size_t)n * n);
    float* b = (float*)malloc(sizeof(float) * (size_t)n);
    for (int32_t i = 0; i < n * n; ++i) Hf[i] = (float)H[i];
    sapo_cholesky_f32(Hf, n);
    for (int32_t i = 0; i < n; ++i) b[i] = -(float)w->grad[i];
    for (int32_t i = 0; i < n; ++i) {
      float s = b[i];
      for (int32_t k = 0; k < i; ++k) s -= Hf[i * n + k] * b[k];
      b[i] = s / Hf[i * n + i];
    }
    for (int32_t i = n - 1; i >= 0; --i) {
      float s = b[i];
      for (int32_t k = i + 1; k < n; ++k) s -= Hf[k * n + i] * b[k];
      b[i] = s / Hf[i * n + i];
    }
    for (int32_t i = 0; i < n; ++i) w->dv[i] = (double)b[i];
    free(Hf);
    free(b);
    return;
  }
  sapo_cholesky(H, n);
  double* b = w->dv;
  for (int32_t i = 0; i < n; ++i) b[i] = -w->grad[i];
  for (int32_t i = 0; i < n; ++i) {
    double s = b[i];
    for (int32_t k = 0; k < i; ++k) s -= H[i * n + k] * b[k];
    b[i] = s / H[i * n + i];
  }
  for (int32_t i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int32_t k = i + 1; k < n; ++k) s -= H[k * n + i] * b[k];
    b[i] = s / H[i * n + i];
  }
}

typedef struct ls_result {
  int accepted;
  int status;
  int iterations;
  double alpha;
  double accepted_cost;
} ls_result;

/* Line coefficients: dp = A dv, dell0 = grad.dv, dell_a0 = dp.(v-v*),
 * d2ell_a = dv.dp (_compute_search_direction_data_serial_batched :2234-2263) and
 * the momentum cost 1/2 (v-v*)^T A (v-v*) (_compute_base_cost :1657-1692). */
static void line_coefficients(world_ctx* w, double* dell0, double* dell_a0, double* d2ell_a, double* mom0) {
  const int32_t n = w->n;
  double d0 = 0.0, da0 = 0.0, d2 = 0.0, m0 = 0.0;
  for (int32_t i = 0; i < n; ++i) {
    double acc = 0.0;
    for (int32_t j = 0; j < n; ++j) acc += w->A[i * n + j] * w->dv[j];
    w->dp[i] = acc;
    d0 += w->grad[i] * w->dv[i];
    da0 += acc * (w->v[i] - w->v_star[i]);
    d2 += w->dv[i] * acc;
  }
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = 0; j < n; ++j)
      m0 += 0.5 * (w->v[i] - w->v_star[i]) * w->A[i * n + j] * (w->v[j] - w->v_star[j]);
  *dell0 = d0;
  *dell_a0 = da0;
  *d2ell_a = d2;
  *mom0 = m0;
}

/* One trial: cost, derivative and (optionally) second derivative at alpha.
 * Trial cost: :2379-2420; derivative :2304-2321; second derivative :2324-2375. */
static double eval_trial(world_ctx* w, double alpha, double mom0, double dell_a0, double d2ell_a, double* deriv,
                         double* deriv2) {
  const int32_t n = w->n;
  for (int32_t i = 0; i < n; ++i) w->vt[i] = w->v[i] + alpha * w->dv[i];
  contact_velocities(w, w->vt, w->tmp_vc);
  const int want_g = deriv2 != NULL;
  const double reg = trial_regularizer(w, w->vt, w->tmp_vc, w->tmp_gamma, deriv ? w->tmp_imp : NULL,
                                       w->t_pd_hdiag, w->t_lim_hdiag, want_g ? w->t_G : NULL);
  const double momentum = mom0 + alpha * dell_a0 + 0.5 * alpha * alpha * d2ell_a;
  if (deriv) {
    double d = 0.0;
    for (int32_t i = 0; i < n; ++i) {
      double value = w->dp[i] * (w->vt[i] - w->v_star[i]);
      value = value - w->dv[i] * w->tmp_imp[i];
      d += value;
    }
    *deriv = d;
  }
  if (deriv2) {
    double out = d2ell_a;
    for (int32_t c = 0; c < w->count; ++c) {
      double dvc[3] = {0, 0, 0};
      for (int32_t r = 0; r < 3; ++r) {
        const double* row = w->J + ((size_t)c * 3 + r) * n;
        double s = 0.0;
        for (int32_t j = 0; j < n; ++j) s += row[j] * w->dv[j];
        dvc[r] = s;
      }
      const double* g = w->t_G + 9 * c;
      const double gx = g[0] * dvc[0] + g[1] * dvc[1] + g[2] * dvc[2];
      const double gy = g[3] * dvc[0] + g[4] * dvc[1] + g[5] * dvc[2];
      const double gz = g[6] * dvc[0] + g[7] * dvc[1] + g[8] * dvc[2];
      out += dvc[0] * gx + dvc[1] * gy + dvc[2] * gz;
    }
    for (int32_t i = 0; i < n; ++i) {
      double h = 0.0;
      if (w->has_pd) h += w->t_pd_hdiag[i];
      if (w->has_lim) h += w->t_lim_hdiag[i];
      out += h * w->dv[i] * w->dv[i];
    }
    *deriv2 = out;
  }
  return momentum + reg;
}

static int armijo_ok(double alpha, double ell, double ell0, double dell0, double c) {
  /* sim/sap_helpers.py:2600-2608 */
  return ell < ell0 + c * alpha * dell0;
}

/* armijo_decay: _run_sap_backtracking sim/contact_solve.py:5108-5305 with the
 * state kernels :2670-2904. */
static ls_result line_search_armijo(world_ctx* w, const sapb_solve_options* o) {
  ls_result r = {0, 0, 0, 0.0, w->cost};
  double dell0, dell_a0, d2ell_a, mom0;
  line_coefficients(w, &dell0, &dell_a0, &d2ell_a, &mom0);
  const double amax = 1.0 / o->rho;
  const double slop_rel = o->line_search_relative_slop;
  double alpha = amax, alpha_prev = amax, ell_prev = w->cost;
  double ell_slop = (slop_rel / 10.0) * dmax(1.0, fabs(w->cost));
  r.alpha = alpha;
  if (o->line_search_max_iterations <= 0) return r;
  if (dell0 >= 0.0 || !isfinite(dell0)) {
    r.status = SAPB_LS_ASCENT_DIRECTION;
    return r;
  }
  double deriv = 0.0;
  double ell = eval_trial(w, alpha, mom0, dell_a0, d2ell_a, &deriv, NULL);
  {
    const double scale = dmax(1.0, 0.5 * (fabs(ell) + fabs(w->cost)));
    const double slop = (slop_rel / 10.0) * scale;
    ell_slop = slop;
    if (deriv < 0.0 || deriv < slop) {
      r.accepted = 1;
      r.accepted_cost = ell;
      r.alpha = alpha;
      return r;
    }
    alpha_prev = alpha;
    ell_prev = ell;
  }
  if (o->line_search_max_iterations <= 1) return r;
  for (int32_t iteration = 1;; ++iteration) {
    alpha = alpha * o->rho;
    ell = eval_trial(w, alpha, mom0, dell_a0, d2ell_a, NULL, NULL);
    const double a = alpha, a_prev = alpha_prev, e_prev = ell_prev;
    const double denom = a - a_prev;
    double dell_approx = 0.0;
    if (fabs(denom) > 0.0) dell_approx = (ell - e_prev) / denom;
    int accept = 0, accept_prev = 0;
    if (fabs(dell_approx) < ell_slop) {
      accept = 1;
    } else if (ell > e_prev && armijo_ok(a, ell, w->cost, dell0, o->armijo_c)) {
      accept = 1;
      if (armijo_ok(a_prev, e_prev, w->cost, dell0, o->armijo_c)) accept_prev = 1;
    }
    if (accept) {
      r.accepted = 1;
      r.iterations = iteration;
      if (accept_prev) {
        r.alpha = a_prev;
        r.accepted_cost = e_prev;
      } else {
        r.alpha = a;
        r.accepted_cost = ell;
      }
      return r;
    }
    if (iteration >= o->line_search_max_iterations - 1) {
      r.alpha = alpha;
      if (armijo_ok(alpha, ell, w->cost, dell0, o->armijo_c)) {
        r.accepted = 1;
        r.iterations = o->line_search_max_iterations;
        r.accepted_cost = ell;
      } else {
        r.status = SAPB_LS_ALPHA_UNDERFLOW;
      }
      return r;
    }
    alpha_prev = a;
    ell_prev = ell;
  }
}

/* monotone_decay: the fused kernel sim/contact_solve.py:2483-2667 driven by
 * _run_unit_decay_line_search :5307-5414 (decay 0.5, min alpha 1e-8, relax
 * 1e-12 relative + 1e-14 absolute).  Trial contact velocities are vc + alpha dvc
 * as in the reference kernel. */
static ls_result line_search_monotone(world_ctx* w, const sapb_solve_options* o) {
  const int32_t n = w->n;
  ls_result r = {0, 0, 0, 1.0, w->cost};
  double base_linear = 0.0, base_quadratic = 0.0, base0 = 0.0;
  for (int32_t i = 0; i < n; ++i)
    for (int32_t j = 0; j < n; ++j) {
      const double ri = w->v[i] - w->v_star[i], rj = w->v[j] - w->v_star[j];
      const double aij = w->A[i * n + j];
      base0 += 0.5 * ri * aij * rj;
      base_linear += w->dv[i] * aij * rj;
      base_quadratic += w->dv[i] * aij * w->dv[j];
    }
  double* dvc = w->tmp_gamma; /* reuse */
  contact_velocities(w, w->dv, dvc);
  const double current = w->cost;
  double alpha = 1.0, trial_cost = current;
  int accepted = 0, status = 0, iterations = 0;
  for (int32_t it = 0; it < o->line_search_max_iterations; ++it) {
    const double momentum = base0 + alpha * base_linear + 0.5 * alpha * alpha * base_quadratic;
    double reg = 0.0;
    for (int32_t c = 0; c < w->count; ++c) {
      double vc[3];
      for (int32_t k = 0; k < 3; ++k) vc[k] = w->vc[3 * c + k] + alpha * dvc[3 * c + k];
      sapo_projection p;
      sapo_project_contact(vc, w->phi0[c], w->w[c], w->mu[c], w->k[c], ctx_tau(w, c), w->beta, w->sigma, w->dt, 0,
                           &p);
      reg += p.cost;
    }
    for (int32_t i = 0; i < n; ++i) {
      const double vi = w->v[i] + alpha * w->dv[i];
      if (w->has_pd && w->pd_active[i]) {
        const double gain = w->pd_gain[i];
        if (gain > 0.0) {
          const double y = w->pd_a[i] - gain * vi;
          reg += (w->dt / gain) * sapo_clamp_antiderivative(y, w->pd_limit[i]);
        }
      }
      if (w->has_lim) {
        if (w->lo_act[i]) {
          const double g = w->lo_rinv[i] * (w->lo_vhat[i] - vi);
          if (g > 0.0) reg += 0.5 * w->lo_r[i] * g * g;
        }
        if (w->up_act[i]) {
          const double g = w->up_rinv[i] * (w->up_vhat[i] + vi);
          if (g > 0.0) reg += 0.5 * w->up_r[i] * g * g;
        }
      }
    }
    trial_cost = momentum + reg;
    iterations += 1;
    const double tol = 1.0e-14 + 1.0e-12 * fabs(current);
    if (trial_cost <= current + tol) {
      accepted = 1;
      break;
    }
    alpha = alpha * 0.5;
    if (alpha < 1.0e-8) {
      status = SAPB_LS_ALPHA_UNDERFLOW;
      break;
    }
  }
  r.accepted = accepted;
  r.status = status;
  r.iterations = iterations;
  r.alpha = alpha;
  r.accepted_cost = accepted ? trial_cost : current;
  return r;
}

/* exact_root: _run_sap_exact sim/contact_solve.py:5700-5861 with the state
 * kernels :2914-3140 (alpha_max 1.5, tolerance 1e-8, cubic seed :2997-3015). */
static ls_result line_search_exact(world_ctx* w, const sapb_solve_options* o) {
  ls_result r = {0, 0, 0, SAPO_EXACT_ALPHA_MAX, w->cost};
  const int32_t max_it = o->line_search_max_iterations;
  if (max_it <= 0) return r;
  double dell0, dell_a0, d2ell_a, mom0;
  line_coefficients(w, &dell0, &dell_a0, &d2ell_a, &mom0);
  const double amax = SAPO_EXACT_ALPHA_MAX;
  if (dell0 >= 0.0 || !isfinite(dell0)) {
    r.status = SAPB_LS_ASCENT_DIRECTION;
    return r;
  }
  double deriv, deriv2;
  const double ell = eval_trial(w, amax, mom0, dell_a0, d2ell_a, &deriv, &deriv2);
  int active = 0;
  double scale = 0, x_lo = 0, x_hi = 0, f_hi = 0, root = 0, mdx = 0, mdx_prev = 0, xtol = 0;
  if (deriv <= 0.0) {
    r.accepted = 1;
    r.alpha = amax;
  } else if (-dell0 < o->cost_abs_tol + o->cost_rel_tol * ell) {
    r.accepted = 1;
    r.alpha = 1.0;
  } else {
    scale = -dell0;
    const double f_upper = deriv / scale;
    if (!isfinite(f_upper) || f_upper <= 0.0) {
      r.status = SAPB_LS_BAD_BRACKET;
    } else {
      const double quad_guess = -dell0 / deriv2;
      double guess = quad_guess;
      if (o->cubic_init) {
        const double h = amax, c0 = w->cost, d0 = dell0, c1 = ell, d1 = deriv;
        const double theta = d0 + d1 - 3.0 * (c1 - c0) / h;
        const double disc = theta * theta - d0 * d1;
        if (isfinite(disc) && disc >= 0.0) {
          const double g = sqrt(disc);
          const double denom = d1 - d0 + 2.0 * g;
          if (denom != 0.0) {
            const double cg = h - h * (d1 + g - theta) / denom;
            if (isfinite(cg) && cg > 0.0 && cg <= h) guess = cg;
          }
        }
      }
      if (guess > amax) guess = amax;
      if (!isfinite(guess) || guess < 0.0 || guess > amax || SAPO_EXACT_F_TOL * guess <= 0.0) {
        r.status = SAPB_LS_BAD_GUESS;
      } else {
        x_lo = 0.0;
        x_hi = amax;
        f_hi = f_upper;
        root = guess;
        mdx = -amax;
        mdx_prev = -amax;
        xtol = SAPO_EXACT_F_TOL * guess;
        r.alpha = guess;
        active = 1;
      }
    }
  }
  for (int32_t iteration = 1; active; ++iteration) {
    double d, d2;
    eval_trial(w, r.alpha, mom0, dell_a0, d2ell_a, &d, &d2);
    const double f = d / scale, df = d2 / scale;
    const double f_upper = f_hi;
    if ((f < 0.0 && f_upper >= 0.0) || (f >= 0.0 && f_upper < 0.0)) {
      x_lo = root;
    } else {
      x_hi = root;
      f_hi = f;
    }
    if (fabs(f) < SAPO_EXACT_F_TOL) {
      r.accepted = 1;
      r.iterations = iteration;
      r.alpha = root;
      break;
    }
    if (iteration >= max_it) {
      r.status = SAPB_LS_ROOT_ITERATION_CAP;
      break;
    }
    const int slow = 2.0 * fabs(f) > fabs(mdx_prev * df);
    mdx_prev = mdx;
    const double bis_mdx = 0.5 * (x_lo - x_hi);
    const double bis_root = x_lo - bis_mdx;
    double n_mdx = 0.0, n_root = root;
    if (fabs(df) > 0.0) {
      n_mdx = f / df;
      n_root = root - n_mdx;
    }
    int use_bisect = slow;
    if (n_root < x_lo || n_root > x_hi) use_bisect = 1;
    if (!isfinite(n_root) || !isfinite(n_mdx)) use_bisect = 1;
    const double next_root = use_bisect ? bis_root : n_root;
    const double next_mdx = use_bisect ? bis_mdx : n_mdx;
    if (fabs(next_mdx) < xtol) {
      r.accepted = 1;
      r.iterations = iteration;
      r.alpha = next_root;
      break;
    }
    root = next_root;
    mdx = next_mdx;
    r.alpha = next_root;
  }
  if (r.accepted) r.accepted_cost = eval_trial(w, r.alpha, mom0, dell_a0, d2ell_a, NULL, NULL);
  return r;
}

/* Norms and the convergence test of
 * _compute_norm_terms_and_update_active_conditional sim/contact_solve.py:1970-2087.
 * Returns 1 if the world stays active. */
static int update_active(world_ctx* w, const sapb_solve_options* o, int32_t iteration, double alpha,
                         double previous_cost, int32_t* converged, int32_t* newton_iterations, double* grad_norm) {
  const int32_t n = w->n;
  double g2 = 0.0, p2 = 0.0, j2 = 0.0;
  for (int32_t i = 0; i < n; ++i) {
    if (!w->part[i]) continue;
    const double s = w->d_scale[i];
    const double g = s * w->grad[i], p = s * w->dyn[i], jc = s * w->impulse[i];
    g2 += g * g;
    p2 += p * p;
    j2 += jc * jc;
  }
  const double gn = sqrt(dmax(g2, 0.0)), pn = sqrt(dmax(p2, 0.0)), jn = sqrt(dmax(j2, 0.0));
  *grad_norm = gn;
  const double opt_tol = o->optimality_abs_tol + o->optimality_rel_tol * dmax(pn, jn);
  const double cost_min_alpha = o->line_search_variant == SAPB_LS_MONOTONE_DECAY ? 0.0 : 0.5;
  int opt = gn <= opt_tol;
  int cost_ok = 0;
  if (iteration > 0 && alpha > cost_min_alpha) {
    const double scale = 0.5 * (fabs(w->cost) + fabs(previous_cost));
    const double tol = o->cost_abs_tol + o->cost_rel_tol * scale;
    if (fabs(w->cost - previous_cost) < tol) cost_ok = 1;
  }
  *newton_iterations = iteration;
  if (opt || cost_ok) {
    *converged = 1;
    return 0;
  }
  if (iteration >= o->max_iterations) return 0;
  *converged = 0;
  return 1;
}

static void solve_world(const sapb_contact_problem* P, const sapb_solve_options* o, const sapb_solve_outputs* out,
                        int32_t e, int use_guess) {
  const int32_t n = P->dof_per_env, C = P->max_contacts;
  world_ctx w;
  memset(&w, 0, sizeof(w));
  w.n = n;
  w.C = C;
  int32_t count = P->contact_count[e];
  if (count > C) count = C;
  if (count < 0) count = 0;
  w.count = count;
  w.A = P->dynamics_matrix + (size_t)e * n * n;
  w.J = P->jacobian + (size_t)e * C * 3 * n;
  w.phi0 = P->phi0 + (size_t)e * C;
  w.w = P->w_eff + (size_t)e * C;
  w.mu = P->mu + (size_t)e * C;
  w.k = P->stiffness + (size_t)e * C;
  w.tau = P->tau_d ? P->tau_d + (size_t)e * C : NULL;
  w.tau_fallback = o->contact_tau_d;
  w.dt = P->dt[e];
  w.beta = o->contact_beta;
  w.sigma = o->contact_sigma;
  const sapb_dof_terms* D = P->dof;
  w.has_pd = D ? D->has_pd : 0;
  w.has_lim = D ? D->has_limits : 0;

  const size_t nd = (size_t)n;
  const size_t nc = (size_t)(count > 0 ? count : 1);
  double* pool = (double*)calloc(nd * 40 + nd * nd + nc * 40, sizeof(double));
  int32_t* ipool = (int32_t*)calloc(nd * 4, sizeof(int32_t));
  double* q = pool;
#define TAKE(ptr, cnt) (ptr = q, q += (cnt))
  TAKE(w.v_star, nd); TAKE(w.v, nd); TAKE(w.a_inv_diag, nd); TAKE(w.d_scale, nd);
  TAKE(w.pd_a, nd); TAKE(w.pd_gain, nd); TAKE(w.pd_limit, nd);
  TAKE(w.lo_vhat, nd); TAKE(w.up_vhat, nd); TAKE(w.lo_r, nd); TAKE(w.up_r, nd);
  TAKE(w.lo_rinv, nd); TAKE(w.up_rinv, nd);
  TAKE(w.impulse, nd); TAKE(w.grad, nd); TAKE(w.dyn, nd);
  TAKE(w.pd_gamma, nd); TAKE(w.pd_hdiag, nd); TAKE(w.lim_grad, nd); TAKE(w.lim_hdiag, nd);
  TAKE(w.dv, nd); TAKE(w.dp, nd); TAKE(w.vt, nd); TAKE(w.tmp_imp, nd);
  TAKE(w.t_pd_hdiag, nd); TAKE(w.t_lim_hdiag, nd);
  TAKE(w.H, nd * nd);
  TAKE(w.vc, nc * 3); TAKE(w.gamma, nc * 3); TAKE(w.ccost, nc); TAKE(w.tmp_vc, nc * 3);
  TAKE(w.tmp_gamma, nc * 3); TAKE(w.G, nc * 9); TAKE(w.t_G, nc * 9);
#undef TAKE
  w.pd_active = ipool;
  w.lo_act = ipool + nd;
  w.up_act = ipool + 2 * nd;
  w.part = ipool + 3 * nd;

  /* Velocity inputs (sim/contact_solve.py:299-338). */
  const size_t base = (size_t)e * n;
  for (int32_t i = 0; i < n; ++i) {
    w.v_star[i] = P->v_star[base + i];
    double v = P->v0[base + i];
    if (P->v_guess) {
      if (use_guess) v = P->v_guess[base + i];
      P->v_guess[base + i] = v;
    }
    w.v[i] = v;
  }
  /* diag(A) data (:405-419). */
  for (int32_t i = 0; i < n; ++i) {
    double d = w.A[i * n + i];
    if (d < 1.0e-12 || !isfinite(d)) d = 1.0e-12;
    w.a_inv_diag[i] = 1.0 / d;
    w.d_scale[i] = 1.0 / sqrt(d);
  }
  /* PD terms (:490-562). */
  for (int32_t i = 0; i < n; ++i) {
    w.pd_active[i] = 0;
    if (!w.has_pd) continue;
    const size_t dof = base + i;
    int32_t coord = D->dof_coord_index[dof];
    if (coord >= D->joint_coord_count) coord = -1;
    int32_t target = D->dof_target_index[dof];
    if (target < 0 || target >= P->num_envs * n) target = (int32_t)dof;
    if (D->joint_target_mode[target] == 0) continue;
    const double kp = (double)D->joint_target_ke[target];
    const double kd = (double)D->joint_target_kd[target];
    if (kp <= 0.0 && kd <= 0.0) continue;
    if (coord < 0 && kp > 0.0) continue;
    double eff[2];
    sapo_effective_pd_gains(kp, kd, w.dt, w.a_inv_diag[i], eff);
    const double gain = w.dt * eff[0] + eff[1];
    if (gain <= 0.0) continue;
    double q0 = 0.0, qd = 0.0;
    if (coord >= 0) {
      q0 = D->joint_q[coord];
      qd = D->joint_target_pos ? (double)D->joint_target_pos[target] : 0.0;
    }
    const double vd = D->joint_target_vel ? (double)D->joint_target_vel[target] : 0.0;
    const double u0 = D->joint_act ? (double)D->joint_act[target] : 0.0;
    w.pd_active[i] = 1;
    w.pd_a[i] = eff[0] * (qd - q0) + eff[1] * vd + u0;
    w.pd_gain[i] = gain;
    w.pd_limit[i] = (double)D->joint_effort_limit[target];
  }
  /* Limit terms (:605-683). */
  for (int32_t i = 0; i < n; ++i) {
    w.lo_act[i] = 0;
    w.up_act[i] = 0;
    w.lo_r[i] = 1.0;
    w.up_r[i] = 1.0;
    if (!w.has_lim) continue;
    const size_t dof = base + i;
    int32_t coord = D->dof_coord_index[dof];
    if (coord >= D->joint_coord_count) coord = -1;
    if (coord < 0 || D->limit_supported[dof] == 0) continue;
    const double ke = D->joint_limit_ke[dof];
    if (ke <= 0.0) continue;
    const double q0 = D->joint_q[coord];
    const double lower = D->joint_limit_lower[dof], upper = D->joint_limit_upper[dof];
    const double speed = dmax(fabs(P->v0[base + i]), fabs(w.v_star[i]));
    const double window = SAPO_LIMIT_WINDOW_FACTOR * w.dt * speed;
    const double kd = D->joint_limit_kd[dof];
    double tau_d = 0.0;
    if (kd > 0.0) tau_d = kd / ke;
    const double bf = SAPO_LIMIT_BETA * SAPO_LIMIT_BETA / (4.0 * SAPO_PI * SAPO_PI);
    const double r_nr = bf * dmax(w.a_inv_diag[i], 1.0e-12);
    const double r_soft = 1.0 / (w.dt * ke * (w.dt + tau_d));
    const double r = dmax(r_nr, r_soft);
    const double rinv = 1.0 / r;
    if (isfinite(lower)) {
      const double g = q0 - lower;
      if (g <= window) {
        w.lo_act[i] = 1;
        w.lo_vhat[i] = -g / (w.dt + tau_d);
        w.lo_r[i] = r;
        w.lo_rinv[i] = rinv;
      }
    }
    if (isfinite(upper)) {
      const double g = upper - q0;
      if (g <= window) {
        w.up_act[i] = 1;
        w.up_vhat[i] = -g / (w.dt + tau_d);
        w.up_r[i] = r;
        w.up_rinv[i] = rinv;
      }
    }
  }
  /* Participating DOFs (:423-488, 3804-3839). */
  for (int32_t c = 0; c < count; ++c) {
    const int32_t bodies[2] = {P->body0 ? P->body0[(size_t)e * C + c] : -1,
                               P->body1 ? P->body1[(size_t)e * C + c] : -1};
    for (int b = 0; b < 2; ++b) {
      const int32_t body = bodies[b];
      if (body < 0 || body >= P->num_bodies || !P->body_dof_start) continue;
      const int32_t s = P->body_dof_start[body], m = P->body_dof_count[body];
      if (s >= 0 && m > 0)
        for (int32_t i = s; i < s + m && i < n; ++i)
          if (i >= 0) w.part[i] = 1;
    }
    for (int32_t i = 0; i < n; ++i)
      if (w.J[((size_t)c * 3 + 0) * n + i] != 0.0 || w.J[((size_t)c * 3 + 1) * n + i] != 0.0 ||
          w.J[((size_t)c * 3 + 2) * n + i] != 0.0)
        w.part[i] = 1;
  }
  for (int32_t i = 0; i < n; ++i)
    if (w.pd_active[i] || w.lo_act[i] || w.up_act[i]) w.part[i] = 1;

  /* Initialization and unconstrained worlds (:340-394). */
  int32_t newton_iterations = 0, ls_total = 0, converged = 0, status = 0;
  double alpha = 1.0, previous_cost = 0.0, grad_norm = 0.0;
  int32_t ws_accepted = 0;
  int unconstrained = count == 0;
  for (int32_t i = 0; i < n; ++i)
    if (w.pd_active[i] || w.lo_act[i] || w.up_act[i]) unconstrained = 0;
  int evaluated = 0;
  if (unconstrained) {
    converged = 1;
    for (int32_t i = 0; i < n; ++i) w.v[i] = w.v_star[i];
  } else {
    for (int32_t i = 0; i < n; ++i)
      if (!w.part[i]) w.v[i] = w.v_star[i];
    /* Candidate starts (no counterpart in the reference): for each impulse
     * set, v_c = v* + A^-1 J^T gamma_c on the participating DOFs; the start
     * with the lowest cost among the plain one and the candidates is taken. */
    if (P->gamma0 && count > 0) {
      const int32_t K = P->gamma0_count > 1 ? P->gamma0_count : 1;
      double best_cost = evaluate(&w, w.v, w.vc, w.gamma, w.ccost, w.impulse, w.grad, w.dyn, w.pd_gamma,
                                  w.pd_hdiag, w.lim_grad, w.lim_hdiag, NULL);
      double* L = (double*)malloc(sizeof(double) * nd * nd);
      double* x = (double*)malloc(sizeof(double) * nd);
      double* vbest = (double*)malloc(sizeof(double) * nd);
      memcpy(L, w.A, sizeof(double) * nd * nd);
      memcpy(vbest, w.v, sizeof(double) * nd);
      if (sapo_cholesky(L, n) == 0) {
        for (int32_t k = 0; k < K; ++k) {
          const double* g0 = P->gamma0 + ((size_t)k * P->num_envs + e) * C * 3;
          for (int32_t i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int32_t c = 0; c < count; ++c)
              for (int32_t r = 0; r < 3; ++r) acc += w.J[((size_t)c * 3 + r) * n + i] * g0[3 * c + r];
            x[i] = acc;
          }
          for (int32_t i = 0; i < n; ++i) {
            double t = x[i];
            for (int32_t q = 0; q < i; ++q) t -= L[i * n + q] * x[q];
            x[i] = t / L[i * n + i];
          }
          for (int32_t i = n - 1; i >= 0; --i) {
            double t = x[i];
            for (int32_t q = i + 1; q < n; ++q) t -= L[q * n + i] * x[q];
            x[i] = t / L[i * n + i];
          }
          for (int32_t i = 0; i < n; ++i) w.v[i] = w.part[i] ? w.v_star[i] + x[i] : w.v_star[i];
          const double cost_c = evaluate(&w, w.v, w.vc, w.gamma, w.ccost, w.impulse, w.grad, w.dyn, w.pd_gamma,
                                         w.pd_hdiag, w.lim_grad, w.lim_hdiag, NULL);
          if (cost_c < best_cost) {
            best_cost = cost_c;
            ws_accepted = k + 1;
            memcpy(vbest, w.v, sizeof(double) * nd);
          }
        }
      }
      memcpy(w.v, vbest, sizeof(double) * nd);
      free(L);
      free(x);
      free(vbest);
    }
    /* Newton loop (:5559-5655 with the body :5474-5557). */
    int32_t it = 0;
    w.cost = evaluate(&w, w.v, w.vc, w.gamma, w.ccost, w.impulse, w.grad, w.dyn, w.pd_gamma, w.pd_hdiag,
                      w.lim_grad, w.lim_hdiag, NULL);
    evaluated = 1;
    int active = o->max_iterations > 0 ? 1 : 0;
    if (o->max_iterations >= 0)
      active = update_active(&w, o, it, alpha, previous_cost, &converged, &newton_iterations, &grad_norm);
    while (active) {
      /* G at the stored vc (:1071-1217). */
      for (int32_t c = 0; c < count; ++c) {
        sapo_projection p;
        sapo_project_contact(w.vc + 3 * c, w.phi0[c], w.w[c], w.mu[c], w.k[c], ctx_tau(&w, c), w.beta, w.sigma, w.dt,
                             1, &p);
        memcpy(w.G + 9 * c, p.g, sizeof(p.g));
      }
      newton_direction(&w, o);
      ls_result r;
      if (o->line_search_variant == SAPB_LS_ARMIJO_DECAY)
        r = line_search_armijo(&w, o);
      else if (o->line_search_variant == SAPB_LS_EXACT_ROOT)
        r = line_search_exact(&w, o);
      else
        r = line_search_monotone(&w, o);
      alpha = r.alpha;
      status = r.status;
      if (r.accepted) ls_total += r.iterations;
      else if (o->line_search_variant == SAPB_LS_MONOTONE_DECAY) ls_total += r.iterations;
      if (r.accepted) {
        previous_cost = w.cost;
        w.cost = r.accepted_cost;
        for (int32_t i = 0; i < n; ++i) w.v[i] = w.v[i] + r.alpha * w.dv[i];
      } else if (o->line_search_variant == SAPB_LS_MONOTONE_DECAY) {
        previous_cost = w.cost;
      }
      ++it;
      w.cost = evaluate(&w, w.v, w.vc, w.gamma, w.ccost, w.impulse, w.grad, w.dyn, w.pd_gamma, w.pd_hdiag,
                        w.lim_grad, w.lim_hdiag, NULL);
      active = update_active(&w, o, it, alpha, previous_cost, &converged, &newton_iterations, &grad_norm);
    }
  }
  /* outputs */
  for (int32_t i = 0; i < n; ++i) out->v[base + i] = w.v[i];
  if (out->contact_gamma) {
    for (int32_t c = 0; c < C; ++c)
      for (int32_t r = 0; r < 3; ++r)
        out->contact_gamma[((size_t)e * C + c) * 3 + r] = (evaluated && c < count) ? w.gamma[3 * c + r] : 0.0;
  }
  /* Modes of the projection at the returned velocity (the active set of the
   * solution); slots beyond the count and unconstrained worlds are NONE. */
  if (out->contact_mode) {
    for (int32_t c = 0; c < C; ++c) {
      int32_t mode = SAPB_CONTACT_MODE_NONE;
      if (evaluated && c < count) {
        sapo_projection p;
        sapo_project_contact(w.vc + 3 * c, w.phi0[c], w.w[c], w.mu[c], w.k[c], ctx_tau(&w, c), w.beta, w.sigma, w.dt,
                             0, &p);
        mode = p.mode;
      }
      out->contact_mode[(size_t)e * C + c] = mode;
    }
  }
  if (out->cost) out->cost[e] = evaluated ? w.cost : 0.0;
  if (out->newton_iterations) out->newton_iterations[e] = newton_iterations;
  if (out->line_search_iterations) out->line_search_iterations[e] = ls_total;
  if (out->converged) out->converged[e] = converged;
  if (out->status) out->status[e] = status;
  if (out->grad_norm) out->grad_norm[e] = grad_norm;
  if (out->warm_start_accepted) out->warm_start_accepted[e] = ws_accepted;
  free(pool);
  free(ipool);
}

int32_t sapo_contact_solve(const sapb_contact_problem* P, const sapb_solve_options* o, const sapb_solve_outputs* out,
                           int32_t num_threads) {
  if (!P || !o || !out || !out->v || P->num_envs < 0 || P->dof_per_env <= 0 || P->max_contacts < 0)
    return SAPB_ERR_INVALID_ARGUMENT;
  if (!P->contact_count || !P->dynamics_matrix || !P->v_star || !P->v0 || !P->dt) return SAPB_ERR_INVALID_ARGUMENT;
  if (P->max_contacts > 0 && (!P->jacobian || !P->phi0 || !P->w_eff || !P->mu || !P->stiffness))
    return SAPB_ERR_INVALID_ARGUMENT;
  if (P->dof && ((P->dof->has_pd || P->dof->has_limits) && (!P->dof->dof_coord_index || !P->dof->joint_q)))
    return SAPB_ERR_INVALID_ARGUMENT;
  const int use_guess = (P->v_guess && P->v_guess_active && P->v_guess_active[0] != 0) ? 1 : 0;
#ifdef _OPENMP
  if (num_threads > 0) omp_set_num_threads(num_threads);
#pragma omp parallel for schedule(dynamic, 4)
#else
  (void)num_threads;
#endif
  for (int32_t e = 0; e < P->num_envs; ++e) solve_world(P, o, out, e, use_guess);
  return SAPB_OK;
}
