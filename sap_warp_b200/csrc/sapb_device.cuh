// sapb_device.cuh -- device helpers shared by the SAP step kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/sapb.h"

namespace sapb {

constexpr double kPi = 3.141592653589793;
constexpr double kSoftNormTol = 1.0e-7;   // sim/contact_solve.py:47
constexpr double kPdBeta = 0.1;           // sim/contact_solve.py:48
constexpr double kLimitBeta = 0.1;        // sim/contact_solve.py:49
constexpr double kLimitWindow = 2.0;      // sim/contact_solve.py:51
constexpr double kExactAlphaMax = 1.5;    // sim/contact_solve.py:52
constexpr double kExactFTol = 1.0e-8;     // sim/contact_solve.py:54

// Per-contact constants of the regularized projection that do not depend on
// the velocity (sim/contact_solve.py:793-823): computed once per solve.
struct ContactConst {
  double rt, rn, rt_inv, rn_inv, vhat_n, mu, mu_hat, factor;
};

__device__ __forceinline__ ContactConst make_contact_const(double phi0, double w_eff, double mu, double k,
                                                           double tau_d, double beta, double sigma, double dt) {
  ContactConst cc;
  double wi = w_eff;
  if (wi < 1.0e-12 || !isfinite(wi)) wi = 1.0e-12;
  const double beta_factor = beta * beta / (4.0 * kPi * kPi);
  const double rn_hard = beta_factor * wi;
  double k_c = k;
  if (k_c <= 0.0 || !isfinite(k_c)) k_c = 1.0;
  const double tau_c = fmax(tau_d, 0.0);
  const double rn_soft = 1.0 / (dt * k_c * (dt + tau_c));
  double rn = fmax(rn_hard, rn_soft);
  double rt = sigma * wi;
  if (rt < 1.0e-30) rt = 1.0e-30;
  if (rn < 1.0e-30) rn = 1.0e-30;
  cc.rt = rt;
  cc.rn = rn;
  cc.rt_inv = 1.0 / rt;
  cc.rn_inv = 1.0 / rn;
  cc.vhat_n = -phi0 / (dt + tau_c);
  double m = mu;
  if (m < 0.0 || !isfinite(m)) m = 0.0;
  cc.mu = m;
  cc.mu_hat = m * rt / rn;
  const double mu_tilde = m * sqrt(rt / rn);
  cc.factor = 1.0 / (1.0 + mu_tilde * mu_tilde);
  return cc;
}

// Projection onto the regularized friction cone (sim/contact_solve.py:825-921):
// returns the mode, writes gamma, the cost and (if G != nullptr) the 3x3
// derivative G = d gamma / d(-vc), row-major.
__device__ __forceinline__ int project_contact(const ContactConst& cc, double vcx, double vcy, double vcz,
                                               double gamma[3], double* cost, double* G) {
  const double y0 = -cc.rt_inv * vcx;
  const double y1 = -cc.rt_inv * vcy;
  const double y2 = cc.rn_inv * (cc.vhat_n - vcz);
  const double m = cc.mu;
  const double yr = sqrt(y0 * y0 + y1 * y1 + kSoftNormTol * kSoftNormTol);
  const double inv_yr = 1.0 / yr;  // yr >= 1e-7 > 0
  const double tx = y0 * inv_yr, ty = y1 * inv_yr;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  int mode = SAPB_CONTACT_MODE_NONE;
  if (G) {
#pragma unroll
    for (int k = 0; k < 9; ++k) G[k] = 0.0;
  }
  if (m <= 1.0e-12) {
    if (y2 > 0.0) {
      g2 = y2;
      if (G) G[8] = cc.rn_inv;
      mode = SAPB_CONTACT_MODE_FRICTIONLESS;
    }
  } else {
    const double mu_hat = cc.mu_hat;
    const double factor = cc.factor;
    if (yr <= m * y2) {
      g0 = y0;
      g1 = y1;
      g2 = y2;
      if (G) {
        G[0] = cc.rt_inv;
        G[4] = cc.rt_inv;
        G[8] = cc.rn_inv;
      }
      mode = SAPB_CONTACT_MODE_STICTION;
    } else if ((-mu_hat * yr < y2) && (y2 < yr / m)) {
      const double gn = (y2 + mu_hat * yr) * factor;
      g0 = m * gn * tx;
      g1 = m * gn * ty;
      g2 = gn;
      if (G) {
        const double p00 = tx * tx, p01 = tx * ty, p11 = ty * ty;
        const double gn_over_yr = gn * inv_yr;
        const double d00 = m * (gn_over_yr * (1.0 - p00) + mu_hat * factor * p00);
        const double d01 = m * (gn_over_yr * (-p01) + mu_hat * factor * p01);
        const double d11 = m * (gn_over_yr * (1.0 - p11) + mu_hat * factor * p11);
        G[0] = d00 * cc.rt_inv;
        G[1] = d01 * cc.rt_inv;
        G[2] = m * factor * tx * cc.rn_inv;
        G[3] = d01 * cc.rt_inv;
        G[4] = d11 * cc.rt_inv;
        G[5] = m * factor * ty * cc.rn_inv;
        G[6] = mu_hat * factor * tx * cc.rt_inv;
        G[7] = mu_hat * factor * ty * cc.rt_inv;
        G[8] = factor * cc.rn_inv;
      }
      mode = SAPB_CONTACT_MODE_SLIDING;
    }
  }
  gamma[0] = g0;
  gamma[1] = g1;
  gamma[2] = g2;
  *cost = 0.5 * (cc.rt * (g0 * g0 + g1 * g1) + cc.rn * g2 * g2);
  return mode;
}

// sim/sap_helpers.py:2251-2276
__device__ __forceinline__ double clamp_limit(double x, double limit) {
  if (limit <= 0.0 || !isfinite(limit)) return x;
  return fmax(-limit, fmin(limit, x));
}
__device__ __forceinline__ double clamp_limit_derivative(double x, double limit) {
  if (limit <= 0.0 || !isfinite(limit)) return 1.0;
  return (-limit <= x && x <= limit) ? 1.0 : 0.0;
}
__device__ __forceinline__ double clamp_limit_antiderivative(double x, double limit) {
  if (limit <= 0.0 || !isfinite(limit)) return 0.5 * x * x;
  if (x < -limit) return -limit * (x + 0.5 * limit);
  if (x <= limit) return 0.5 * x * x;
  return limit * (x - 0.5 * limit);
}

// sim/sap_helpers.py:2305-2341
__device__ __forceinline__ void effective_pd_gains(double kp, double kd, double dt, double delassus, double* kp_eff,
                                                   double* kd_eff) {
  *kp_eff = 0.0;
  *kd_eff = 0.0;
  if (kp <= 0.0 && kd <= 0.0) return;
  const double beta_factor = kPdBeta * kPdBeta / (4.0 * kPi * kPi);
  const double r_nr = beta_factor * fmax(delassus, 1.0e-12);
  const double common = dt * kp + kd;
  if (common <= 0.0) return;
  const double r = 1.0 / (dt * common);
  if (r >= r_nr) {
    *kp_eff = kp;
    *kd_eff = kd;
    return;
  }
  if (dt * kp > kd && kp > 0.0) {
    const double tau = kd / kp;
    *kp_eff = 1.0 / (dt * (dt + tau) * r_nr);
    *kd_eff = tau * *kp_eff;
  } else if (kd > 0.0) {
    const double tau_inv = kp / kd;
    *kd_eff = 1.0 / (dt * (1.0 + dt * tau_inv) * r_nr);
    *kp_eff = tau_inv * *kd_eff;
  } else {
    *kp_eff = 1.0 / (dt * dt * r_nr);
    *kd_eff = 0.0;
  }
}

// Reciprocal for pivots on a serial critical path.  Newton-Raphson iteration
// for 1/d (x <- x + x (1 - d x), each step squaring the relative error) from
// the FP32 reciprocal as seed: two steps take the ~2^-23 seed error to below
// 2^-52, i.e. within an ulp or two of the correctly rounded quotient.  Values
// outside the FP32 range (or not finite) use the IEEE division.
__device__ __forceinline__ double fast_recip(double d) {
  const double ad = fabs(d);
  if (!(ad > 1.0e-30 && ad < 1.0e30)) return 1.0 / d;
  double x = (double)__frcp_rn((float)d);
  double e = fma(-d, x, 1.0);
  x = fma(x, e, x);
  e = fma(-d, x, 1.0);
  return fma(x, e, x);
}
__device__ __forceinline__ float fast_recip(float d) { return __frcp_rn(d); }

template <int NT>
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum K values over the block; every thread receives the totals.  `red` is a
// shared buffer of at least K * (NT / 32) doubles.  Contains two barriers.
template <int NT, int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* red) {
  constexpr int W = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = warp_sum<NT>(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) red[k * W + warp] = v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < W; ++w) s += red[k * W + w];
    v[k] = s;
  }
  __syncthreads();
}

}  // namespace sapb
