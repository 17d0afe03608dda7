// sapb_linesearch.cuh -- the three SAP line searches and the per-trial
// regularizer sums, shared by the dense and the tree-blocked solve kernels.
//
// A world type W provides: count (live contacts), dofs(), cc(c) (contact
// constants), Cn(slot) (per-contact FP64 arrays), V(slot) (per-DOF FP64
// arrays), flags (per-DOF bits) and red (block reduction scratch of at least
// 8 * warps doubles).  PP provides `o` (sapb_solve_options) and `dof`
// (sapb_dof_terms; only has_pd / has_limits are read here).  The line
// coefficients c4 = {dell0, dell_a0, d2ell_a, mom0} are computed by the
// caller (they need the world's A and J products).
#pragma once

#include "sapb_device.cuh"

namespace sapb {

// Flag bits of the per-DOF flags array.
constexpr int kFlagPd = 1, kFlagLo = 2, kFlagUp = 4, kFlagPart = 8;

// Vector slots inside off_vec (each ldJ doubles).
enum Vec {
  V_V = 0, V_VSTAR, V_DV, V_GRAD, V_ARES, V_DP, V_DSCALE, V_AINV, V_PDA, V_PDGAIN, V_PDLIM,
  V_LOVHAT, V_UPVHAT, V_LOR, V_UPR, V_LORINV, V_UPRINV, V_HDIAG, V_TMP0, V_SAVE, V_BEST, V_DINV, V_DV2, V_END
};
// Contact slots inside off_con (each C doubles).
enum Con {
  C_RT = 0, C_RN, C_RTINV, C_RNINV, C_VHAT, C_MU, C_MUHAT, C_FACTOR, C_VC, C_DVC = C_VC + 3, C_GAMMA = C_DVC + 3,
  C_END = C_GAMMA + 3
};

// Regularizer terms along the line at step alpha (contact, PD and limit
// costs), the impulse projection onto dv, and (want2) the curvature.
// Restates _replace_trial_cost_with_sap_line_search_cost :2379-2420, the line
// derivative :2304-2321 and the second derivative :2324-2375, using
// vc(alpha) = vc + alpha * dvc.
template <int NT, class W, class PP>
__device__ void line_terms(const W& w, const PP& P, double dt, double alpha, bool want2,
                           double out3[3]) {
  const int tid = threadIdx.x;
  double reg = 0.0, proj = 0.0, curv = 0.0;
  for (int c = tid; c < w.count; c += NT) {
    const ContactConst cc = w.cc(c);
    const double dx = w.Cn(C_DVC + 0)[c], dy = w.Cn(C_DVC + 1)[c], dz = w.Cn(C_DVC + 2)[c];
    double g[3], cost, G[9];
    project_contact(cc, w.Cn(C_VC + 0)[c] + alpha * dx, w.Cn(C_VC + 1)[c] + alpha * dy,
                    w.Cn(C_VC + 2)[c] + alpha * dz, g, &cost, want2 ? G : nullptr);
    reg += cost;
    proj += g[0] * dx + g[1] * dy + g[2] * dz;
    if (want2) {
      curv += dx * (G[0] * dx + G[1] * dy + G[2] * dz) + dy * (G[3] * dx + G[4] * dy + G[5] * dz) +
              dz * (G[6] * dx + G[7] * dy + G[8] * dz);
    }
  }
  if (P.dof.has_pd || P.dof.has_limits) {
    for (int i = tid; i < w.dofs(); i += NT) {
      const double vi = w.V(V_V)[i] + alpha * w.V(V_DV)[i];
      const double dvi = w.V(V_DV)[i];
      const int fl = w.flags[i];
      double hd = 0.0;
      if (P.dof.has_pd && (fl & kFlagPd)) {
        const double gain = w.V(V_PDGAIN)[i], lim = w.V(V_PDLIM)[i];
        const double y = w.V(V_PDA)[i] - gain * vi;
        proj += dvi * dt * clamp_limit(y, lim);
        hd += dt * gain * clamp_limit_derivative(y, lim);
        if (gain > 0.0) reg += (dt / gain) * clamp_limit_antiderivative(y, lim);
      }
      if (P.dof.has_limits) {
        if (fl & kFlagLo) {
          const double g = w.V(V_LORINV)[i] * (w.V(V_LOVHAT)[i] - vi);
          if (g > 0.0) {
            proj += dvi * g;
            hd += w.V(V_LORINV)[i];
            reg += 0.5 * w.V(V_LOR)[i] * g * g;
          }
        }
        if (fl & kFlagUp) {
          const double g = w.V(V_UPRINV)[i] * (w.V(V_UPVHAT)[i] + vi);
          if (g > 0.0) {
            proj -= dvi * g;
            hd += w.V(V_UPRINV)[i];
            reg += 0.5 * w.V(V_UPR)[i] * g * g;
          }
        }
      }
      curv += hd * dvi * dvi;
    }
  }
  double r[3] = {reg, proj, curv};
  block_sum<NT, 3>(r, w.red);
  out3[0] = r[0];
  out3[1] = r[1];
  out3[2] = r[2];
}

// The regularizer terms of line_terms at 4 KT step sizes at once: warp q of
// each group of four warps evaluates alpha[q], alpha[q + 4], ...,
// alpha[q + 4 (KT - 1)] (the same per-step sums and order for any KT), the
// groups split the contacts and DOFs, lanes stride over them, warp-shuffle
// sums, one barrier to publish.  reg[k] for every k and the impulse
// projection onto dv at alpha[0].  (With 128 threads: one group, warp q sums
// everything.)
template <int NT, int KT, class W, class PP>
__device__ void line_termsK(const W& w, const PP& P, double dt, const double (&alpha)[4 * KT],
                            double (&reg)[4 * KT], double* proj0) {
  static_assert(NT % 128 == 0, "groups of four warps");
  constexpr int NG = NT / 128;
  constexpr int NR = 4 * KT + 4;  // reduction slots per group
  static_assert(NG * NR <= 8 * (NT / 32), "reduction scratch");
  const int tid = threadIdx.x, lane = tid & 31, q = (tid >> 5) & 3, grp = tid >> 7;
  const int first = grp * 32 + lane;
  constexpr int stride = 32 * NG;
  double a[KT], rs[KT];
#pragma unroll
  for (int t = 0; t < KT; ++t) {
    a[t] = alpha[q + 4 * t];
    rs[t] = 0.0;
  }
  double ps = 0.0;
  for (int c = first; c < w.count; c += stride) {
    const ContactConst cc = w.cc(c);
    const double dx = w.Cn(C_DVC + 0)[c], dy = w.Cn(C_DVC + 1)[c], dz = w.Cn(C_DVC + 2)[c];
    const double vx = w.Cn(C_VC + 0)[c], vy = w.Cn(C_VC + 1)[c], vz = w.Cn(C_VC + 2)[c];
#pragma unroll
    for (int t = 0; t < KT; ++t) {
      double g[3], cost;
      project_contact(cc, vx + a[t] * dx, vy + a[t] * dy, vz + a[t] * dz, g, &cost, nullptr);
      rs[t] += cost;
      if (t == 0) ps += g[0] * dx + g[1] * dy + g[2] * dz;
    }
  }
  if (P.dof.has_pd || P.dof.has_limits) {
    for (int i = first; i < w.dofs(); i += stride) {
      const double dvi = w.V(V_DV)[i];
      const int fl = w.flags[i];
#pragma unroll
      for (int t = 0; t < KT; ++t) {
        const double vi = w.V(V_V)[i] + a[t] * dvi;
        if (P.dof.has_pd && (fl & kFlagPd)) {
          const double gain = w.V(V_PDGAIN)[i], lim = w.V(V_PDLIM)[i];
          const double y = w.V(V_PDA)[i] - gain * vi;
          if (t == 0) ps += dvi * dt * clamp_limit(y, lim);
          if (gain > 0.0) rs[t] += (dt / gain) * clamp_limit_antiderivative(y, lim);
        }
        if (P.dof.has_limits) {
          if (fl & kFlagLo) {
            const double g = w.V(V_LORINV)[i] * (w.V(V_LOVHAT)[i] - vi);
            if (g > 0.0) {
              if (t == 0) ps += dvi * g;
              rs[t] += 0.5 * w.V(V_LOR)[i] * g * g;
            }
          }
          if (fl & kFlagUp) {
            const double g = w.V(V_UPRINV)[i] * (w.V(V_UPVHAT)[i] + vi);
            if (g > 0.0) {
              if (t == 0) ps -= dvi * g;
              rs[t] += 0.5 * w.V(V_UPR)[i] * g * g;
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int t = 0; t < KT; ++t) rs[t] += __shfl_xor_sync(0xffffffffu, rs[t], o);
    ps += __shfl_xor_sync(0xffffffffu, ps, o);
  }
  __syncthreads();  // earlier readers of red are done
  if (lane == 0) {
#pragma unroll
    for (int t = 0; t < KT; ++t) w.red[grp * NR + 4 * t + q] = rs[t];
    w.red[grp * NR + 4 * KT + q] = ps;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4 * KT; ++k) {
    double s = w.red[k];
#pragma unroll
    for (int g = 1; g < NG; ++g) s += w.red[g * NR + k];
    reg[k] = s;
  }
  double p0 = w.red[4 * KT];
#pragma unroll
  for (int g = 1; g < NG; ++g) p0 += w.red[g * NR + 4 * KT];
  *proj0 = p0;
}

struct LsResult {
  int accepted, status, iterations;
  double alpha, accepted_cost;
};

__device__ __forceinline__ bool armijo_ok(double alpha, double ell, double ell0, double dell0, double c) {
  return ell < ell0 + c * alpha * dell0;  // sim/sap_helpers.py:2600-2608
}

// armijo_decay backtracking (sim/contact_solve.py:2670-2904, driver :5108-5305).
template <int NT, int KT, class W, class PP>
__device__ LsResult ls_armijo(const W& w, const PP& P, double dt, double cost, const double (&c4)[4]) {
  const sapb_solve_options& o = P.o;
  LsResult r{0, 0, 0, 0.0, cost};
  const double dell0 = c4[0], dell_a0 = c4[1], d2ell_a = c4[2], mom0 = c4[3];
  const double amax = 1.0 / o.rho;
  const double slop_rel = o.line_search_relative_slop;
  double alpha = amax, alpha_prev = amax, ell_prev = cost;
  double ell_slop = (slop_rel / 10.0) * fmax(1.0, fabs(cost));
  r.alpha = alpha;
  if (o.line_search_max_iterations <= 0) return r;
  if (dell0 >= 0.0 || !isfinite(dell0)) {
    r.status = SAPB_LS_ASCENT_DIRECTION;
    return r;
  }
  // Trial steps amax * rho^k, evaluated 4 KT at a time (the same products as
  // the sequential backtracking, so the same decisions).
  constexpr int NB = 4 * KT;
  double al[NB], rg[NB], p0;
  al[0] = alpha;
  for (int q = 1; q < NB; ++q) al[q] = al[q - 1] * o.rho;
  line_termsK<NT, KT>(w, P, dt, al, rg, &p0);
  int base = 0;
  double ell = mom0 + alpha * dell_a0 + 0.5 * alpha * alpha * d2ell_a + rg[0];
  const double deriv = dell_a0 + alpha * d2ell_a - p0;
  {
    const double scale = fmax(1.0, 0.5 * (fabs(ell) + fabs(cost)));
    const double slop = (slop_rel / 10.0) * scale;
    ell_slop = slop;
    if (deriv < 0.0 || deriv < slop) {
      r.accepted = 1;
      r.accepted_cost = ell;
      return r;
    }
    alpha_prev = alpha;
    ell_prev = ell;
  }
  if (o.line_search_max_iterations <= 1) return r;
  for (int iteration = 1;; ++iteration) {
    alpha = alpha * o.rho;
    if (iteration - base >= NB) {
      base = iteration;
      al[0] = alpha;
      for (int q = 1; q < NB; ++q) al[q] = al[q - 1] * o.rho;
      line_termsK<NT, KT>(w, P, dt, al, rg, &p0);
    }
    ell = mom0 + alpha * dell_a0 + 0.5 * alpha * alpha * d2ell_a + rg[iteration - base];
    const double a = alpha, a_prev = alpha_prev, e_prev = ell_prev;
    const double denom = a - a_prev;
    double dell_approx = 0.0;
    if (fabs(denom) > 0.0) dell_approx = (ell - e_prev) / denom;
    int accept = 0, accept_prev = 0;
    if (fabs(dell_approx) < ell_slop) {
      accept = 1;
    } else if (ell > e_prev && armijo_ok(a, ell, cost, dell0, o.armijo_c)) {
      accept = 1;
      if (armijo_ok(a_prev, e_prev, cost, dell0, o.armijo_c)) accept_prev = 1;
    }
    if (accept) {
      r.accepted = 1;
      r.iterations = iteration;
      r.alpha = accept_prev ? a_prev : a;
      r.accepted_cost = accept_prev ? e_prev : ell;
      return r;
    }
    if (iteration >= o.line_search_max_iterations - 1) {
      r.alpha = alpha;
      if (armijo_ok(alpha, ell, cost, dell0, o.armijo_c)) {
        r.accepted = 1;
        r.iterations = o.line_search_max_iterations;
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

// monotone_decay (fused kernel sim/contact_solve.py:2483-2667).
template <int NT, int KT, class W, class PP>
__device__ LsResult ls_monotone(const W& w, const PP& P, double dt, double cost, const double (&c4)[4]) {
  const sapb_solve_options& o = P.o;
  LsResult r{0, 0, 0, 1.0, cost};
  const double base_linear = c4[1], base_quadratic = c4[2], base0 = c4[3];
  double alpha = 1.0, trial = cost;
  constexpr int NB = 4 * KT;
  double al[NB], rg[NB], p0;
  int base = -NB;
  for (int it = 0; it < o.line_search_max_iterations; ++it) {
    if (it - base >= NB) {  // halvings evaluated 4 KT at a time
      base = it;
      al[0] = alpha;
      for (int q = 1; q < NB; ++q) al[q] = al[q - 1] * 0.5;
      line_termsK<NT, KT>(w, P, dt, al, rg, &p0);
    }
    trial = base0 + alpha * base_linear + 0.5 * alpha * alpha * base_quadratic + rg[it - base];
    r.iterations += 1;
    const double tol = 1.0e-14 + 1.0e-12 * fabs(cost);
    if (trial <= cost + tol) {
      r.accepted = 1;
      break;
    }
    alpha = alpha * 0.5;
    if (alpha < 1.0e-8) {
      r.status = SAPB_LS_ALPHA_UNDERFLOW;
      break;
    }
  }
  r.alpha = alpha;
  r.accepted_cost = r.accepted ? trial : cost;
  return r;
}

// exact_root (sim/contact_solve.py:2914-3140, driver :5700-5861).
template <int NT, class W, class PP>
__device__ LsResult ls_exact(const W& w, const PP& P, double dt, double cost, const double (&c4)[4]) {
  const sapb_solve_options& o = P.o;
  LsResult r{0, 0, 0, kExactAlphaMax, cost};
  const int max_it = o.line_search_max_iterations;
  if (max_it <= 0) return r;
  const double dell0 = c4[0], dell_a0 = c4[1], d2ell_a = c4[2], mom0 = c4[3];
  const double amax = kExactAlphaMax;
  if (dell0 >= 0.0 || !isfinite(dell0)) {
    r.status = SAPB_LS_ASCENT_DIRECTION;
    return r;
  }
  double t3[3];
  line_terms<NT>(w, P, dt, amax, true, t3);
  const double ell = mom0 + amax * dell_a0 + 0.5 * amax * amax * d2ell_a + t3[0];
  const double deriv = dell_a0 + amax * d2ell_a - t3[1];
  const double deriv2 = d2ell_a + t3[2];
  bool active = false;
  double scale = 0, x_lo = 0, x_hi = 0, f_hi = 0, root = 0, mdx = 0, mdx_prev = 0, xtol = 0;
  if (deriv <= 0.0) {
    r.accepted = 1;
    r.alpha = amax;
  } else if (-dell0 < o.cost_abs_tol + o.cost_rel_tol * ell) {
    r.accepted = 1;
    r.alpha = 1.0;
  } else {
    scale = -dell0;
    const double f_upper = deriv / scale;
    if (!isfinite(f_upper) || f_upper <= 0.0) {
      r.status = SAPB_LS_BAD_BRACKET;
    } else {
      double guess = -dell0 / deriv2;
      if (o.cubic_init) {
        const double h = amax, c0 = cost, d0 = dell0, c1 = ell, d1 = deriv;
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
      if (!isfinite(guess) || guess < 0.0 || guess > amax || kExactFTol * guess <= 0.0) {
        r.status = SAPB_LS_BAD_GUESS;
      } else {
        x_lo = 0.0;
        x_hi = amax;
        f_hi = f_upper;
        root = guess;
        mdx = -amax;
        mdx_prev = -amax;
        xtol = kExactFTol * guess;
        r.alpha = guess;
        active = true;
      }
    }
  }
  for (int iteration = 1; active; ++iteration) {
    line_terms<NT>(w, P, dt, r.alpha, true, t3);
    const double d = dell_a0 + r.alpha * d2ell_a - t3[1];
    const double d2 = d2ell_a + t3[2];
    const double f = d / scale, df = d2 / scale;
    const double f_upper = f_hi;
    if ((f < 0.0 && f_upper >= 0.0) || (f >= 0.0 && f_upper < 0.0)) {
      x_lo = root;
    } else {
      x_hi = root;
      f_hi = f;
    }
    if (fabs(f) < kExactFTol) {
      r.accepted = 1;
      r.iterations = iteration;
      r.alpha = root;
      break;
    }
    if (iteration >= max_it) {
      r.status = SAPB_LS_ROOT_ITERATION_CAP;
      break;
    }
    const bool slow = 2.0 * fabs(f) > fabs(mdx_prev * df);
    mdx_prev = mdx;
    const double bis_mdx = 0.5 * (x_lo - x_hi);
    const double bis_root = x_lo - bis_mdx;
    double n_mdx = 0.0, n_root = root;
    if (fabs(df) > 0.0) {
      n_mdx = f / df;
      n_root = root - n_mdx;
    }
    bool use_bisect = slow;
    if (n_root < x_lo || n_root > x_hi) use_bisect = true;
    if (!isfinite(n_root) || !isfinite(n_mdx)) use_bisect = true;
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
  if (r.accepted) {
    line_terms<NT>(w, P, dt, r.alpha, false, t3);
    r.accepted_cost = mom0 + r.alpha * dell_a0 + 0.5 * r.alpha * r.alpha * d2ell_a + t3[0];
  }
  return r;
}

}  // namespace sapb
