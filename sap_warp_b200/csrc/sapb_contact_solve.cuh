// sapb_contact_solve.cuh -- fused SAP stage-2 Newton solve, one CTA per world.
//
// Restates SapContactSolve.solve (sim/contact_solve.py:6129-6285) as ONE
// persistent launch.  A CTA pulls a world index from a device counter, stages
// the world's contact Jacobian J in shared memory once, and runs prepare
// (:4285-4429), the Newton loop (:5474-5655) and the chosen line search
// (:2207-3175) on chip.  The dynamics matrix A is read through L1 (it is the
// only per-world array re-read from outside shared memory; 3-4 passes per
// Newton iteration hit L1/L2).  Per line-search trial the kernel touches
// O(contacts + DOFs) data because the contact velocity along the search line
// is vc + alpha * (J dv) (vc is linear in v); the reference issues ~35
// launches per Newton iteration and re-reads A and J on every trial.
//
// Precision: the gradient, costs, line search, velocity update and the
// convergence test are FP64.  The Hessian H = A + J^T G J + diag and its LDL^T
// factorization run in HT (double, or float for the mixed path).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <type_traits>

#include "sapb_device.cuh"
#include "sapb_internal.h"
#include "sapb_ldlt.cuh"
#include "sapb_linesearch.cuh"

namespace sapb {

struct SolveParams {
  sapb_contact_problem p;
  sapb_dof_terms dof;  // copy of *p.dof (has_pd/has_limits 0 if none)
  sapb_solve_options o;
  sapb_solve_outputs out;
  int32_t use_guess_flag_ptr_valid;
  int32_t* queue;      // work counter (zeroed before launch)
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Shared-memory layout of one world.  ldJ: room for the 4-wide Hessian tiles
// and odd, so thread-per-row reads of J are free of bank conflicts.  ldH odd
// for conflict-free column reads in the factorization.
struct Layout {
  int n, C, ldJ, ldH, nb, nw;
  size_t off_J, off_scr, off_H, off_G, off_vec, off_con, off_flags, off_tri, total;
  static constexpr int kVecs = 23;
  static constexpr int kConPer = 17;
  static constexpr int kMinWarps = 4;  // partial-sum scratch of at least four warps
};

// warps: of the CTA (the partial-sum scratch holds one row per warp)
__host__ __device__ inline Layout make_layout(int n, int C, int hsize, int warps = 4) {
  Layout L;
  L.n = n;
  L.C = C;
  L.nw = warps > Layout::kMinWarps ? warps : Layout::kMinWarps;
  L.ldJ = (n + 3) / 4 * 4 + 1;
  L.ldH = (n % 2 == 0) ? n + 1 : n;
  L.nb = (n + 3) / 4;
  size_t o = 0;
  L.off_J = o;
  o = align_up(o + sizeof(double) * (size_t)3 * C * L.ldJ, 16);
  L.off_scr = o;  // the partial sums of the DOF products, or two staged impulse sets
  {
    const size_t part = sizeof(double) * 3 * (size_t)L.nw * 64;
    const size_t gam = sizeof(double) * 6 * (size_t)(C > 0 ? C : 1);
    o = align_up(o + (part > gam ? part : gam), 16);
  }
  L.off_H = o;
  o = align_up(o + (size_t)hsize * n * L.ldH, 16);
  L.off_G = o;
  o = align_up(o + (size_t)hsize * 9 * (size_t)(C > 0 ? C : 1), 16);
  L.off_vec = o;
  o = align_up(o + sizeof(double) * (size_t)Layout::kVecs * L.ldJ, 16);
  L.off_con = o;
  o = align_up(o + sizeof(double) * (size_t)Layout::kConPer * (C > 0 ? C : 1), 16);
  L.off_flags = o;
  o = align_up(o + sizeof(int) * (size_t)L.ldJ, 16);
  L.off_tri = o;  // (i << 8 | j) of the lower triangle below row 0, columns descending
  o = align_up(o + sizeof(uint16_t) * (size_t)(n * (n - 1) / 2 + 1), 16);
  L.total = o;
  return L;
}

static_assert(V_END <= Layout::kVecs, "vector slots");
static_assert(C_END <= Layout::kConPer, "contact slots");

template <int NT, typename HT, int NS>
struct World {
  Layout L;
  const double* A;  // global, this world's [n][n]
  double* J;
  HT* GJ;           // scratch: the partial sums of the DOF products, or staged impulse sets
  HT* H;
  HT* G;            // [C][9], in the Hessian's type
  double* vec;
  double* con;
  int* flags;
  const uint16_t* tri;
  double* red;
  int* factor_ok;  // shared: whether the last Newton factorization's pivots were all positive and finite
  int n, count;
  // DOF count and leading dimensions: compile-time constants when NS > 0.
  __device__ __forceinline__ int dofs() const { return NS > 0 ? NS : n; }
  __device__ __forceinline__ int ldJ() const { return NS > 0 ? (NS + 3) / 4 * 4 + 1 : L.ldJ; }
  __device__ __forceinline__ int ldH() const { return NS > 0 ? ((NS % 2 == 0) ? NS + 1 : NS) : L.ldH; }
  __device__ __forceinline__ int nb() const { return NS > 0 ? (NS + 3) / 4 : (n + 3) / 4; }
  // shift of the kernel's triangle list (built for L.n DOFs) to this world's n
  __device__ __forceinline__ int tri_shift() const { return L.n - dofs(); }
  __device__ double* V(int k) const { return vec + (size_t)k * ldJ(); }
  __device__ double* Cn(int k) const { return con + (size_t)k * L.C; }
  __device__ double* part(int which, int warp) const {
    return reinterpret_cast<double*>(GJ) + ((size_t)which * L.nw + warp) * 64;
  }
  __device__ ContactConst cc(int c) const {
    ContactConst x;
    x.rt = Cn(C_RT)[c];
    x.rn = Cn(C_RN)[c];
    x.rt_inv = Cn(C_RTINV)[c];
    x.rn_inv = Cn(C_RNINV)[c];
    x.vhat_n = Cn(C_VHAT)[c];
    x.mu = Cn(C_MU)[c];
    x.mu_hat = Cn(C_MUHAT)[c];
    x.factor = Cn(C_FACTOR)[c];
    return x;
  }
};

// vc-type products: rows r < 3*count of J times x (length n, shared) into the
// contact slots `slot..slot+2`.  One thread per row.
template <int NT, typename HT, int NS>
__device__ void contact_rows_times(const World<NT, HT, NS>& w, const double* x, int slot) {
  const int rows = 3 * w.count;
  for (int r = threadIdx.x; r < rows; r += NT) {
    const double* row = w.J + (size_t)r * w.ldJ();
    double s0 = 0.0, s1 = 0.0;
    int j = 0;
    for (; j + 1 < w.dofs(); j += 2) {
      s0 += row[j] * x[j];
      s1 += row[j + 1] * x[j + 1];
    }
    if (j < w.dofs()) s0 += row[j] * x[j];
    const int c = r / 3, k = r - 3 * c;
    w.Cn(slot + k)[c] = s0 + s1;
  }
}

// Partial sums of the per-DOF products over a warp's share of the columns of
// A and of the contacts: part(0)[i] = sum_j A[j][i] x[j], part(1)[i] =
// sum_j A[j][i] y[j], part(2)[i] = sum_c J_c[:, i] . gamma_c.  Lanes own DOFs
// i = lane and lane + 32, so a warp reads consecutive addresses.
template <int NT, typename HT, int NS>
__device__ void dof_partials(const World<NT, HT, NS>& w, const double* x, const double* y, bool with_gamma) {
  constexpr int NW = NT / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int n = w.dofs();
  const int jchunk = (n + NW - 1) / NW;
  const int j0 = warp * jchunk, j1 = min(n, j0 + jchunk);
  const int cchunk = (w.count + NW - 1) / NW;
  const int c0 = warp * cchunk, c1 = min(w.count, c0 + cchunk);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int i = lane + 32 * h;
    if (i >= n) continue;
    double a = 0.0, b = 0.0, g = 0.0;
    for (int j = j0; j < j1; ++j) {
      const double aij = __ldg(w.A + (size_t)j * n + i);
      a += aij * x[j];
      if (y) b += aij * y[j];
    }
    if (with_gamma) {
      const int ld = w.ldJ();
      for (int c = c0; c < c1; ++c) {
        const double* Jc = w.J + (size_t)(3 * c) * ld + i;
        g += Jc[0] * w.Cn(C_GAMMA + 0)[c] + Jc[ld] * w.Cn(C_GAMMA + 1)[c] + Jc[2 * ld] * w.Cn(C_GAMMA + 2)[c];
      }
    }
    w.part(0, warp)[i] = a;
    w.part(1, warp)[i] = b;
    w.part(2, warp)[i] = g;
  }
}

template <int NT, typename HT, int NS>
__device__ __forceinline__ double sum_partials(const World<NT, HT, NS>& w, int which, int i) {
  constexpr int NW = NT / 32;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < NW; ++k) s += w.part(which, k)[i];
  return s;
}

// Objective at the current v (shared V_V): contact gamma and cost, A(v-v*),
// J^T gamma, PD and limit terms, gradient.  Returns {cost, |g|^2, |p|^2, |jc|^2}
// (scaled, over participating DOFs) to every thread.  Restates
// _solver_update_active sim/contact_solve.py:4080-4136.
template <int NT, typename HT, int NS>
__device__ void evaluate(const World<NT, HT, NS>& w, const SolveParams& P, double dt, double out4[4]) {
  const int tid = threadIdx.x;
  contact_rows_times<NT, HT, NS>(w, w.V(V_V), C_VC);
  for (int i = tid; i < w.dofs(); i += NT) w.V(V_TMP0)[i] = w.V(V_V)[i] - w.V(V_VSTAR)[i];
  __syncthreads();
  double csum = 0.0;
  for (int c = tid; c < w.count; c += NT) {
    double g[3], cost;
    project_contact(w.cc(c), w.Cn(C_VC + 0)[c], w.Cn(C_VC + 1)[c], w.Cn(C_VC + 2)[c], g, &cost, nullptr);
    w.Cn(C_GAMMA + 0)[c] = g[0];
    w.Cn(C_GAMMA + 1)[c] = g[1];
    w.Cn(C_GAMMA + 2)[c] = g[2];
    csum += cost;
  }
  __syncthreads();
  dof_partials<NT, HT, NS>(w, w.V(V_TMP0), w.V(V_V), true);
  __syncthreads();
  double model_cost = 0.0, g2 = 0.0, p2 = 0.0, j2 = 0.0;
  const double* v = w.V(V_V);
  const double* vs = w.V(V_VSTAR);
  for (int i = tid; i < w.dofs(); i += NT) {
    const double a_res = sum_partials<NT, HT, NS>(w, 0, i);
    const double a_v = sum_partials<NT, HT, NS>(w, 1, i);
    double imp = sum_partials<NT, HT, NS>(w, 2, i);
    const double vi = v[i];
    double mc = 0.5 * (vi - vs[i]) * a_res;
    const int fl = w.flags[i];
    double pdg = 0.0, hd = 0.0;
    if (P.dof.has_pd && (fl & kFlagPd)) {
      const double gain = w.V(V_PDGAIN)[i], lim = w.V(V_PDLIM)[i];
      const double y = w.V(V_PDA)[i] - gain * vi;
      pdg = dt * clamp_limit(y, lim);
      hd += dt * gain * clamp_limit_derivative(y, lim);
      if (gain > 0.0) mc += (dt / gain) * clamp_limit_antiderivative(y, lim);
    }
    double lg = 0.0;
    if (P.dof.has_limits) {
      double lc = 0.0;
      if (fl & kFlagLo) {
        const double g = w.V(V_LORINV)[i] * (w.V(V_LOVHAT)[i] - vi);
        if (g > 0.0) {
          lg += g;
          hd += w.V(V_LORINV)[i];
          lc += 0.5 * w.V(V_LOR)[i] * g * g;
        }
      }
      if (fl & kFlagUp) {
        const double g = w.V(V_UPRINV)[i] * (w.V(V_UPVHAT)[i] + vi);
        if (g > 0.0) {
          lg -= g;
          hd += w.V(V_UPRINV)[i];
          lc += 0.5 * w.V(V_UPR)[i] * g * g;
        }
      }
      mc += lc;
    }
    imp += pdg + lg;
    const double grad = a_res - imp;
    w.V(V_ARES)[i] = a_res;
    w.V(V_GRAD)[i] = grad;
    w.V(V_HDIAG)[i] = hd;
    model_cost += mc;
    if (fl & kFlagPart) {
      const double s = w.V(V_DSCALE)[i];
      const double gs = s * grad, ps = s * a_v, js = s * imp;
      g2 += gs * gs;
      p2 += ps * ps;
      j2 += js * js;
    }
  }
  double r[4] = {csum + model_cost, g2, p2, j2};
  block_sum<NT, 4>(r, w.red);
  out4[0] = r[0];
  out4[1] = r[1];
  out4[2] = r[2];
  out4[3] = r[3];
}

// H (lower triangle, HT) <- the lower triangle of the FP64 n x n matrix M in
// global memory (+ diag_add on the diagonal): flat coalesced reads, four
// loads in flight per thread.
template <int NT, typename HT, int NS>
__device__ __forceinline__ void load_lower(const World<NT, HT, NS>& w, const double* M, const double* diag_add,
                                           double shift) {
  const int tid = threadIdx.x;
  const int n = w.dofs(), ldH = w.ldH();
  const int total = n * n;
  for (int k0 = tid; k0 < total; k0 += 4 * NT) {
    double val[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = k0 + u * NT;
      val[u] = k < total ? __ldg(M + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int k = k0 + u * NT;
      if (k < total) {
        const int i = k / n, j = k - i * n;
        if (j < i) w.H[(size_t)i * ldH + j] = HT(val[u]);
        else if (j == i) w.H[(size_t)i * ldH + j] = HT(val[u] + (diag_add ? diag_add[i] : 0.0) + shift);
      }
    }
  }
}

// H = A + J^T G J + diag(PD + limit + shift), lower triangle, in HT.
// G at the stored vc per contact; each thread owns one 4x4 tile of H and one
// of KS slices of the contacts and accumulates J_c^T (G_c J_c) for its tile
// in registers (G J formed per contact for the tile's columns: no staging,
// no barriers between contacts); the slices of a tile are summed by warp
// shuffles (KS a power of two) or add into H in turn, in a fixed order
// (deterministic).
template <int NT, typename HT, int NS>
__device__ void assemble_hessian(const World<NT, HT, NS>& w, double diag_shift) {
  const int tid = threadIdx.x;
  const int n = w.dofs(), ldJ = w.ldJ(), ldH = w.ldH(), nb = w.nb();
  // G at the current contact velocities (sim/contact_solve.py:1071-1217).
  for (int c = tid; c < w.count; c += NT) {
    double g[3], cost, G[9];
    project_contact(w.cc(c), w.Cn(C_VC + 0)[c], w.Cn(C_VC + 1)[c], w.Cn(C_VC + 2)[c], g, &cost, G);
#pragma unroll
    for (int k = 0; k < 9; ++k) w.G[9 * c + k] = HT(G[k]);
  }
  // H lower = A lower + diagonal terms
  load_lower<NT, HT, NS>(w, w.A, w.V(V_HDIAG), diag_shift);
  const int tiles = nb * (nb + 1) / 2;
  int ks = NT / (tiles > 0 ? tiles : 1);
  if (ks < 1) ks = 1;
  if (ks > 4) ks = 4;
  const int items = tiles * ks;
  // This thread's item (a thread holds at most one: items <= NT is checked
  // on the host; n <= 64 gives tiles <= 136, ks >= 1).
  const bool has_item = tid < items;
  int bi = 0, bj = 0, slice = 0;
  if (has_item) {
    const int t = tid / ks;
    slice = tid - t * ks;
    while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
    bj = t - bi * (bi + 1) / 2;
  }
  HT acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) acc[a][b] = HT(0);
  __syncthreads();  // G ready, H initialised
  if (has_item) {
    // this slice's contacts; per contact G J for the tile's 4 columns, then
    // the tile's rank-3 update J_c[:, 4 bi..]^T (G J_c)[:, 4 bj..]
    const int per = (w.count + ks - 1) / ks;
    const int c0 = slice * per, c1 = min(w.count, c0 + per);
    for (int c = c0; c < c1; ++c) {
      const double* Jc = w.J + (size_t)(3 * c) * ldJ;
      HT ja[3][4], jb[3][4], G[9];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          ja[k][q] = HT(Jc[(size_t)k * ldJ + 4 * bi + q]);
          jb[k][q] = HT(Jc[(size_t)k * ldJ + 4 * bj + q]);
        }
#pragma unroll
      for (int k = 0; k < 9; ++k) G[k] = w.G[9 * c + k];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        HT gj[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) gj[q] = G[3 * k] * jb[0][q] + G[3 * k + 1] * jb[1][q] + G[3 * k + 2] * jb[2][q];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[a][q] += ja[k][a] * gj[q];
      }
    }
  }
  auto add_tile = [&]() {
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = 4 * bi + a;
      if (i >= n) continue;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int j = 4 * bj + b;
        if (j > i || j >= n) continue;
        w.H[(size_t)i * ldH + j] += acc[a][b];
      }
    }
  };
  if ((ks & (ks - 1)) == 0) {
    // the ks slices of a tile are ks consecutive lanes of one warp: sum them
    // by shuffles (fixed order), slice 0 adds the tile
    for (int o = ks >> 1; o > 0; o >>= 1) {
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += __shfl_down_sync(0xffffffffu, acc[a][b], o);
    }
    if (has_item && slice == 0) add_tile();
    __syncthreads();
  } else {
    for (int s = 0; s < ks; ++s) {
      if (has_item && slice == s) add_tile();
      __syncthreads();
    }
  }
}

// Newton direction dv = -H^-1 grad: in-place LDL^T of the lower triangle of
// H (unit L stored below the diagonal unscaled as H_ik = L_ik d_k, D on the
// diagonal, 1/d_k in V_DINV) by the whole block (ldlt_blocked), then the two
// triangular solves by warp 0 (ldlt_solve_warp).  Mathematically the
// Cholesky solve of the reference's BlockCholeskySolverBatched
// (sim/blocked_cholesky.py:414-604).  (A single-warp factorization measured
// 3x slower than the block-wide one on 35 x 35: its 35 dependent steps each
// wait on a shuffle and a shared-memory round trip.  A four-column blocked
// warp solve measured no faster than the column-by-column one.)  A pivot
// that is not positive / finite makes dv NaN.
template <int NT, typename HT, int NS, int LB>
__device__ void factor_and_solve(const World<NT, HT, NS>& w) {
  HT* dinv = reinterpret_cast<HT*>(w.V(V_DINV));
  ldlt_blocked<NT, HT, LB>(w.H, w.dofs(), w.ldH(), dinv, w.tri, w.tri_shift());
  if ((threadIdx.x >> 5) == 0) {
    const bool ok = ldlt_pivots_ok_warp<HT>(w.H, w.dofs(), w.ldH());
    if (threadIdx.x == 0) *w.factor_ok = ok ? 1 : 0;
    ldlt_solve_warp<HT>(w.H, w.dofs(), w.ldH(), dinv, w.V(V_GRAD), w.V(V_DV), true, ok);
  }
  __syncthreads();
}

// out = -H^-1 rhs (vector slots) with the LDL^T in H and V_DINV, by warp
// `warp` alone (no block barrier).  A pivot that is not positive / finite
// makes out NaN.
template <int NT, typename HT, int NS>
__device__ void solve_warp(const World<NT, HT, NS>& w, int rhs_slot, int out_slot, int warp) {
  if ((threadIdx.x >> 5) == warp) {
    const HT* dinv = reinterpret_cast<const HT*>(w.V(V_DINV));
    const bool ok = ldlt_pivots_ok_warp<HT>(w.H, w.dofs(), w.ldH());
    ldlt_solve_warp<HT>(w.H, w.dofs(), w.ldH(), dinv, w.V(rhs_slot), w.V(out_slot), true, ok);
  }
}

// Line coefficients (sim/contact_solve.py:2234-2263, 1657-1692):
// dp = A dv, dvc = J dv and {dell0, dell_a0, d2ell_a, mom0}.
template <int NT, typename HT, int NS>
__device__ void line_coefficients(const World<NT, HT, NS>& w, double c4[4]) {
  const int tid = threadIdx.x;
  contact_rows_times<NT, HT, NS>(w, w.V(V_DV), C_DVC);
  dof_partials<NT, HT, NS>(w, w.V(V_DV), nullptr, false);
  __syncthreads();
  double d0 = 0.0, da0 = 0.0, d2 = 0.0, m0 = 0.0;
  const double* v = w.V(V_V);
  const double* vs = w.V(V_VSTAR);
  const double* dv = w.V(V_DV);
  for (int i = tid; i < w.dofs(); i += NT) {
    const double acc = sum_partials<NT, HT, NS>(w, 0, i);
    w.V(V_DP)[i] = acc;
    const double ri = v[i] - vs[i];
    d0 += w.V(V_GRAD)[i] * dv[i];
    da0 += acc * ri;
    d2 += dv[i] * acc;
    m0 += 0.5 * ri * w.V(V_ARES)[i];
  }
  double r[4] = {d0, da0, d2, m0};
  block_sum<NT, 4>(r, w.red);  // its barriers also publish dvc / dp
  c4[0] = r[0];
  c4[1] = r[1];
  c4[2] = r[2];
  c4[3] = r[3];
}

template <int NS> struct LdltBlocks { static constexpr int kCount = 1; static constexpr int kW[1] = {4}; };
template <> struct LdltBlocks<35> { static constexpr int kCount = 2; static constexpr int kW[2] = {5, 4}; };
template <> struct LdltBlocks<18> { static constexpr int kCount = 2; static constexpr int kW[2] = {6, 4}; };
template <> struct LdltBlocks<13> { static constexpr int kCount = 2; static constexpr int kW[2] = {4, 5}; };
template <> struct LdltBlocks<6> { static constexpr int kCount = 1; static constexpr int kW[1] = {6}; };

// One world of the persistent solve: stage its J and constants, the
// candidate starts, the Newton loop, the outputs.  NS: the world's DOF count
// at compile time (0: n_rt at run time); the shared-memory layout L may be
// sized for more DOFs (n_max) than the world has.
template <int NT, typename HT, int NS, int LSV, int LB>
__device__ __forceinline__ void solve_world(const SolveParams& P, const Layout& L, unsigned char* smem, double* red,
                                            unsigned long long& s_partmask, int& s_factor_ok, const int e,
                                            const int n_max, const int n_rt, const bool use_guess) {
  const int tid = threadIdx.x;
  const int C = P.p.max_contacts;
  const int n = NS > 0 ? NS : n_rt;
  World<NT, HT, NS> w{L,
                  P.p.dynamics_matrix + (size_t)e * n_max * n_max,
                  reinterpret_cast<double*>(smem + L.off_J),
                  reinterpret_cast<HT*>(smem + L.off_scr),
                  reinterpret_cast<HT*>(smem + L.off_H),
                  reinterpret_cast<HT*>(smem + L.off_G),
                  reinterpret_cast<double*>(smem + L.off_vec),
                  reinterpret_cast<double*>(smem + L.off_con),
                  reinterpret_cast<int*>(smem + L.off_flags),
                  reinterpret_cast<const uint16_t*>(smem + L.off_tri),
                  red,
                  &s_factor_ok,
                  n,
                  0};
  int count = P.p.contact_count[e];
  if (count > C) count = C;
  if (count < 0) count = 0;
  w.count = count;
  const double dt = P.p.dt[e];
  const size_t base = (size_t)e * n_max;

  // ---- stage J, per-contact constants and vectors -------------------------
  {
    const int rows = 3 * count;
    const double* Jg = P.p.jacobian + (size_t)e * C * 3 * n_max;
    const int ldj = w.ldJ();
    // Flat copy of the contiguous rows*n block by asynchronous 8-byte
    // copies (all in flight at once, completed before the barrier after the
    // per-DOF setup below; the rows land at stride ldj).
    const int total = rows * n;
    for (int k = tid; k < total; k += NT) {
      const int r = k / n, j = k - r * n;
      const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(w.J + (size_t)r * ldj + j));
      asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(Jg + k) : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    // zero padding columns n..ldj-1
    for (int k = tid; k < rows * (ldj - n); k += NT) {
      const int r = k / (ldj - n), j = n + (k - r * (ldj - n));
      w.J[(size_t)r * ldj + j] = 0.0;
    }
    for (int c = tid; c < count; c += NT) {
      const size_t ci = (size_t)e * C + c;
      const double tau = P.p.tau_d ? P.p.tau_d[ci] : P.o.contact_tau_d;
      const ContactConst cc = make_contact_const(P.p.phi0[ci], P.p.w_eff[ci], P.p.mu[ci], P.p.stiffness[ci], tau,
                                                 P.o.contact_beta, P.o.contact_sigma, dt);
      w.Cn(C_RT)[c] = cc.rt;
      w.Cn(C_RN)[c] = cc.rn;
      w.Cn(C_RTINV)[c] = cc.rt_inv;
      w.Cn(C_RNINV)[c] = cc.rn_inv;
      w.Cn(C_VHAT)[c] = cc.vhat_n;
      w.Cn(C_MU)[c] = cc.mu;
      w.Cn(C_MUHAT)[c] = cc.mu_hat;
      w.Cn(C_FACTOR)[c] = cc.factor;
    }
    for (int i = tid; i < w.ldJ(); i += NT) {
      if (i < n) {
        w.V(V_VSTAR)[i] = P.p.v_star[base + i];
        double v = P.p.v0[base + i];
        if (P.p.v_guess) {
          if (use_guess) v = P.p.v_guess[base + i];
          P.p.v_guess[base + i] = v;
        }
        w.V(V_V)[i] = v;
        double d = __ldg(w.A + (size_t)i * n + i);
        if (d < 1.0e-12 || !isfinite(d)) d = 1.0e-12;
        w.V(V_AINV)[i] = 1.0 / d;
        w.V(V_DSCALE)[i] = 1.0 / sqrt(d);
      } else {
        for (int k = 0; k < Layout::kVecs; ++k) w.V(k)[i] = 0.0;
      }
    }
  }
  // ---- PD and limit terms (sim/contact_solve.py:490-683) ------------------
  for (int i = tid; i < n; i += NT) {
    int fl = 0;
    const sapb_dof_terms& D = P.dof;
    // the per-DOF arrays: the solve's layout, or the model's global DOF order
    const size_t dof = D.world_dof_start ? (size_t)D.world_dof_start[e] + i : base + i;
    if (D.has_pd) {
      int coord = D.dof_coord_index[dof];
      if (coord >= D.joint_coord_count) coord = -1;
      int target = D.dof_target_index[dof];
      const int ndof = D.world_dof_start ? D.world_dof_start[P.p.num_envs] : P.p.num_envs * n_max;
      if (target < 0 || target >= ndof) target = (int)dof;
      if (D.joint_target_mode[target] != 0) {
        const double kp = (double)D.joint_target_ke[target], kd = (double)D.joint_target_kd[target];
        if (!(kp <= 0.0 && kd <= 0.0) && !(coord < 0 && kp > 0.0)) {
          double kpe, kde;
          effective_pd_gains(kp, kd, dt, w.V(V_AINV)[i], &kpe, &kde);
          const double gain = dt * kpe + kde;
          if (gain > 0.0) {
            double q0 = 0.0, qd = 0.0;
            if (coord >= 0) {
              q0 = D.joint_q[coord];
              qd = D.joint_target_pos ? (double)D.joint_target_pos[target] : 0.0;
            }
            const double vd = D.joint_target_vel ? (double)D.joint_target_vel[target] : 0.0;
            const double u0 = D.joint_act ? (double)D.joint_act[target] : 0.0;
            fl |= kFlagPd;
            w.V(V_PDA)[i] = kpe * (qd - q0) + kde * vd + u0;
            w.V(V_PDGAIN)[i] = gain;
            w.V(V_PDLIM)[i] = (double)D.joint_effort_limit[target];
          }
        }
      }
    }
    w.V(V_LOR)[i] = 1.0;
    w.V(V_UPR)[i] = 1.0;
    if (D.has_limits) {
      int coord = D.dof_coord_index[dof];
      if (coord >= D.joint_coord_count) coord = -1;
      const double ke = coord >= 0 ? D.joint_limit_ke[dof] : 0.0;
      if (coord >= 0 && D.limit_supported[dof] != 0 && ke > 0.0) {
        const double q0 = D.joint_q[coord];
        const double lower = D.joint_limit_lower[dof], upper = D.joint_limit_upper[dof];
        const double speed = fmax(fabs(P.p.v0[base + i]), fabs(w.V(V_VSTAR)[i]));
        const double window = kLimitWindow * dt * speed;
        const double kd = D.joint_limit_kd[dof];
        const double tau_d = kd > 0.0 ? kd / ke : 0.0;
        const double bf = kLimitBeta * kLimitBeta / (4.0 * kPi * kPi);
        const double r_nr = bf * fmax(w.V(V_AINV)[i], 1.0e-12);
        const double r_soft = 1.0 / (dt * ke * (dt + tau_d));
        const double rr = fmax(r_nr, r_soft);
        if (isfinite(lower) && q0 - lower <= window) {
          fl |= kFlagLo;
          w.V(V_LOVHAT)[i] = -(q0 - lower) / (dt + tau_d);
          w.V(V_LOR)[i] = rr;
          w.V(V_LORINV)[i] = 1.0 / rr;
        }
        if (isfinite(upper) && upper - q0 <= window) {
          fl |= kFlagUp;
          w.V(V_UPVHAT)[i] = -(upper - q0) / (dt + tau_d);
          w.V(V_UPR)[i] = rr;
          w.V(V_UPRINV)[i] = 1.0 / rr;
        }
      }
    }
    w.flags[i] = fl;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");  // this thread's J copies
  __syncthreads();
  // ---- participating DOFs (sim/contact_solve.py:423-488) ------------------
  // A DOF takes part if a model term acts on it or a contact's body DOF
  // range or J column covers it.  The contacts mark their DOFs in a 64-bit
  // mask in parallel (n <= 60 here).
  if (tid == 0) s_partmask = 0ull;
  __syncthreads();
  for (int c = tid; c < count; c += NT) {
    const size_t ci = (size_t)e * C + c;
    unsigned long long mk = 0ull;
    if (P.p.body_dof_start) {
      const int bs[2] = {P.p.body0 ? P.p.body0[ci] : -1, P.p.body1 ? P.p.body1[ci] : -1};
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int b = bs[q];
        if (b < 0 || b >= P.p.num_bodies) continue;
        const int s = P.p.body_dof_start[b], m = P.p.body_dof_count[b];
        if (s < 0 || m <= 0 || s >= n) continue;
        const int hi = s + m < n ? s + m : n;
        mk |= ((1ull << (hi - s)) - 1ull) << s;
      }
    }
    const double* Jc = w.J + (size_t)(3 * c) * w.ldJ();
    if (mk != (1ull << n) - 1ull)
      for (int j = 0; j < n; ++j)
        if (Jc[j] != 0.0 || Jc[w.ldJ() + j] != 0.0 || Jc[2 * w.ldJ() + j] != 0.0) mk |= 1ull << j;
    atomicOr(&s_partmask, mk);
  }
  __syncthreads();
  int any_model_term = 0;
  for (int i = tid; i < n; i += NT) {
    const int model = (w.flags[i] & (kFlagPd | kFlagLo | kFlagUp)) ? 1 : 0;
    any_model_term |= model;
    if (model || ((s_partmask >> i) & 1ull)) w.flags[i] |= kFlagPart;
  }
  const int model_terms = __syncthreads_or(any_model_term);
  const bool unconstrained = (count == 0) && !model_terms;
  // ---- input check: a NaN / Inf in A, J, the contact parameters, v* or
  // the start velocity leaves the world unsolved (SAPB_WORLD_NOT_FINITE)
  int bad = 0;
  for (int k = tid; k < n * n; k += NT)
    if (!isfinite(__ldg(w.A + k))) bad = 1;
  {
    const int ldj = w.ldJ(), tot = 3 * count * n;
    for (int k = tid; k < tot; k += NT) {
      const int r = k / n, j = k - r * n;
      if (!isfinite(w.J[(size_t)r * ldj + j])) bad = 1;
    }
  }
  for (int c = tid; c < count; c += NT) {
    const size_t ci = (size_t)e * C + c;
    if (!isfinite(P.p.phi0[ci]) || !isfinite(P.p.w_eff[ci]) || !isfinite(P.p.mu[ci]) ||
        !isfinite(P.p.stiffness[ci]) || (P.p.tau_d && !isfinite(P.p.tau_d[ci])))
      bad = 1;
  }
  for (int i = tid; i < n; i += NT)
    if (!isfinite(w.V(V_VSTAR)[i]) || !isfinite(w.V(V_V)[i])) bad = 1;
  const bool not_finite = __syncthreads_or(bad) != 0;

  int newton_iterations = 0, ls_total = 0, converged = 0, status = 0;
  double cost = 0.0, previous_cost = 0.0, alpha = 1.0, grad_norm = 0.0;
  int ws_accepted = 0;
  bool evaluated = false;
  if (not_finite) {
    status = SAPB_WORLD_NOT_FINITE;  // v stays the start velocity
  } else if (unconstrained) {
    converged = 1;
    for (int i = tid; i < n; i += NT) w.V(V_V)[i] = w.V(V_VSTAR)[i];
    __syncthreads();
  } else {
    for (int i = tid; i < n; i += NT)
      if (!(w.flags[i] & kFlagPart)) w.V(V_V)[i] = w.V(V_VSTAR)[i];
    __syncthreads();
    // Candidate starts (no counterpart in the reference): v_candidate_count
    // start velocities, then gamma0_count impulse sets with v_c = base +
    // A^-1 J^T gamma_c (base v* or gamma0_base), each taken on the
    // participating DOFs (v* on the others), A factored once in this
    // kernel's factor precision or read from the free motion's factor;
    // the start with the lowest cost among the plain start (unless skipped)
    // and the candidates is taken.  Its evaluation seeds iteration 0 when it
    // was the last one evaluated.
    bool have_e4 = false;
    double e4_seed[4] = {0.0, 0.0, 0.0, 0.0};
    const int KV = P.p.v_candidates ? (P.p.v_candidate_count > 1 ? P.p.v_candidate_count : 1) : 0;
    const int KG = P.p.gamma0 ? (P.p.gamma0_count > 1 ? P.p.gamma0_count : 1) : 0;
    if ((KV > 0 || KG > 0) && count > 0) {
      // the plain start competes unless the caller skips it; it stays the
      // fallback when no candidate's cost is finite
      double best_cost = 1.0e300;
      if (!P.o.skip_plain_start) {
        double e4p[4];
        evaluate<NT, HT, NS>(w, P, dt, e4p);
        best_cost = e4p[0];
      }
      for (int i = tid; i < n; i += NT) w.V(V_SAVE)[i] = w.V(V_V)[i];
      bool last_is_best = false;
      auto try_start = [&](int index) {  // V(V_V) holds the candidate
        __syncthreads();
        double e4c[4];
        evaluate<NT, HT, NS>(w, P, dt, e4c);
        last_is_best = false;
        if (e4c[0] < best_cost) {
          best_cost = e4c[0];
          ws_accepted = index;
          last_is_best = true;
          for (int q = 0; q < 4; ++q) e4_seed[q] = e4c[q];
          for (int i = tid; i < n; i += NT) w.V(V_BEST)[i] = w.V(V_V)[i];
        }
      };
      for (int k = 0; k < KV; ++k) {
        const double* vk = P.p.v_candidates + ((size_t)k * P.p.num_envs + e) * n_max;
        for (int i = tid; i < n; i += NT)
          w.V(V_V)[i] = (w.flags[i] & kFlagPart) ? __ldg(vk + i) : w.V(V_VSTAR)[i];
        try_start(k + 1);
      }
      if (KG > 0) {
        const double* base_g = P.p.gamma0_base ? P.p.gamma0_base + (size_t)e * n_max : nullptr;
        // a world whose candidate impulses are all zero starts at the base
        int nz = 0;
        for (int q = tid; q < KG * 3 * count; q += NT) {
          const int kk = q / (3 * count), r = q - kk * 3 * count;
          if (__ldg(P.p.gamma0 + ((size_t)kk * P.p.num_envs + e) * C * 3 + r) != 0.0) nz = 1;
        }
        if (!__syncthreads_or(nz)) {
          for (int i = tid; i < n; i += NT)
            w.V(V_V)[i] = (w.flags[i] & kFlagPart) && base_g ? __ldg(base_g + i) : w.V(V_VSTAR)[i];
          try_start(KV + 1);
        } else {
          const int ldj = w.ldJ();
          if (P.p.dynamics_factor) {
            // the free motion's LDL^T of A
            const double* Lg = P.p.dynamics_factor + (size_t)e * n_max * n_max;
            load_lower<NT, HT, NS>(w, Lg, nullptr, 0.0);
            HT* dinv = reinterpret_cast<HT*>(w.V(V_DINV));
            for (int i = tid; i < n; i += NT) dinv[i] = fast_recip(HT(__ldg(Lg + (size_t)i * n + i)));
            __syncthreads();
          } else {
            load_lower<NT, HT, NS>(w, w.A, nullptr, 0.0);
            __syncthreads();
            ldlt_blocked<NT, HT, LB>(w.H, n, w.ldH(), reinterpret_cast<HT*>(w.V(V_DINV)), w.tri,
                                     w.tri_shift());  // the factor of A
          }
          // Two sets at a time: stage their impulses in the (here unused)
          // scratch, form J^T gamma for both (threads 0-63 set k0, 64-127
          // set k0+1), solve both with the factor on warps 0 and 1, then
          // evaluate the candidates in order.
          double* gs = reinterpret_cast<double*>(w.GJ);
          for (int k0 = 0; k0 < KG; k0 += 2) {
            const int nk = KG - k0 < 2 ? KG - k0 : 2;
            for (int q = tid; q < nk * 3 * count; q += NT) {
              const int kk = q / (3 * count), r = q - kk * 3 * count;
              gs[q] = __ldg(P.p.gamma0 + ((size_t)(k0 + kk) * P.p.num_envs + e) * C * 3 + r);
            }
            __syncthreads();
            {
              const int kk = tid >> 6, i = tid & 63;
              if (kk < nk && i < n) {
                const double* g = gs + kk * 3 * count;
                double acc = 0.0;
                for (int c = 0; c < count; ++c) {
                  const double* Jc = w.J + (size_t)(3 * c) * ldj;
                  acc += Jc[i] * g[3 * c] + Jc[ldj + i] * g[3 * c + 1] + Jc[2 * ldj + i] * g[3 * c + 2];
                }
                w.V(kk == 0 ? V_GRAD : V_DP)[i] = -acc;  // the solves give -H^-1 rhs
              }
            }
            __syncthreads();
            solve_warp<NT, HT, NS>(w, V_GRAD, V_DV, 0);
            if (nk > 1) solve_warp<NT, HT, NS>(w, V_DP, V_DV2, 1);
            __syncthreads();
            for (int kk = 0; kk < nk; ++kk) {
              const double* dvk = w.V(kk == 0 ? V_DV : V_DV2);
              for (int i = tid; i < n; i += NT)
                w.V(V_V)[i] = (w.flags[i] & kFlagPart)
                                  ? (base_g ? __ldg(base_g + i) : w.V(V_VSTAR)[i]) + dvk[i]
                                  : w.V(V_VSTAR)[i];
              try_start(KV + k0 + kk + 1);
            }
          }
        }
      }
      if (last_is_best) {
        have_e4 = true;
      } else {
        const int src = ws_accepted > 0 ? V_BEST : V_SAVE;
        for (int i = tid; i < n; i += NT) w.V(V_V)[i] = w.V(src)[i];
      }
      __syncthreads();
    }
    const double cost_min_alpha = LSV == SAPB_LS_MONOTONE_DECAY ? 0.0 : 0.5;
    int it = 0;
    bool active = true;
    for (;;) {
      double e4[4];
      if (have_e4) {
        for (int k = 0; k < 4; ++k) e4[k] = e4_seed[k];
        have_e4 = false;
      } else {
        evaluate<NT, HT, NS>(w, P, dt, e4);
      }
      evaluated = true;
      cost = e4[0];
      // convergence test (sim/contact_solve.py:2043-2087)
      const double gn = sqrt(fmax(e4[1], 0.0)), pn = sqrt(fmax(e4[2], 0.0)), jn = sqrt(fmax(e4[3], 0.0));
      grad_norm = gn;
      const double opt_tol = P.o.optimality_abs_tol + P.o.optimality_rel_tol * fmax(pn, jn);
      const bool opt = gn <= opt_tol;
      bool cost_ok = false;
      if (it > 0 && alpha > cost_min_alpha) {
        const double sc = 0.5 * (fabs(cost) + fabs(previous_cost));
        const double tol = P.o.cost_abs_tol + P.o.cost_rel_tol * sc;
        if (fabs(cost - previous_cost) < tol) cost_ok = true;
      }
      newton_iterations = it;
      if (opt || cost_ok) {
        converged = 1;
        active = false;
      } else if (it >= P.o.max_iterations) {
        active = false;
      } else {
        converged = 0;
      }
      if (!active) break;
      // Newton direction
      assemble_hessian<NT, HT, NS>(w, P.o.diag_shift);
      factor_and_solve<NT, HT, NS, LB>(w);
      if (!*w.factor_ok) {  // H not SPD (uniform: published by the barrier above)
        status = SAPB_WORLD_NOT_SPD;
        converged = 0;
        break;
      }
      LsResult r;
      double c4[4];
      line_coefficients<NT, HT, NS>(w, c4);
      if constexpr (LSV == SAPB_LS_ARMIJO_DECAY)
        r = ls_armijo<NT, 1>(w, P, dt, cost, c4);
      else if constexpr (LSV == SAPB_LS_EXACT_ROOT)
        r = ls_exact<NT>(w, P, dt, cost, c4);
      else
        r = ls_monotone<NT, 1>(w, P, dt, cost, c4);
      alpha = r.alpha;
      status = r.status;
      constexpr bool mono = LSV == SAPB_LS_MONOTONE_DECAY;
      if (r.accepted || mono) ls_total += r.iterations;
      if (r.accepted) {
        previous_cost = cost;
        for (int i = tid; i < n; i += NT) w.V(V_V)[i] += r.alpha * w.V(V_DV)[i];
      } else if (mono) {
        previous_cost = cost;
      }
      __syncthreads();
      ++it;
    }
  }
  // ---- outputs ------------------------------------------------------------
  for (int i = tid; i < n_max; i += NT) P.out.v[base + i] = i < n ? w.V(V_V)[i] : 0.0;
  for (int c = tid; c < C; c += NT) {
    const size_t ci = (size_t)e * C + c;
    const bool live = evaluated && c < count;
    if (P.out.contact_gamma) {
      P.out.contact_gamma[ci * 3 + 0] = live ? w.Cn(C_GAMMA + 0)[c] : 0.0;
      P.out.contact_gamma[ci * 3 + 1] = live ? w.Cn(C_GAMMA + 1)[c] : 0.0;
      P.out.contact_gamma[ci * 3 + 2] = live ? w.Cn(C_GAMMA + 2)[c] : 0.0;
    }
    if (P.out.contact_mode) {
      int mode = SAPB_CONTACT_MODE_NONE;
      if (live) {
        double g[3], cst;
        mode = project_contact(w.cc(c), w.Cn(C_VC + 0)[c], w.Cn(C_VC + 1)[c], w.Cn(C_VC + 2)[c], g, &cst, nullptr);
      }
      P.out.contact_mode[ci] = mode;
    }
  }
  if (tid == 0) {
    if (P.out.cost) P.out.cost[e] = evaluated ? cost : 0.0;
    if (P.out.newton_iterations) P.out.newton_iterations[e] = newton_iterations;
    if (P.out.line_search_iterations) P.out.line_search_iterations[e] = ls_total;
    if (P.out.converged) P.out.converged[e] = converged;
    if (P.out.status) P.out.status[e] = status;
    if (P.out.grad_norm) P.out.grad_norm[e] = grad_norm;
    if (P.out.warm_start_accepted) P.out.warm_start_accepted[e] = ws_accepted;
  }
  __syncthreads();
}

// LSV: the line search, fixed at compile time (SAPB_LS_ARMIJO_DECAY,
// SAPB_LS_EXACT_ROOT or SAPB_LS_MONOTONE_DECAY) so that one instantiation
// holds the code of one search only (smaller instruction footprint).  LB:
// the column-block width of the LDL^T factorization (a variant the
// autotuner chooses: the best width depends on the DOF count).
template <int NT, typename HT, int MINB, int NS, int LSV, int LB>
__global__ void __launch_bounds__(NT, MINB) contact_solve_kernel(const SolveParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[8 * (NT / 32)];
  __shared__ int s_next;
  __shared__ unsigned long long s_partmask;
  __shared__ int s_factor_ok;
  const int tid = threadIdx.x;
  // n_max: the DOF slots of a world in the arrays (and the shared-memory
  // layout); a world's own DOF count may be smaller (dof_count, generic
  // kernel only), its arrays compact at the start of its slots
  const int n_max = NS > 0 ? NS : P.p.dof_per_env, C = P.p.max_contacts;
  const Layout L = make_layout(n_max, C, (int)sizeof(HT), NT / 32);
  const bool use_guess = P.use_guess_flag_ptr_valid && P.p.v_guess_active[0] != 0;
  build_triangle_list<NT>(reinterpret_cast<uint16_t*>(smem + L.off_tri), n_max);

  if (tid == 0) s_next = atomicAdd(P.queue, 1);
  for (;;) {
    // Take the prefetched index, claim the next world and warm L2 with its A
    // and J (prefetch.global.L2 is a hint and has no alignment rule).
    __syncthreads();
    const int ticket = s_next;
    if (ticket >= P.p.num_envs) break;
    const int e = P.p.world_order ? P.p.world_order[ticket] : ticket;
    __syncthreads();
    if (tid == 0) s_next = atomicAdd(P.queue, 1);
    __syncthreads();
    if (e < 0 || e >= P.p.num_envs) continue;
    {
      const int nt = s_next;
      const int nx = nt < P.p.num_envs ? (P.p.world_order ? P.p.world_order[nt] : nt) : P.p.num_envs;
      if (nx >= 0 && nx < P.p.num_envs) {
        const char* a0 = reinterpret_cast<const char*>(P.p.dynamics_matrix + (size_t)nx * n_max * n_max);
        const size_t abytes = sizeof(double) * (size_t)n_max * n_max;
        int cnt = P.p.contact_count[nx];
        cnt = cnt < 0 ? 0 : (cnt > C ? C : cnt);
        const char* j0 = reinterpret_cast<const char*>(P.p.jacobian + (size_t)nx * C * 3 * n_max);
        const size_t jbytes = sizeof(double) * (size_t)cnt * 3 * n_max;
        for (size_t off = (size_t)tid * 128; off < abytes; off += (size_t)NT * 128)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(a0 + off));
        for (size_t off = (size_t)tid * 128; off < jbytes; off += (size_t)NT * 128)
          asm volatile("prefetch.global.L2 [%0];" ::"l"(j0 + off));
        if (P.p.v_candidates) {
          const int KV = P.p.v_candidate_count > 1 ? P.p.v_candidate_count : 1;
          const size_t vbytes = sizeof(double) * (size_t)n_max;
          for (int k = 0; k < KV; ++k) {
            const char* v0p =
                reinterpret_cast<const char*>(P.p.v_candidates + ((size_t)k * P.p.num_envs + nx) * n_max);
            for (size_t off = (size_t)tid * 128; off < vbytes; off += (size_t)NT * 128)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(v0p + off));
          }
        }
        if (P.p.gamma0) {
          if (P.p.dynamics_factor) {
            const char* f0 = reinterpret_cast<const char*>(P.p.dynamics_factor + (size_t)nx * n_max * n_max);
            for (size_t off = (size_t)tid * 128; off < abytes; off += (size_t)NT * 128)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(f0 + off));
          }
          const int K = P.p.gamma0_count > 1 ? P.p.gamma0_count : 1;
          const size_t gbytes = sizeof(double) * (size_t)cnt * 3;
          for (int k = 0; k < K; ++k) {
            const char* g0 = reinterpret_cast<const char*>(P.p.gamma0 + ((size_t)k * P.p.num_envs + nx) * C * 3);
            for (size_t off = (size_t)tid * 128; off < gbytes; off += (size_t)NT * 128)
              asm volatile("prefetch.global.L2 [%0];" ::"l"(g0 + off));
          }
        }
      }
    }

    int n_world = n_max;
    if (NS == 0 && P.p.dof_count) {
      n_world = P.p.dof_count[e];
      n_world = n_world < 1 ? 1 : (n_world > n_max ? n_max : n_world);
    }
    if constexpr (NS == 0) {
      if (P.p.dof_count) {
        // each world's own DOF count: the specialised code of its size class
        switch (n_world) {
          case 35:
            solve_world<NT, HT, 35, LSV, LdltBlocks<35>::kW[0]>(P, L, smem, red, s_partmask, s_factor_ok, e,
                                                                 n_max, 35, use_guess);
            continue;
          case 18:
            solve_world<NT, HT, 18, LSV, LdltBlocks<18>::kW[0]>(P, L, smem, red, s_partmask, s_factor_ok, e,
                                                                 n_max, 18, use_guess);
            continue;
          case 13:
            solve_world<NT, HT, 13, LSV, LdltBlocks<13>::kW[0]>(P, L, smem, red, s_partmask, s_factor_ok, e,
                                                                 n_max, 13, use_guess);
            continue;
          case 6:
            solve_world<NT, HT, 6, LSV, LdltBlocks<6>::kW[0]>(P, L, smem, red, s_partmask, s_factor_ok, e,
                                                                 n_max, 6, use_guess);
            continue;
          default:
            break;
        }
      }
    }
    solve_world<NT, HT, NS, LSV, LB>(P, L, smem, red, s_partmask, s_factor_ok, e, n_max, n_world, use_guess);
  }
}

template <int NT, typename HT, int MINB, int NS, int LSV, int LB>
cudaError_t launch_solve_ls(const SolveParams& P, cudaStream_t stream, int* blocks_out) {
  const Layout L = make_layout(P.p.dof_per_env, P.p.max_contacts, (int)sizeof(HT), NT / 32);
  auto kern = contact_solve_kernel<NT, HT, MINB, NS, LSV, LB>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
  if (err != cudaSuccess) return err;
  int dev = 0;
  err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  int sms = 0;
  err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (err != cudaSuccess) return err;
  int per_sm = 0;
  err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, L.total);
  if (err != cudaSuccess) return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (blocks_out && P.p.num_envs == 0) {  // occupancy query only
    *blocks_out = per_sm;
    return cudaSuccess;
  }
  const int k = (P.o.ctas_per_sm > 0 && P.o.ctas_per_sm < per_sm) ? P.o.ctas_per_sm : per_sm;
  int blocks = sms * k;
  if (blocks > P.p.num_envs) blocks = P.p.num_envs;
  if (blocks < 1) blocks = 1;
  if (blocks_out) *blocks_out = blocks;
  err = cudaMemsetAsync(P.queue, 0, sizeof(int32_t), stream);
  if (err != cudaSuccess) return err;
  kern<<<blocks, NT, L.total, stream>>>(P);
  return cudaGetLastError();
}

template <int NT, typename HT, int MINB, int NS, int LB>
static cudaError_t launch_solve(const SolveParams& P, cudaStream_t stream, int* blocks_out) {
  switch (P.o.line_search_variant) {
    case SAPB_LS_ARMIJO_DECAY:
      return launch_solve_ls<NT, HT, MINB, NS, SAPB_LS_ARMIJO_DECAY, LB>(P, stream, blocks_out);
    case SAPB_LS_EXACT_ROOT:
      return launch_solve_ls<NT, HT, MINB, NS, SAPB_LS_EXACT_ROOT, LB>(P, stream, blocks_out);
    default:
      return launch_solve_ls<NT, HT, MINB, NS, SAPB_LS_MONOTONE_DECAY, LB>(P, stream, blocks_out);
  }
}

// LDL^T block widths instantiated per DOF specialisation (the first is the
// default), from measurements on B200: 35 DOFs = 7 blocks of 5 is fastest
// in both precisions; wider blocks lengthen the serial diagonal chain and
// the register block, narrower ones add barriers.

// One Hessian precision of the kernels of one DOF specialisation NS (every
// line search, every LDL^T block width), instantiated in a translation unit
// of its own (sapb_solve_n*_f32.cu / _f64.cu) so they compile in parallel.
template <int NS, bool FP32>
cudaError_t launch_solve_np(const SolveParams& P, cudaStream_t stream, int* blocks_out) {
  using HT = typename std::conditional<FP32, float, double>::type;
  constexpr int MINB = FP32 ? 4 : 3;
  if constexpr (LdltBlocks<NS>::kCount > 1) {
    if (P.o.ldlt_block == LdltBlocks<NS>::kW[1])
      return launch_solve<128, HT, MINB, NS, LdltBlocks<NS>::kW[LdltBlocks<NS>::kCount > 1 ? 1 : 0]>(P, stream,
                                                                                                      blocks_out);
  }
  return launch_solve<128, HT, MINB, NS, LdltBlocks<NS>::kW[0]>(P, stream, blocks_out);  // the default (0 or unknown)
}

template <int NS>
inline cudaError_t launch_solve_ns(const SolveParams& P, bool fp32, cudaStream_t stream, int* blocks_out) {
  return fp32 ? launch_solve_np<NS, true>(P, stream, blocks_out) : launch_solve_np<NS, false>(P, stream, blocks_out);
}

// The runtime-size kernel with 256 threads (eight warps) per world, the
// default LDL^T width: for worlds whose shared memory leaves one or two CTAs
// per SM (sapb_solve_options.threads_per_cta = 256), instantiated in
// sapb_solve_nwide_f32.cu / _f64.cu.
template <bool FP32>
cudaError_t launch_solve_wide(const SolveParams& P, cudaStream_t stream, int* blocks_out) {
  using HT = typename std::conditional<FP32, float, double>::type;
  return launch_solve<256, HT, FP32 ? 2 : 1, 0, LdltBlocks<0>::kW[0]>(P, stream, blocks_out);
}
extern template cudaError_t launch_solve_wide<true>(const SolveParams&, cudaStream_t, int*);
extern template cudaError_t launch_solve_wide<false>(const SolveParams&, cudaStream_t, int*);

// The runtime-size kernels (128 and 256 threads) are the largest: each line
// search's kernel is instantiated in a translation unit of its own
// (sapb_solve_n{generic,wide}_f{32,64}_{armijo,exact,monotone}.cu).
#define SAPB_RUNTIME_SIZE_KERNELS(X, LSV)                                         \
  X(128, float, 4, 0, LSV, LdltBlocks<0>::kW[0])                                \
  X(128, double, 3, 0, LSV, LdltBlocks<0>::kW[0])                               \
  X(256, float, 2, 0, LSV, LdltBlocks<0>::kW[0])                                \
  X(256, double, 1, 0, LSV, LdltBlocks<0>::kW[0])
#define SAPB_EXTERN_LS(NT, HT, MINB, NS, LSV, LB) \
  extern template cudaError_t launch_solve_ls<NT, HT, MINB, NS, LSV, LB>(const SolveParams&, cudaStream_t, int*);
SAPB_RUNTIME_SIZE_KERNELS(SAPB_EXTERN_LS, SAPB_LS_ARMIJO_DECAY)
SAPB_RUNTIME_SIZE_KERNELS(SAPB_EXTERN_LS, SAPB_LS_EXACT_ROOT)
SAPB_RUNTIME_SIZE_KERNELS(SAPB_EXTERN_LS, SAPB_LS_MONOTONE_DECAY)
#undef SAPB_EXTERN_LS

#define SAPB_EXTERN_SOLVE(NS)                                                                  \
  extern template cudaError_t launch_solve_np<NS, true>(const SolveParams&, cudaStream_t, int*); \
  extern template cudaError_t launch_solve_np<NS, false>(const SolveParams&, cudaStream_t, int*);
SAPB_EXTERN_SOLVE(35)
SAPB_EXTERN_SOLVE(18)
SAPB_EXTERN_SOLVE(13)
SAPB_EXTERN_SOLVE(6)
SAPB_EXTERN_SOLVE(0)
#undef SAPB_EXTERN_SOLVE

}  // namespace sapb

