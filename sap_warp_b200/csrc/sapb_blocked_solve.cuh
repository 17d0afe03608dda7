// sapb_blocked_solve.cuh -- SAP stage-2 Newton solve of worlds made of many
// small trees (for example 64 free bodies: 384 DOFs), one CTA per world.
//
// Same algorithm as the dense kernel (SapContactSolve.solve,
// sim/contact_solve.py:6129-6285: prepare, the Newton loop, the line
// searches, the convergence test), on a tree-blocked layout: A is the list of
// its diagonal tree blocks, each contact row holds the columns of the (at
// most two) trees it touches, and the Newton Hessian
// H = A + sum_c J_c^T G_c J_c is block sparse -- one NB x NB block per tree
// plus one per pair of trees that share a contact.  The reference keeps A and
// J dense (sim/contact_jacobian.py:110-150, 404-562: zero blocks between trees
// materialised) and factors the dense H (sim/blocked_cholesky.py:414-604);
// the blocked LDL^T below computes the same factorization up to rounding.
//
// Per world and solve (the contact set is fixed during the Newton loop):
//  - symbolic phase (one warp): 64-bit adjacency masks of the trees, an
//    elimination order by rounds of independent low-degree trees (minimum
//    degree first, shallow elimination tree) with the fill it creates, the
//    elimination-tree levels, and the slots of the off-diagonal factor blocks;
//  - per Newton iteration: G_c per contact, diagonal and off-diagonal blocks
//    of H from per-tree contact lists (fixed summation order: deterministic),
//    left-looking block LDL^T level by level (the blocks of one level are
//    independent; each level runs as block-wide phases over flat work
//    lists), forward / backward block solves the same way.
// Precision as in the dense kernel: gradient, costs, line search, update and
// convergence test in FP64; H and its factor in HT (double or float).
//
// Trees of different sizes (an arm among free bodies) share one block size
// NB: a tree of fewer DOFs is padded with the identity in its block of A and
// zero columns in the rows, so its padded velocities stay at zero through
// the Newton loop (zero gradient, identity Hessian there); the per-DOF
// vectors in global memory are the world's own DOFs, mapped at load and
// store.
#pragma once
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <cstring>

#include "sapb_device.cuh"
#include "sapb_internal.h"
#include "sapb_linesearch.cuh"

namespace sapb {

namespace blk {

constexpr int kBMaxTrees = 64;

struct BlockedParams {
  sapb_blocked_problem p;
  sapb_dof_terms dof;  // the drive / limit terms (all zero without)
  sapb_solve_options o;
  sapb_solve_outputs out;
  int32_t use_guess_flag_ptr_valid;
  int32_t* queue;
  int32_t capacity;  // off-diagonal factor blocks one world may hold
  int32_t nd;        // DOFs of a world in the global per-DOF vectors
};

// The per-DOF vectors the blocked kernel keeps, mapped from the V_* slots the
// line searches name.  Slot kBVecs-1 holds the saved plain start while a
// candidate start is evaluated (V_SAVE) and, without drive / limit terms,
// absorbs their slots (which nothing then reads); with them, kBTermVecs
// more slots follow (bterm).
__host__ __device__ constexpr int bslot(int k) {
  return k == V_V ? 0 : k == V_VSTAR ? 1 : k == V_DV ? 2 : k == V_GRAD ? 3 : k == V_ARES ? 4 : k == V_DP ? 5
       : k == V_DSCALE ? 6 : k == V_TMP0 ? 7 : 8;
}
static_assert(bslot(V_SAVE) == 8, "the saved start has the spare slot");
constexpr int kBVecs = 9;
__host__ __device__ constexpr int bterm(int k) {
  return k == V_AINV ? 0 : k == V_PDA ? 1 : k == V_PDGAIN ? 2 : k == V_PDLIM ? 3 : k == V_LOVHAT ? 4
       : k == V_UPVHAT ? 5 : k == V_LOR ? 6 : k == V_UPR ? 7 : k == V_LORINV ? 8 : k == V_UPRINV ? 9
       : k == V_HDIAG ? 10 : -1;
}
constexpr int kBTermVecs = 11;

// Integer scratch inside off_int.
enum BInt {
  BI_ORDER = 0,                         // [64] tree eliminated at step s
  BI_LVL = BI_ORDER + kBMaxTrees,       // [64] elimination-tree level
  BI_BASE = BI_LVL + kBMaxTrees,        // [64] first off-diagonal slot of a column block
  BI_LSTART = BI_BASE + kBMaxTrees,     // [65] level -> first entry of BI_LNODES
  BI_LNODES = BI_LSTART + kBMaxTrees + 1,  // [64] column blocks by level, elimination order within
  BI_CSTART = BI_LNODES + kBMaxTrees,   // [65] tree -> first entry of its contact list
  BI_CNT = BI_CSTART + kBMaxTrees + 1,  // [64] contacts per tree / level cursor
  BI_UOFF = BI_CNT + kBMaxTrees,        // [65] by BI_LNODES position: first update item of a block
  BI_ROFF = BI_UOFF + kBMaxTrees + 1,   // [65] by BI_LNODES position: first off-diagonal row of a block
  BI_MISC = BI_ROFF + kBMaxTrees + 1,   // [4] slots used, level count, bad pivot
  BI_END = BI_MISC + 4
};

struct BLayout {
  int T, NB, n, C, cap;
  size_t off_vec, off_con, off_G, off_F, off_Y, off_dinv, off_zd, off_flags, off_mask, off_int, off_list, off_tree,
      off_slot, off_JA, total;
};

__host__ __device__ inline size_t balign(size_t x) { return (x + 15) / 16 * 16; }

// terms: the worlds carry drive / limit terms (their vector slots)
__host__ __device__ inline BLayout make_blayout(int T, int NB, int C, int hsize, int cap, bool terms = false) {
  BLayout L;
  L.T = T;
  L.NB = NB;
  L.n = T * NB;
  L.C = C > 0 ? C : 1;
  L.cap = cap;
  const size_t bb = (size_t)NB * NB * hsize;
  size_t o = 0;
  L.off_vec = o;
  o = balign(o + sizeof(double) * (size_t)(kBVecs + (terms ? kBTermVecs : 0)) * L.n);
  L.off_con = o;
  o = balign(o + sizeof(double) * (size_t)C_END * L.C);
  L.off_G = o;
  o = balign(o + (size_t)hsize * 9 * L.C);
  L.off_F = o;
  o = balign(o + bb * T);
  L.off_dinv = o;
  o = balign(o + (size_t)hsize * L.n);
  L.off_zd = o;
  o = balign(o + (size_t)hsize * L.n);
  L.off_flags = o;
  o = balign(o + sizeof(int) * (size_t)L.n);
  L.off_mask = o;  // adjacency, column and row structure of the trees
  o = balign(o + sizeof(uint64_t) * 3 * kBMaxTrees);
  L.off_int = o;
  o = balign(o + sizeof(int) * (size_t)BI_END);
  L.off_list = o;  // (contact << 1 | side) per tree, 2 C entries
  o = balign(o + sizeof(uint16_t) * 2 * (size_t)L.C);
  L.off_tree = o;  // int8 tree of each side of each contact
  o = balign(o + 2 * (size_t)L.C);
  L.off_slot = o;  // uint8 row tree / column tree of each off-diagonal slot
  o = balign(o + 2 * (size_t)(cap > 0 ? cap : 1));
  L.off_JA = o;  // FP32 copy of the J row blocks for the FP32 Hessian assembly
  o = balign(o + (hsize == 4 ? sizeof(float) * (size_t)L.C * 6 * NB : 0));
  L.off_Y = o;
  o = balign(o + bb * (size_t)(cap > 0 ? cap : 1));
  L.total = o;
  return L;
}

}  // namespace blk

using namespace blk;

template <int NT, typename HT, int NB>
struct BWorld {
  // -- the world interface of the line searches --
  int count, n, C;
  double* vec;
  double* con;
  int* flags;
  double* red;
  __device__ __forceinline__ int dofs() const { return n; }
  bool terms;  // drive / limit terms: their slots after the kBVecs
  int has_pd, has_limits;
  double dt;
  __device__ __forceinline__ double* V(int k) const {
    const int t = terms ? bterm(k) : -1;
    return vec + (size_t)(t >= 0 ? kBVecs + t : bslot(k)) * n;
  }
  __device__ __forceinline__ double* Cn(int k) const { return con + (size_t)k * C; }
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
  // -- blocked data --
  int T;
  const double* A;  // global [T][NB][NB] of this world
  const double* J;  // global [C][3][2 NB] of this world
  const int8_t* tree;  // [C][2]
  HT* G;               // [C][9]
  HT* F;               // [T][NB][NB] diagonal blocks: H, then unit L below the diagonal and D on it
  HT* Y;               // [cap][NB][NB] off-diagonal blocks: H, then L_ij D_j
  HT* dinv;            // [n] 1 / D
  HT* zd;              // [n] forward-solve scratch D^-1 z
  uint64_t* adj;       // [64] tree adjacency (then with fill)
  uint64_t* colm;      // [64] trees below column block p in the factor (later in the order)
  uint64_t* rowm;      // [64] column blocks k with a block in row j
  int* iw;             // BInt scratch
  const uint16_t* list;  // per-tree (contact << 1 | side)
  uint8_t* slot_row;
  uint8_t* slot_col;
  float* JA;  // [C][3][2 NB] FP32 copy of J (FP32 Hessian only)
  __device__ __forceinline__ const double* jrow(int c, int k) const { return J + ((size_t)c * 3 + k) * (2 * NB); }
  // slot of the off-diagonal block (row tree i, column block k); i must lie in colm[k]
  __device__ __forceinline__ int slot(int i, int k) const {
    return iw[BI_BASE + k] + __popcll(colm[k] & ((1ull << i) - 1ull));
  }
};

// rows of J times x (per DOF vector, FP64) into the contact slots slot..slot+2
template <int NT, typename HT, int NB>
__device__ void brows_times(const BWorld<NT, HT, NB>& w, const double* x, int slot) {
  for (int r = threadIdx.x; r < 3 * w.count; r += NT) {
    const int c = r / 3, k = r - 3 * c;
    const double* jr = w.jrow(c, k);
    double s = 0.0;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
      const int t = w.tree[2 * c + side];
      if (t < 0) continue;
      const double* xt = x + t * NB;
#pragma unroll
      for (int b = 0; b < NB; ++b) s += __ldg(jr + side * NB + b) * xt[b];
    }
    w.Cn(slot + k)[c] = s;
  }
}

// Objective at V_V: contact impulses and costs, A(v - v*), J^T gamma, the
// gradient and the scaled norms of the convergence test (the dense kernel's
// evaluate, sim/contact_solve.py:4080-4136, without PD / limit terms).
template <int NT, typename HT, int NB>
__device__ void bevaluate(const BWorld<NT, HT, NB>& w, double out4[4]) {
  const int tid = threadIdx.x;
  brows_times<NT, HT, NB>(w, w.V(V_V), C_VC);
  for (int i = tid; i < w.n; i += NT) w.V(V_TMP0)[i] = w.V(V_V)[i] - w.V(V_VSTAR)[i];
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
  double model_cost = 0.0, g2 = 0.0, p2 = 0.0, j2 = 0.0;
  for (int i = tid; i < w.n; i += NT) {
    const int t = i / NB, a = i - t * NB;
    const double* Ar = w.A + ((size_t)t * NB + a) * NB;
    const double* res = w.V(V_TMP0) + t * NB;
    const double* vt = w.V(V_V) + t * NB;
    double a_res = 0.0, a_v = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const double aij = __ldg(Ar + b);
      a_res += aij * res[b];
      a_v += aij * vt[b];
    }
    double imp = 0.0;
    {
      const int q0 = w.iw[BI_CSTART + t], q1 = w.iw[BI_CSTART + t + 1];
      int q = q0;
      for (; q + 4 <= q1; q += 4) {  // four contacts' loads in flight, sum in list order
        double jv[4][3];
        int cc[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int ent = w.list[q + u];
          cc[u] = ent >> 1;
          const double* j0 = w.jrow(ent >> 1, 0) + (ent & 1) * NB + a;
#pragma unroll
          for (int k = 0; k < 3; ++k) jv[u][k] = __ldg(j0 + k * 2 * NB);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
          imp += jv[u][0] * w.Cn(C_GAMMA + 0)[cc[u]] + jv[u][1] * w.Cn(C_GAMMA + 1)[cc[u]] +
                 jv[u][2] * w.Cn(C_GAMMA + 2)[cc[u]];
      }
      for (; q < q1; ++q) {
        const int c = w.list[q] >> 1, side = w.list[q] & 1;
        const double* j0 = w.jrow(c, 0) + side * NB + a;
        imp += __ldg(j0) * w.Cn(C_GAMMA + 0)[c] + __ldg(j0 + 2 * NB) * w.Cn(C_GAMMA + 1)[c] +
               __ldg(j0 + 4 * NB) * w.Cn(C_GAMMA + 2)[c];
      }
    }
    double mc = 0.5 * w.V(V_TMP0)[i] * a_res;
    if (w.terms) {  // drive and limit terms (as the dense solve's evaluate)
      const double vi = vt[a], dt = w.dt;
      const int fl = w.flags[i];
      double pdg = 0.0, lg = 0.0, hd = 0.0;
      if (w.has_pd && (fl & kFlagPd)) {
        const double gain = w.V(V_PDGAIN)[i], lim = w.V(V_PDLIM)[i];
        const double y = w.V(V_PDA)[i] - gain * vi;
        pdg = dt * clamp_limit(y, lim);
        hd += dt * gain * clamp_limit_derivative(y, lim);
        if (gain > 0.0) mc += (dt / gain) * clamp_limit_antiderivative(y, lim);
      }
      if (w.has_limits) {
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
      w.V(V_HDIAG)[i] = hd;
    }
    const double grad = a_res - imp;
    w.V(V_ARES)[i] = a_res;
    w.V(V_GRAD)[i] = grad;
    model_cost += mc;
    if (w.flags[i] & kFlagPart) {
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

// Line coefficients (sim/contact_solve.py:2234-2263, 1657-1692): dvc = J dv,
// dp = A dv and {dell0, dell_a0, d2ell_a, mom0}.
template <int NT, typename HT, int NB>
__device__ void line_coefficients(const BWorld<NT, HT, NB>& w, double c4[4]) {
  const int tid = threadIdx.x;
  brows_times<NT, HT, NB>(w, w.V(V_DV), C_DVC);
  double d0 = 0.0, da0 = 0.0, d2 = 0.0, m0 = 0.0;
  const double* v = w.V(V_V);
  const double* vs = w.V(V_VSTAR);
  const double* dv = w.V(V_DV);
  for (int i = tid; i < w.n; i += NT) {
    const int t = i / NB, a = i - t * NB;
    const double* Ar = w.A + ((size_t)t * NB + a) * NB;
    double acc = 0.0;
#pragma unroll
    for (int b = 0; b < NB; ++b) acc += __ldg(Ar + b) * dv[t * NB + b];
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

// Element idx (row k: k * 2 NB + side * NB + column) of contact c's J row
// block as HT: from the FP32 copy in shared memory when H is FP32, else the
// FP64 rows in global memory.
template <int NT, typename HT, int NB>
__device__ __forceinline__ HT jval(const BWorld<NT, HT, NB>& w, int c, int idx) {
  if constexpr (sizeof(HT) == 4)
    return w.JA[c * 6 * NB + idx];
  else
    return HT(__ldg(w.J + (size_t)c * 6 * NB + idx));
}

// Row a of one H block: acc[b] += sum over the list entries e0..e1
// (contact << 1 | side sb) of (J_{c,sa}[:, a])^T G_c J_{c,sb}[:, b], with
// sa = sb (a tree's diagonal block) or sa = 1 - sb restricted to contacts
// whose side sa lies on tree `other` (an off-diagonal block).  y = ja^T G is
// formed once per contact and shared by the NB entries of the row; the sum
// runs in list order.
template <int NT, typename HT, int NB, bool kDiag>
__device__ __forceinline__ void sum_block_row(const BWorld<NT, HT, NB>& w, int e0, int e1, int a, int other,
                                              HT (&acc)[NB]) {
  for (int e = e0; e < e1; ++e) {
    const int ent = w.list[e];
    const int c = ent >> 1, sb = ent & 1, sa = kDiag ? sb : 1 - sb;
    if (!kDiag && w.tree[2 * c + sa] != other) continue;
    const HT* G = w.G + 9 * c;
    HT ja[3], jb[3][NB];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      ja[k] = jval<NT, HT, NB>(w, c, k * 2 * NB + sa * NB + a);
#pragma unroll
      for (int b = 0; b < NB; ++b) jb[k][b] = jval<NT, HT, NB>(w, c, k * 2 * NB + sb * NB + b);
    }
    HT y[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) y[k] = ja[0] * G[k] + ja[1] * G[3 + k] + ja[2] * G[6 + k];
#pragma unroll
    for (int b = 0; b < NB; ++b) acc[b] += y[0] * jb[0][b] + y[1] * jb[1][b] + y[2] * jb[2][b];
  }
}

// H = A + J^T G J + shift I in the block layout: F (tree blocks, lower
// triangle) and Y (off-diagonal blocks of the factor's structure; blocks
// that only fill-in creates start at zero).
template <int NT, typename HT, int NB>
__device__ void bassemble(const BWorld<NT, HT, NB>& w, double diag_shift) {
  const int tid = threadIdx.x;
  if (tid == 0) w.iw[BI_MISC + 2] = 0;  // bad-pivot flag of the factorization that follows
  for (int c = tid; c < w.count; c += NT) {
    double g[3], cost, G[9];
    project_contact(w.cc(c), w.Cn(C_VC + 0)[c], w.Cn(C_VC + 1)[c], w.Cn(C_VC + 2)[c], g, &cost, G);
#pragma unroll
    for (int k = 0; k < 9; ++k) w.G[9 * c + k] = HT(G[k]);
  }
  __syncthreads();
  // one item per block row: the NB rows of each tree's diagonal block, then
  // the NB rows of each off-diagonal slot
  const int ndiag = w.T * NB;
  const int nslots = w.iw[BI_MISC + 0];
  const int total = ndiag + nslots * NB;
  for (int item = tid; item < total; item += NT) {
    HT acc[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) acc[b] = HT(0);
    if (item < ndiag) {
      const int t = item / NB, a = item - t * NB;
      sum_block_row<NT, HT, NB, true>(w, w.iw[BI_CSTART + t], w.iw[BI_CSTART + t + 1], a, -1, acc);
      const double* Ar = w.A + ((size_t)t * NB + a) * NB;
      HT* Fr = w.F + (t * NB + a) * NB;
#pragma unroll
      for (int b = 0; b < NB; ++b)
        if (b <= a)
          Fr[b] = HT(__ldg(Ar + b) + (a == b ? diag_shift + (w.terms ? w.V(V_HDIAG)[t * NB + a] : 0.0) : 0.0)) +
                  acc[b];
    } else {
      const int q = item - ndiag;
      const int sl = q / NB, a = q - sl * NB;
      const int i = w.slot_row[sl], p = w.slot_col[sl];
      sum_block_row<NT, HT, NB, false>(w, w.iw[BI_CSTART + p], w.iw[BI_CSTART + p + 1], a, i, acc);
      HT* Yr = w.Y + ((size_t)sl * NB + a) * NB;
#pragma unroll
      for (int b = 0; b < NB; ++b) Yr[b] = acc[b];
    }
  }
  __syncthreads();
}

// Position idx in [b0, b1) of BI_LNODES whose work range [off[idx],
// off[idx + 1]) holds flat item u (off = BI_UOFF or BI_ROFF; blocks with no
// work have empty ranges and are never returned).
__device__ __forceinline__ int find_block(const int* off, int b0, int b1, int u) {
  int lo = b0, hi = b1 - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= u) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The m-th tree (in increasing index) of the mask cj.
__device__ __forceinline__ int nth_tree(uint64_t cj, int m) {
  for (int z = 0; z < m; ++z) cj &= cj - 1;
  return __ffsll((long long)cj) - 1;
}

// Left-looking block LDL^T, one elimination-tree level at a time.  Each level
// is three block-wide phases over flat work lists (no per-block loops that
// diverge within a warp): (A) every entry of the level's column blocks j
// minus the contributions of the finished blocks k below them (rowm[j]);
// (B) a thread per block factors its NB x NB diagonal block in registers;
// (C) every row of the off-diagonal blocks, Y_ij <- M_ij L_jj^-T.
template <int NT, typename HT, int NB>
__device__ void bfactor(const BWorld<NT, HT, NB>& w) {
  constexpr int tri = NB * (NB + 1) / 2;
  const int tid = threadIdx.x;
  const int nlev = w.iw[BI_MISC + 1];
  const int* uoff = w.iw + BI_UOFF;
  const int* roff = w.iw + BI_ROFF;
  for (int l = 0; l < nlev; ++l) {
    const int b0 = w.iw[BI_LSTART + l], b1 = w.iw[BI_LSTART + l + 1];
    // (A) updates
    const int u0 = uoff[b0], u1 = uoff[b1];
    for (int u = u0 + tid; u < u1; u += NT) {
      const int idx = find_block(uoff, b0, b1, u);
      const int j = w.iw[BI_LNODES + idx];
      const uint64_t rj = w.rowm[j];
      const int item = u - uoff[idx];
      if (item < tri) {
        int a = 0;
        while ((a + 1) * (a + 2) / 2 <= item) ++a;
        const int b = item - a * (a + 1) / 2;
        HT sum = HT(0);
        uint64_t r = rj;
        while (r) {
          const int k = __ffsll((long long)r) - 1;
          r &= r - 1;
          const HT* Yjk = w.Y + (size_t)w.slot(j, k) * NB * NB;
          const HT* dk = w.dinv + k * NB;
#pragma unroll
          for (int e = 0; e < NB; ++e) sum += Yjk[a * NB + e] * dk[e] * Yjk[b * NB + e];
        }
        w.F[(j * NB + a) * NB + b] -= sum;
      } else {
        const int q = item - tri;
        const int m = q / (NB * NB), ab = q - m * NB * NB;
        const int a = ab / NB, b = ab - a * NB;
        const int i = nth_tree(w.colm[j], m);
        HT sum = HT(0);
        uint64_t r = rj;
        while (r) {
          const int k = __ffsll((long long)r) - 1;
          r &= r - 1;
          if (!((w.colm[k] >> i) & 1ull)) continue;
          const HT* Yik = w.Y + (size_t)w.slot(i, k) * NB * NB;
          const HT* Yjk = w.Y + (size_t)w.slot(j, k) * NB * NB;
          const HT* dk = w.dinv + k * NB;
#pragma unroll
          for (int e = 0; e < NB; ++e) sum += Yik[a * NB + e] * dk[e] * Yjk[b * NB + e];
        }
        w.Y[(size_t)w.slot(i, j) * NB * NB + ab] -= sum;
      }
    }
    if (u1 > u0) __syncthreads();
    // (B) diagonal blocks, a thread per block, in registers
    for (int idx = b0 + tid; idx < b1; idx += NT) {
      const int j = w.iw[BI_LNODES + idx];
      HT* Fj = w.F + j * NB * NB;
      HT Lr[NB][NB], Dr[NB], Rr[NB];
#pragma unroll
      for (int a = 0; a < NB; ++a)
#pragma unroll
        for (int b = 0; b <= a; ++b) Lr[a][b] = Fj[a * NB + b];
      bool ok = true;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        HT d = Lr[b][b];
#pragma unroll
        for (int e = 0; e < b; ++e) d -= Lr[b][e] * Lr[b][e] * Dr[e];
        Dr[b] = d;
        Rr[b] = fast_recip(d);
        ok = ok && d > HT(0) && isfinite(double(d));
#pragma unroll
        for (int a = b + 1; a < NB; ++a) {
          HT v = Lr[a][b];
#pragma unroll
          for (int e = 0; e < b; ++e) v -= Lr[a][e] * Lr[b][e] * Dr[e];
          Lr[a][b] = v * Rr[b];
        }
      }
#pragma unroll
      for (int a = 0; a < NB; ++a) {
#pragma unroll
        for (int b = 0; b < a; ++b) Fj[a * NB + b] = Lr[a][b];
        Fj[a * NB + a] = Dr[a];
        w.dinv[j * NB + a] = Rr[a];
      }
      if (!ok) w.iw[BI_MISC + 2] = 1;
    }
    __syncthreads();
    // (C) off-diagonal rows
    const int r0 = roff[b0], r1 = roff[b1];
    for (int u = r0 + tid; u < r1; u += NT) {
      const int idx = find_block(roff, b0, b1, u);
      const int j = w.iw[BI_LNODES + idx];
      const int row = u - roff[idx];
      const int m = row / NB, a = row - m * NB;
      const int i = nth_tree(w.colm[j], m);
      const HT* Fj = w.F + j * NB * NB;
      HT* y = w.Y + (size_t)w.slot(i, j) * NB * NB + a * NB;
      HT yv[NB];
#pragma unroll
      for (int b = 0; b < NB; ++b) {
        HT sum = y[b];
#pragma unroll
        for (int e = 0; e < b; ++e) sum -= yv[e] * Fj[b * NB + e];
        yv[b] = sum;
      }
#pragma unroll
      for (int b = 0; b < NB; ++b) y[b] = yv[b];
    }
    if (r1 > r0) __syncthreads();
  }
}

// dv = -H^-1 grad with the block factor: forward L z = b (levels up), then
// L^T x = D^-1 z (levels down).  Per level: a thread per block row gathers
// the off-diagonal products, then a thread per block solves with its
// diagonal block.  A bad pivot makes dv NaN (as in the dense kernel).
template <int NT, typename HT, int NB>
__device__ void bsolve(const BWorld<NT, HT, NB>& w) {
  const int tid = threadIdx.x;
  const int nlev = w.iw[BI_MISC + 1];
  double* dv = w.V(V_DV);
  const double* grad = w.V(V_GRAD);
  for (int l = 0; l < nlev; ++l) {
    const int b0 = w.iw[BI_LSTART + l], b1 = w.iw[BI_LSTART + l + 1];
    for (int u = tid; u < (b1 - b0) * NB; u += NT) {
      const int j = w.iw[BI_LNODES + b0 + u / NB], a = u % NB;
      HT z = HT(-grad[j * NB + a]);
      uint64_t r = w.rowm[j];
      while (r) {
        const int k = __ffsll((long long)r) - 1;
        r &= r - 1;
        const HT* Yjk = w.Y + (size_t)w.slot(j, k) * NB * NB + a * NB;
        const HT* zk = w.zd + k * NB;
#pragma unroll
        for (int e = 0; e < NB; ++e) z -= Yjk[e] * zk[e];
      }
      w.zd[j * NB + a] = z;  // the block's own zd is not read in this level
    }
    __syncthreads();
    for (int idx = b0 + tid; idx < b1; idx += NT) {
      const int j = w.iw[BI_LNODES + idx];
      const HT* Fj = w.F + j * NB * NB;
      HT z[NB];
#pragma unroll
      for (int a = 0; a < NB; ++a) {
        HT v = w.zd[j * NB + a];
#pragma unroll
        for (int e = 0; e < a; ++e) v -= Fj[a * NB + e] * z[e];
        z[a] = v;
      }
#pragma unroll
      for (int a = 0; a < NB; ++a) w.zd[j * NB + a] = z[a] * w.dinv[j * NB + a];
    }
    __syncthreads();
  }
  for (int l = nlev - 1; l >= 0; --l) {
    const int b0 = w.iw[BI_LSTART + l], b1 = w.iw[BI_LSTART + l + 1];
    for (int u = tid; u < (b1 - b0) * NB; u += NT) {
      const int j = w.iw[BI_LNODES + b0 + u / NB], b = u % NB;
      HT sum = HT(0);
      uint64_t cc = w.colm[j];
      while (cc) {
        const int i = __ffsll((long long)cc) - 1;
        cc &= cc - 1;
        const HT* Yij = w.Y + (size_t)w.slot(i, j) * NB * NB + b;
#pragma unroll
        for (int a = 0; a < NB; ++a) sum += Yij[a * NB] * HT(dv[i * NB + a]);
      }
      dv[j * NB + b] = double(w.zd[j * NB + b] - w.dinv[j * NB + b] * sum);
    }
    __syncthreads();
    for (int idx = b0 + tid; idx < b1; idx += NT) {
      const int j = w.iw[BI_LNODES + idx];
      const HT* Fj = w.F + j * NB * NB;
      HT x[NB];
#pragma unroll
      for (int a = NB - 1; a >= 0; --a) {
        HT v = HT(dv[j * NB + a]);
#pragma unroll
        for (int c = a + 1; c < NB; ++c) v -= Fj[c * NB + a] * x[c];
        x[a] = v;
      }
#pragma unroll
      for (int a = 0; a < NB; ++a) dv[j * NB + a] = double(x[a]);
    }
    __syncthreads();
  }
  if (w.iw[BI_MISC + 2]) {
    const double nanv = __longlong_as_double(0x7ff8000000000000ULL);
    for (int i = tid; i < w.n; i += NT) dv[i] = nanv;
    __syncthreads();
  }
}

// Symbolic phase (warp 0): elimination order on the tree adjacency in rounds
// -- each round eliminates a greedy independent set (tree order) of the
// remaining trees whose degree is at most max(minimum degree, 2), so a chain
// of trees (a stack of boxes) is halved per round instead of peeled from one
// end, which keeps the elimination tree shallow -- with the fill, the row
// structure, elimination-tree levels, slot bases and level lists.  Returns
// false (to every thread) when the factor needs more off-diagonal blocks than
// the world's capacity.
template <int NT, typename HT, int NB>
__device__ bool bsymbolic(const BWorld<NT, HT, NB>& w, int cap) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int T = w.T;
  if (warp == 0) {
    uint64_t rem = T == 64 ? ~0ull : ((1ull << T) - 1ull);
    uint64_t a0 = lane < T ? w.adj[lane] : 0ull, a1 = lane + 32 < T ? w.adj[lane + 32] : 0ull;
    const bool own0 = lane < T, own1 = lane + 32 < T;
    int s = 0;
    while (rem) {
      // degrees of the remaining trees and the round's candidates: degree
      // <= max(minimum degree, 2)
      const int d0 = own0 && ((rem >> lane) & 1ull) ? __popcll(a0 & rem) : INT_MAX;
      const int d1 = own1 && ((rem >> (lane + 32)) & 1ull) ? __popcll(a1 & rem) : INT_MAX;
      const int dmin = __reduce_min_sync(0xffffffffu, min(d0, d1));
      const int thr = max(dmin, 2);
      const uint64_t cand = (uint64_t)__ballot_sync(0xffffffffu, d0 <= thr) |
                            ((uint64_t)__ballot_sync(0xffffffffu, d1 <= thr) << 32);
      // greedy independent set of candidates in tree order, eliminated together
      uint64_t sel = 0ull, m = cand;
      while (m) {
        const int p = __ffsll((long long)m) - 1;
        m &= m - 1;
        const uint64_t ap = __shfl_sync(0xffffffffu, p < 32 ? a0 : a1, p & 31);
        if (!(ap & sel)) sel |= 1ull << p;
      }
      // their column structures (the selected trees are pairwise non-adjacent,
      // so one's fill leaves another's adjacency unchanged), then the fill
      m = sel;
      while (m) {
        const int p = __ffsll((long long)m) - 1;
        m &= m - 1;
        const uint64_t ap = __shfl_sync(0xffffffffu, p < 32 ? a0 : a1, p & 31);
        const uint64_t col = ap & rem & ~(1ull << p);
        if (lane == 0) {
          w.colm[p] = col;
          w.iw[BI_ORDER + s] = p;
        }
        ++s;
        if (own0 && ((col >> lane) & 1ull)) a0 |= col & ~(1ull << lane);
        if (own1 && ((col >> (lane + 32)) & 1ull)) a1 |= col & ~(1ull << (lane + 32));
      }
      rem &= ~sel;
    }
    __syncwarp();
    for (int j = lane; j < T; j += 32) {
      uint64_t r = 0ull;
      for (int k = 0; k < T; ++k)
        if ((w.colm[k] >> j) & 1ull) r |= 1ull << k;
      w.rowm[j] = r;
    }
    __syncwarp();
    if (lane == 0) {
      int nslots = 0, maxl = 0;
      for (int s = 0; s < T; ++s) {
        const int p = w.iw[BI_ORDER + s];
        int l = 0;
        uint64_t r = w.rowm[p];
        while (r) {
          const int k = __ffsll((long long)r) - 1;
          r &= r - 1;
          l = max(l, w.iw[BI_LVL + k] + 1);
        }
        w.iw[BI_LVL + p] = l;
        maxl = max(maxl, l);
        w.iw[BI_BASE + p] = nslots;
        nslots += __popcll(w.colm[p]);
      }
      const int nlev = maxl + 1;
      w.iw[BI_MISC + 0] = nslots;
      w.iw[BI_MISC + 1] = nlev;
      w.iw[BI_MISC + 2] = 0;
      for (int l = 0; l <= nlev; ++l) w.iw[BI_LSTART + l] = 0;
      for (int s = 0; s < T; ++s) w.iw[BI_LSTART + w.iw[BI_LVL + w.iw[BI_ORDER + s]] + 1] += 1;
      for (int l = 0; l < nlev; ++l) w.iw[BI_LSTART + l + 1] += w.iw[BI_LSTART + l];
      for (int l = 0; l < nlev; ++l) w.iw[BI_CNT + l] = w.iw[BI_LSTART + l];
      for (int s = 0; s < T; ++s) {
        const int p = w.iw[BI_ORDER + s];
        w.iw[BI_LNODES + w.iw[BI_CNT + w.iw[BI_LVL + p]]++] = p;
      }
      // flat work offsets of the factorization's update and row phases
      constexpr int tri = NB * (NB + 1) / 2;
      int u = 0, r = 0;
      for (int idx = 0; idx < T; ++idx) {
        const int p = w.iw[BI_LNODES + idx];
        const int nc = __popcll(w.colm[p]);
        w.iw[BI_UOFF + idx] = u;
        w.iw[BI_ROFF + idx] = r;
        if (w.rowm[p]) u += tri + nc * NB * NB;
        r += nc * NB;
      }
      w.iw[BI_UOFF + T] = u;
      w.iw[BI_ROFF + T] = r;
    }
  }
  __syncthreads();
  const int nslots = w.iw[BI_MISC + 0];
  if (nslots > cap) return false;
  // slot owners (row tree i, column block p), rows in increasing tree index
  for (int p = threadIdx.x; p < T; p += NT) {
    uint64_t cc = w.colm[p];
    int sl = w.iw[BI_BASE + p];
    while (cc) {
      const int i = __ffsll((long long)cc) - 1;
      cc &= cc - 1;
      w.slot_row[sl] = (uint8_t)i;
      w.slot_col[sl] = (uint8_t)p;
      ++sl;
    }
  }
  __syncthreads();
  return true;
}

template <int NT, typename HT, int NB, int LSV>
__global__ void __launch_bounds__(NT, 1) blocked_solve_kernel(const BlockedParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[8 * (NT / 32)];
  __shared__ int s_next;
  __shared__ int s_tstart[kBMaxTrees], s_tcount[kBMaxTrees];
  __shared__ int s_bad_layout;
  const int tid = threadIdx.x;
  const int T = P.p.trees_per_env, C = P.p.max_contacts;
  const int n = T * NB;
  const bool terms = P.dof.has_pd || P.dof.has_limits;
  const BLayout L = make_blayout(T, NB, C, (int)sizeof(HT), P.capacity, terms);
  const bool use_guess = P.use_guess_flag_ptr_valid && P.p.v_guess_active[0] != 0;

  // tree t's DOFs in the global vectors: s_tstart[t] .. + s_tcount[t]; an
  // invalid map (decreasing, a tree above NB, beyond the world) leaves its
  // trees empty and every world NOT_FINITE
  if (tid == 0) s_bad_layout = 0;
  __syncthreads();
  for (int t = tid; t < T; t += NT) {
    int st = t * NB, cnt = NB;
    if (P.p.tree_dof_start) {
      st = P.p.tree_dof_start[t];
      cnt = P.p.tree_dof_start[t + 1] - st;
    }
    if (st < 0 || cnt < 0 || cnt > NB || st + cnt > P.nd) {
      s_bad_layout = 1;
      st = 0;
      cnt = 0;
    }
    s_tstart[t] = st;
    s_tcount[t] = cnt;
  }
  __syncthreads();
  auto gidx = [&](int i) {
    const int t = i / NB, a = i - t * NB;
    return a < s_tcount[t] ? s_tstart[t] + a : -1;
  };

  if (tid == 0) s_next = atomicAdd(P.queue, 1);
  for (;;) {
    __syncthreads();
    const int ticket = s_next;
    if (ticket >= P.p.num_envs) break;
    const int e = P.p.world_order ? P.p.world_order[ticket] : ticket;
    __syncthreads();
    if (tid == 0) s_next = atomicAdd(P.queue, 1);
    __syncthreads();
    if (e < 0 || e >= P.p.num_envs) continue;

    BWorld<NT, HT, NB> w;
    w.terms = terms;
    w.has_pd = P.dof.has_pd;
    w.has_limits = P.dof.has_limits;
    w.n = n;
    w.C = L.C;
    w.T = T;
    w.vec = reinterpret_cast<double*>(smem + L.off_vec);
    w.con = reinterpret_cast<double*>(smem + L.off_con);
    w.flags = reinterpret_cast<int*>(smem + L.off_flags);
    w.red = red;
    w.A = P.p.tree_mass + (size_t)e * T * NB * NB;
    w.J = P.p.jacobian + (size_t)e * C * 3 * 2 * NB;
    w.tree = reinterpret_cast<const int8_t*>(smem + L.off_tree);
    w.G = reinterpret_cast<HT*>(smem + L.off_G);
    w.F = reinterpret_cast<HT*>(smem + L.off_F);
    w.Y = reinterpret_cast<HT*>(smem + L.off_Y);
    w.dinv = reinterpret_cast<HT*>(smem + L.off_dinv);
    w.zd = reinterpret_cast<HT*>(smem + L.off_zd);
    w.adj = reinterpret_cast<uint64_t*>(smem + L.off_mask);
    w.colm = w.adj + kBMaxTrees;
    w.rowm = w.colm + kBMaxTrees;
    w.iw = reinterpret_cast<int*>(smem + L.off_int);
    w.list = reinterpret_cast<const uint16_t*>(smem + L.off_list);
    w.slot_row = reinterpret_cast<uint8_t*>(smem + L.off_slot);
    w.slot_col = w.slot_row + (L.cap > 0 ? L.cap : 1);
    w.JA = reinterpret_cast<float*>(smem + L.off_JA);
    int count = P.p.contact_count[e];
    if (count > C) count = C;
    if (count < 0) count = 0;
    w.count = count;
    const double dt = P.p.dt[e];
    const size_t base = (size_t)e * P.nd;
    int8_t* tree_w = reinterpret_cast<int8_t*>(smem + L.off_tree);
    uint16_t* list_w = reinterpret_cast<uint16_t*>(smem + L.off_list);

    // ---- contacts, vectors, adjacency -------------------------------------
    for (int t = tid; t < kBMaxTrees; t += NT) w.adj[t] = 0ull;
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
      int t0 = P.p.contact_tree[2 * ci], t1 = P.p.contact_tree[2 * ci + 1];
      if (t0 < 0 || t0 >= T) t0 = -1;
      if (t1 < 0 || t1 >= T || t1 == t0) t1 = -1;
      tree_w[2 * c] = (int8_t)t0;
      tree_w[2 * c + 1] = (int8_t)t1;
    }
    if constexpr (sizeof(HT) == 4) {
      for (int k = tid; k < count * 6 * NB; k += NT) w.JA[k] = (float)__ldg(w.J + k);
    }
    bool bad = s_bad_layout != 0;  // NaN / Inf in the world's inputs
    for (int i = tid; i < n; i += NT) {
      const int gi = gidx(i);
      double vs = 0.0, v = 0.0;  // padded DOFs: zero
      if (gi >= 0) {
        vs = P.p.v_star[base + gi];
        v = P.p.v0[base + gi];
        if (P.p.v_guess) {
          if (use_guess) v = P.p.v_guess[base + gi];
          P.p.v_guess[base + gi] = v;
        }
      }
      w.V(V_VSTAR)[i] = vs;
      w.V(V_V)[i] = v;
      bad = bad || !isfinite(vs) || !isfinite(v);
      const int t = i / NB, a = i - t * NB;
      const double* Ar = w.A + ((size_t)t * NB + a) * NB;
      for (int b = 0; b < NB; ++b) bad = bad || !isfinite(__ldg(Ar + b));
      double d = __ldg(Ar + a);
      if (d < 1.0e-12 || !isfinite(d)) d = 1.0e-12;
      w.V(V_DSCALE)[i] = 1.0 / sqrt(d);
      w.flags[i] = 0;
    }
    for (int k = tid; k < count * 6 * NB; k += NT) bad = bad || !isfinite(__ldg(w.J + k));
    for (int c = tid; c < count; c += NT)  // the contact constants formed above
      for (int q = C_RT; q < C_VC; ++q) bad = bad || !isfinite(w.Cn(q)[c]);
    bad = __syncthreads_or(bad) != 0;
    w.dt = dt;
    // drive and limit terms of the world's own DOFs (sim/contact_solve.py:
    // 490-683, as in the dense solve); a DOF they act on takes part
    bool wterms = false;
    if (terms) {
      const sapb_dof_terms& D = P.dof;
      const int ndof = P.p.num_envs * P.nd;
      for (int i = tid; i < n; i += NT) {
        const int gi = gidx(i);
        const int t = i / NB, a = i - t * NB;
        double d = __ldg(w.A + ((size_t)t * NB + a) * NB + a);
        if (d < 1.0e-12 || !isfinite(d)) d = 1.0e-12;
        w.V(V_AINV)[i] = 1.0 / d;
        w.V(V_LOR)[i] = 1.0;
        w.V(V_UPR)[i] = 1.0;
        w.V(V_HDIAG)[i] = 0.0;
        int fl = 0;
        if (gi >= 0) {
          const size_t dof = base + gi;
          if (D.has_pd) {
            int coord = D.dof_coord_index[dof];
            if (coord >= D.joint_coord_count) coord = -1;
            int target = D.dof_target_index[dof];
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
          if (D.has_limits) {
            int coord = D.dof_coord_index[dof];
            if (coord >= D.joint_coord_count) coord = -1;
            const double ke = coord >= 0 ? D.joint_limit_ke[dof] : 0.0;
            if (coord >= 0 && D.limit_supported[dof] != 0 && ke > 0.0) {
              const double q0 = D.joint_q[coord];
              const double lower = D.joint_limit_lower[dof], upper = D.joint_limit_upper[dof];
              const double speed = fmax(fabs(P.p.v0[base + gi]), fabs(w.V(V_VSTAR)[i]));
              const double window = kLimitWindow * dt * speed;
              const double kdl = D.joint_limit_kd[dof];
              const double tau_d = kdl > 0.0 ? kdl / ke : 0.0;
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
        }
        if (fl) fl |= kFlagPart;
        w.flags[i] = fl;
        wterms = wterms || fl != 0;
      }
    }
    wterms = __syncthreads_or(wterms) != 0;
    for (int c = tid; c < count; c += NT) {
      const int t0 = tree_w[2 * c], t1 = tree_w[2 * c + 1];
      if (t0 >= 0 && t1 >= 0) {
        atomicOr(reinterpret_cast<unsigned long long*>(&w.adj[t0]), 1ull << t1);
        atomicOr(reinterpret_cast<unsigned long long*>(&w.adj[t1]), 1ull << t0);
      }
    }
    // per-tree contact lists in contact order (count, scan, fill)
    for (int t = tid; t < T; t += NT) {
      int k = 0;
      for (int c = 0; c < count; ++c) k += (tree_w[2 * c] == t) + (tree_w[2 * c + 1] == t);
      w.iw[BI_CNT + t] = k;
    }
    __syncthreads();
    if (tid == 0) {
      int s = 0;
      for (int t = 0; t < T; ++t) {
        w.iw[BI_CSTART + t] = s;
        s += w.iw[BI_CNT + t];
      }
      w.iw[BI_CSTART + T] = s;
    }
    __syncthreads();
    for (int t = tid; t < T; t += NT) {
      int q = w.iw[BI_CSTART + t];
      for (int c = 0; c < count; ++c) {
        if (tree_w[2 * c] == t) list_w[q++] = (uint16_t)(c << 1);
        if (tree_w[2 * c + 1] == t) list_w[q++] = (uint16_t)((c << 1) | 1);
      }
      if (w.iw[BI_CNT + t] > 0)
        for (int a = 0; a < NB; ++a) w.flags[t * NB + a] |= kFlagPart;
    }
    __syncthreads();
    const bool fits = bsymbolic<NT, HT, NB>(w, L.cap);

    int newton_iterations = 0, ls_total = 0, converged = 0, status = 0, accepted = 0;
    double cost = 0.0, previous_cost = 0.0, alpha = 1.0, grad_norm = 0.0;
    bool evaluated = false;
    if (bad) {
      status = SAPB_WORLD_NOT_FINITE;  // not solved: v = the start velocity
    } else if (!fits) {
      status = SAPB_WORLD_FACTOR_CAPACITY;
      for (int i = tid; i < n; i += NT) w.V(V_V)[i] = w.V(V_VSTAR)[i];
      __syncthreads();
    } else if (count == 0 && !wterms) {
      converged = 1;
      for (int i = tid; i < n; i += NT) w.V(V_V)[i] = w.V(V_VSTAR)[i];
      __syncthreads();
    } else {
      for (int i = tid; i < n; i += NT)
        if (!(w.flags[i] & kFlagPart)) w.V(V_V)[i] = w.V(V_VSTAR)[i];
      __syncthreads();
      // Candidate start (no counterpart in the reference): v_c = v* +
      // A^-1 J^T gamma0, tree by tree since A is block diagonal (one thread
      // per tree with contacts: J_t^T gamma over its contact list, then its
      // 6x6 block factored and solved in registers, FP64).  Taken when its
      // cost is below the plain start's; its evaluation then seeds
      // iteration 0.
      bool have_e4 = false;
      double e4_seed[4] = {0.0, 0.0, 0.0, 0.0};
      if (P.p.gamma0) {
        double e4p[4];
        bevaluate<NT, HT, NB>(w, e4p);
        for (int i = tid; i < n; i += NT) w.V(V_SAVE)[i] = w.V(V_V)[i];
        for (int t = tid; t < T; t += NT) {
          const int q0 = w.iw[BI_CSTART + t], q1 = w.iw[BI_CSTART + t + 1];
          if (q1 == q0) continue;  // no contact: v* already
          double r[NB];
#pragma unroll
          for (int a = 0; a < NB; ++a) r[a] = 0.0;
          for (int q = q0; q < q1; ++q) {
            const int ent = w.list[q];
            const int c = ent >> 1, side = ent & 1;
            const double* Jc = w.J + (size_t)c * 3 * 2 * NB + side * NB;
            const double* g = P.p.gamma0 + ((size_t)e * C + c) * 3;
            const double g0 = __ldg(g), g1 = __ldg(g + 1), g2 = __ldg(g + 2);
#pragma unroll
            for (int a = 0; a < NB; ++a)
              r[a] += __ldg(Jc + a) * g0 + __ldg(Jc + 2 * NB + a) * g1 + __ldg(Jc + 4 * NB + a) * g2;
          }
          double Lr[NB][NB], Dr[NB];
          const double* At = w.A + (size_t)t * NB * NB;
#pragma unroll
          for (int a = 0; a < NB; ++a)
#pragma unroll
            for (int b = 0; b <= a; ++b) Lr[a][b] = __ldg(At + a * NB + b);
#pragma unroll
          for (int b = 0; b < NB; ++b) {
            double d = Lr[b][b];
#pragma unroll
            for (int q = 0; q < b; ++q) d -= Lr[b][q] * Lr[b][q] * Dr[q];
            Dr[b] = d;
#pragma unroll
            for (int a = b + 1; a < NB; ++a) {
              double v = Lr[a][b];
#pragma unroll
              for (int q = 0; q < b; ++q) v -= Lr[a][q] * Lr[b][q] * Dr[q];
              Lr[a][b] = v / d;
            }
          }
#pragma unroll
          for (int a = 0; a < NB; ++a)
#pragma unroll
            for (int q = 0; q < a; ++q) r[a] -= Lr[a][q] * r[q];
#pragma unroll
          for (int a = 0; a < NB; ++a) r[a] /= Dr[a];
#pragma unroll
          for (int a = NB - 1; a >= 0; --a)
#pragma unroll
            for (int q = a + 1; q < NB; ++q) r[a] -= Lr[q][a] * r[q];
#pragma unroll
          for (int a = 0; a < NB; ++a) w.V(V_V)[t * NB + a] = w.V(V_VSTAR)[t * NB + a] + r[a];
        }
        __syncthreads();
        double e4c[4];
        bevaluate<NT, HT, NB>(w, e4c);
        if (e4c[0] < e4p[0]) {
          accepted = 1;
          have_e4 = true;
          for (int q = 0; q < 4; ++q) e4_seed[q] = e4c[q];
        } else {
          for (int i = tid; i < n; i += NT) w.V(V_V)[i] = w.V(V_SAVE)[i];
          __syncthreads();
        }
      }
      const double cost_min_alpha = LSV == SAPB_LS_MONOTONE_DECAY ? 0.0 : 0.5;
      for (int it = 0;; ++it) {
        double e4[4];
        if (have_e4) {
          for (int q = 0; q < 4; ++q) e4[q] = e4_seed[q];
          have_e4 = false;
        } else {
          bevaluate<NT, HT, NB>(w, e4);
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
          break;
        }
        if (it >= P.o.max_iterations) break;
        bassemble<NT, HT, NB>(w, P.o.diag_shift);
        bfactor<NT, HT, NB>(w);
        bsolve<NT, HT, NB>(w);
        double c4[4];
        line_coefficients<NT, HT, NB>(w, c4);
        LsResult r;
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
      }
    }
    // ---- outputs ------------------------------------------------------------
    for (int i = tid; i < n; i += NT) {
      const int gi = gidx(i);
      if (gi >= 0) P.out.v[base + gi] = w.V(V_V)[i];
    }
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
      if (P.out.warm_start_accepted) P.out.warm_start_accepted[e] = accepted;
    }
    __syncthreads();
  }
}

namespace blk {

template <typename HT>
int blocked_capacity(int T, int NB, int C, bool terms = false) {
  const BLayout L0 = make_blayout(T, NB, C, (int)sizeof(HT), 0, terms);
  const size_t per = (size_t)NB * NB * sizeof(HT) + 2;
  if (L0.total + 64 > kMaxSmemPerBlock) return 0;
  size_t cap = (kMaxSmemPerBlock - L0.total - 64) / per;
  const size_t most = (size_t)T * (T - 1) / 2;
  if (cap > most) cap = most;
  return (int)cap;
}

template <int NT, typename HT, int NB, int LSV>
cudaError_t launch_blocked_ls(const BlockedParams& P, cudaStream_t stream) {
  const BLayout L = make_blayout(P.p.trees_per_env, NB, P.p.max_contacts, (int)sizeof(HT), P.capacity,
                                 P.dof.has_pd || P.dof.has_limits);
  auto kern = blocked_solve_kernel<NT, HT, NB, LSV>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total);
  if (err != cudaSuccess) return err;
  int dev = 0, sms = 0, per_sm = 0;
  if ((err = cudaGetDevice(&dev)) != cudaSuccess) return err;
  if ((err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return err;
  if ((err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, L.total)) != cudaSuccess)
    return err;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  int blocks = sms * per_sm;
  if (blocks > P.p.num_envs) blocks = P.p.num_envs;
  if (blocks < 1) blocks = 1;
  if ((err = cudaMemsetAsync(P.queue, 0, sizeof(int32_t), stream)) != cudaSuccess) return err;
  kern<<<blocks, NT, L.total, stream>>>(P);
  return cudaGetLastError();
}

template <int NT, typename HT, int NB>
cudaError_t launch_blocked_nt(const BlockedParams& P, cudaStream_t stream) {
  switch (P.o.line_search_variant) {
    case SAPB_LS_ARMIJO_DECAY:
      return launch_blocked_ls<NT, HT, NB, SAPB_LS_ARMIJO_DECAY>(P, stream);
    case SAPB_LS_EXACT_ROOT:
      return launch_blocked_ls<NT, HT, NB, SAPB_LS_EXACT_ROOT>(P, stream);
    default:
      return launch_blocked_ls<NT, HT, NB, SAPB_LS_MONOTONE_DECAY>(P, stream);
  }
}

// One block size's kernels (both Hessian precisions, 128 or 256 threads per
// world, every line search), instantiated in a translation unit of its own
// (sapb_blocked_nb{6,7,12}.cu) so they compile in parallel.
template <int NB>
cudaError_t launch_blocked(const BlockedParams& P, bool fp32, int threads, cudaStream_t stream) {
  if (threads == 128)
    return fp32 ? launch_blocked_nt<128, float, NB>(P, stream) : launch_blocked_nt<128, double, NB>(P, stream);
  return fp32 ? launch_blocked_nt<256, float, NB>(P, stream) : launch_blocked_nt<256, double, NB>(P, stream);
}
extern template cudaError_t launch_blocked<6>(const BlockedParams&, bool, int, cudaStream_t);
extern template cudaError_t launch_blocked<7>(const BlockedParams&, bool, int, cudaStream_t);
extern template cudaError_t launch_blocked<12>(const BlockedParams&, bool, int, cudaStream_t);

}  // namespace blk

}  // namespace sapb
