// sapb_ldlt.cuh -- blocked LDL^T of a small symmetric positive definite matrix
// held in shared memory by one thread block (the per-world dense factor of
// the reference's BlockCholeskySolverBatched, sim/blocked_cholesky.py:414-604,
// as LDL^T: no square roots).
#pragma once

#include <cstdint>

#include "sapb_device.cuh"

namespace sapb {

// Column-descending list of the lower triangle below row 0: entries
// (i << 8 | j) for j = n-1 .. 1, i = j .. n-1.  The trailing triangle of
// columns > k is its first m(m+1)/2 entries, m = n-1-k.  n <= 256.
template <int NT>
__device__ __forceinline__ void build_triangle_list(uint16_t* tri, int n) {
  for (int j = n - 1 - (int)threadIdx.x; j >= 1; j -= NT) {
    const int off = (n - 1 - j) * (n - j) / 2;
    for (int i = j; i < n; ++i) tri[off + (i - j)] = (uint16_t)((i << 8) | j);
  }
}

// In-place right-looking LDL^T of the lower triangle of H (row stride ldH;
// tri: the triangle list of build_triangle_list for n + tri_shift DOFs):
// afterwards H_ik = L_ik d_k below the diagonal (L unit lower), d_k on it,
// dinv[k] = 1/d_k.  B-column blocks, two barriers per block:
// every thread factors the block's diagonal block in
// registers (it is final once the previous trailing update is done), the rows
// under it (the panel) are solved against it in registers, one per thread;
// after the panel's barrier threads below bs write the block's rows back
// while the trailing update runs.  The arithmetic is the right-looking
// recurrence on the stored form W_ik = L_ik d_k:
//   d_k = H_kk - sum_{e<k} W_ke^2 / d_e,  W_ik = H_ik - sum_{e<k} W_ie W_ke / d_e.
// H must be complete when called (barrier before); complete on return.
template <int NT, typename T, int B>
__device__ void ldlt_blocked(T* H, int n, int ldH, T* dinv, const uint16_t* tri, int tri_shift = 0) {
  static_assert(B >= 1 && B <= 8, "block width");
  const int tid = threadIdx.x;
  for (int K = 0; K < n; K += B) {
    const int bs = min(B, n - K);
    const int rest = n - K - bs;
    // (1) the diagonal block, in registers (padding rows: identity)
    T W[B][B], R[B];
#pragma unroll
    for (int a = 0; a < B; ++a)
#pragma unroll
      for (int b = 0; b <= a; ++b)
        W[a][b] = (a < bs) ? H[(size_t)(K + a) * ldH + K + b] : (a == b ? T(1) : T(0));
#pragma unroll
    for (int b = 0; b < B; ++b) {
      T d = W[b][b];
#pragma unroll
      for (int e = 0; e < b; ++e) d -= W[b][e] * R[e] * W[b][e];
      W[b][b] = d;
      R[b] = fast_recip(d);
#pragma unroll
      for (int a = b + 1; a < B; ++a) {
        T v = W[a][b];
#pragma unroll
        for (int e = 0; e < b; ++e) v -= W[a][e] * R[e] * W[b][e];
        W[a][b] = v;
      }
    }
    // The factored rows go back to H only once every thread has read the
    // block: after the panel's barrier (the trailing update never touches
    // the diagonal block), or after a barrier of its own for the last block.
    auto store_block = [&]() {
      if (tid < bs) {
#pragma unroll
        for (int a = 0; a < B; ++a) {
          if (a != tid) continue;
#pragma unroll
          for (int b = 0; b <= a; ++b) H[(size_t)(K + a) * ldH + K + b] = W[a][b];
          dinv[K + a] = R[a];
        }
      }
    };
    if (rest <= 0) {
      __syncthreads();
      store_block();
      __syncthreads();
      break;
    }
    // (2) panel rows: P L_K^T = H_panel (forward substitution over the block columns)
    for (int t = tid; t < rest; t += NT) {
      const int i = K + bs + t;
      T p[B];
#pragma unroll
      for (int c = 0; c < B; ++c) {
        if (c < bs) {
          T h = H[(size_t)i * ldH + K + c];
#pragma unroll
          for (int m2 = 0; m2 < c; ++m2) h -= p[m2] * (W[c][m2] * R[m2]);
          p[c] = h;
          H[(size_t)i * ldH + K + c] = h;
        }
      }
    }
    __syncthreads();
    store_block();
    // (3) trailing update of entries (i, j), j >= K + bs: the first
    // rest*(rest+1)/2 entries of the column-descending triangle list.
    const int cnt = rest * (rest + 1) / 2;
    for (int e = tid; e < cnt; e += NT) {
      const int ij = tri[e];
      const int i = (ij >> 8) - tri_shift, j = (ij & 255) - tri_shift;
      T acc = H[(size_t)i * ldH + j];
#pragma unroll
      for (int c = 0; c < B; ++c)
        if (c < bs) acc -= H[(size_t)i * ldH + K + c] * R[c] * H[(size_t)j * ldH + K + c];
      H[(size_t)i * ldH + j] = acc;
    }
    __syncthreads();
  }
}

// x <- -A^-1 x (neg) or A^-1 x with the LDL^T that ldlt_blocked left in H
// and dinv, by the whole block: forward L z = b, zd = D^-1 z, backward
// L^T x = zd, over the same blocks as the factorization.  Per block every
// thread solves the small diagonal system in registers, then threads update
// the remaining rows (one row each); two barriers per block.  x (FP64 or T)
// holds the intermediate vectors; the arithmetic is in T.  A pivot that is
// not positive / finite makes x NaN.  x complete on entry (barrier before)
// and on return.
template <int NT, typename T, typename X>
__device__ void ldlt_solve_blocked(const T* H, int n, int ldH, const T* dinv, X* x, bool neg) {
  const int tid = threadIdx.x;
  constexpr int B = sizeof(T) == 4 ? 8 : 6;
  bool ok = true;
  for (int k = 0; k < n; ++k) {
    const T d = H[(size_t)k * ldH + k];
    if (!(d > T(0)) || !isfinite(double(d))) ok = false;
  }
  const T sgn = neg ? T(-1) : T(1);
  // forward
  for (int K = 0; K < n; K += B) {
    const int bs = min(B, n - K);
    T z[B], R[B];
#pragma unroll
    for (int a = 0; a < B; ++a) {
      R[a] = a < bs ? dinv[K + a] : T(0);
      T v = a < bs ? T(x[K + a]) : T(0);
      if (K == 0) v *= sgn;
#pragma unroll
      for (int e = 0; e < a; ++e)
        if (a < bs) v -= H[(size_t)(K + a) * ldH + K + e] * R[e] * z[e];
      z[a] = v;
    }
    __syncthreads();  // every thread has read the block's entries of x
    if (tid < bs) {
#pragma unroll
      for (int a = 0; a < B; ++a)
        if (a == tid) x[K + a] = X(z[a] * R[a]);
    }
    for (int i = K + bs + tid; i < n; i += NT) {
      T acc = T(x[i]);
      if (K == 0) acc *= sgn;
#pragma unroll
      for (int c = 0; c < B; ++c)
        if (c < bs) acc -= H[(size_t)i * ldH + K + c] * R[c] * z[c];
      x[i] = X(acc);
    }
    __syncthreads();
  }
  // backward
  const int last = ((n - 1) / B) * B;
  for (int K = last; K >= 0; K -= B) {
    const int bs = min(B, n - K);
    T xb[B];
#pragma unroll
    for (int a = B - 1; a >= 0; --a) {
      if (a >= bs) {
        xb[a] = T(0);
        continue;
      }
      T v = T(x[K + a]);
      const T ra = dinv[K + a];
#pragma unroll
      for (int c = a + 1; c < B; ++c)
        if (c < bs) v -= H[(size_t)(K + c) * ldH + K + a] * ra * xb[c];
      xb[a] = v;
    }
    __syncthreads();
    if (tid < bs) {
#pragma unroll
      for (int a = 0; a < B; ++a)
        if (a == tid) x[K + a] = X(xb[a]);
    }
    for (int i = tid; i < K; i += NT) {
      T acc = T(0);
#pragma unroll
      for (int c = 0; c < B; ++c)
        if (c < bs) acc += H[(size_t)(K + c) * ldH + i] * xb[c];
      x[i] = X(T(x[i]) - dinv[i] * acc);
    }
    __syncthreads();
  }
  if (!ok) {
    for (int i = tid; i < n; i += NT) x[i] = X(__longlong_as_double(0x7ff8000000000000ULL));
    __syncthreads();
  }
}

// x = A^-1 b (or -A^-1 b with neg) by the calling warp alone (all 32 lanes;
// no block barrier) with the LDL^T that ldlt_blocked left in H and dinv:
// lanes own rows lane and lane + 32 (n <= 64); forward z = D^-1 L^-1 b with
// the pivot broadcast by shuffles, then backward x = L^-T z.  b is read before
// x is written (they may alias).  `ok` false (a pivot not positive / finite,
// ldlt_pivots_ok_warp) makes x NaN.
template <typename T>
__device__ void ldlt_solve_warp(const T* H, int n, int ldH, const T* dinv, const double* b, double* x,
                                bool neg, bool ok) {
  const int lane = threadIdx.x & 31;
  const T sg = neg ? T(-1) : T(1);
  T h0 = lane < n ? sg * T(b[lane]) : T(0);
  T h1 = lane + 32 < n ? sg * T(b[lane + 32]) : T(0);
  for (int k = 0; k < n; ++k) {
    const T zk = __shfl_sync(0xffffffffu, k < 32 ? h0 : h1, k & 31) * dinv[k];
    if (lane == (k & 31)) {
      if (k < 32) h0 = zk;
      else h1 = zk;
    }
    if (lane > k && lane < n) h0 -= H[(size_t)lane * ldH + k] * zk;
    if (lane + 32 > k && lane + 32 < n) h1 -= H[(size_t)(lane + 32) * ldH + k] * zk;
  }
  T s0 = T(0), s1 = T(0);
  for (int i = n - 1; i >= 0; --i) {
    T xi_local = T(0);
    if (lane == (i & 31)) {
      xi_local = i < 32 ? h0 - s0 * dinv[i] : h1 - s1 * dinv[i];
      if (i < 32) h0 = xi_local;
      else h1 = xi_local;
    }
    const T xi = __shfl_sync(0xffffffffu, xi_local, i & 31);
    if (lane < i) s0 += H[(size_t)i * ldH + lane] * xi;
    if (lane + 32 < i) s1 += H[(size_t)i * ldH + lane + 32] * xi;
  }
  const double nanv = __longlong_as_double(0x7ff8000000000000ULL);
  __syncwarp();
  if (lane < n) x[lane] = ok ? double(h0) : nanv;
  if (lane + 32 < n) x[lane + 32] = ok ? double(h1) : nanv;
}

// Whether every pivot of a stored LDL^T is positive and finite (the warp's
// lanes check two each), returned to every lane.
template <typename T>
__device__ bool ldlt_pivots_ok_warp(const T* H, int n, int ldH) {
  const int lane = threadIdx.x & 31;
  bool ok = true;
  for (int k = lane; k < n; k += 32) {
    const T d = H[(size_t)k * ldH + k];
    if (!(d > T(0)) || !isfinite(double(d))) ok = false;
  }
  return __all_sync(0xffffffffu, ok);
}

}  // namespace sapb
