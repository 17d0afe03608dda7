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

// In-place right-looking LDL^T of the lower triangle of H (row stride ldH):
// afterwards H_ik = L_ik d_k below the diagonal (L unit lower), d_k on it,
// dinv[k] = 1/d_k.  8-column blocks: the diagonal block by warp 0, the panel
// and the trailing update by the whole block, three barriers per block.
// H must be complete when called (barrier before); complete on return.
template <int NT, typename T>
__device__ void ldlt_blocked(T* H, int n, int ldH, T* dinv, const uint16_t* tri) {
  const int tid = threadIdx.x;
  constexpr int B = 8;
  const int lane = tid & 31;
  for (int K = 0; K < n; K += B) {
    const int bs = min(B, n - K);
    // (1) diagonal block, unblocked, by warp 0
    if (tid < 32) {
      for (int s = 0; s < bs; ++s) {
        const int ks = K + s;
        const T rinv = fast_recip(H[(size_t)ks * ldH + ks]);
        if (lane == 0) dinv[ks] = rinv;
        const int m = bs - s - 1;  // trailing entries (a, c), s < c <= a < bs
        for (int q = lane; q < m * (m + 1) / 2; q += 32) {
          int a = 0;
          while ((a + 1) * (a + 2) / 2 <= q) ++a;
          const int c = q - a * (a + 1) / 2;
          const int i = ks + 1 + a, j = ks + 1 + c;
          H[(size_t)i * ldH + j] -= (H[(size_t)i * ldH + ks] * rinv) * H[(size_t)j * ldH + ks];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    const int rest = n - K - bs;
    if (rest <= 0) break;
    // (2) panel rows: P L_K^T = H_panel (forward substitution over the block columns)
    for (int t = tid; t < rest; t += NT) {
      const int i = K + bs + t;
      T p[B];
#pragma unroll
      for (int c = 0; c < B; ++c) {
        if (c < bs) {
          T h = H[(size_t)i * ldH + K + c];
#pragma unroll
          for (int m2 = 0; m2 < B; ++m2)
            if (m2 < c) h -= p[m2] * (H[(size_t)(K + c) * ldH + K + m2] * dinv[K + m2]);
          p[c] = h;
          H[(size_t)i * ldH + K + c] = h;
        }
      }
    }
    __syncthreads();
    // (3) trailing update of entries (i, j), j >= K + bs: the first
    // rest*(rest+1)/2 entries of the column-descending triangle list.
    const int cnt = rest * (rest + 1) / 2;
    for (int e = tid; e < cnt; e += NT) {
      const int ij = tri[e];
      const int i = ij >> 8, j = ij & 255;
      T acc = H[(size_t)i * ldH + j];
#pragma unroll
      for (int c = 0; c < B; ++c)
        if (c < bs) acc -= H[(size_t)i * ldH + K + c] * dinv[K + c] * H[(size_t)j * ldH + K + c];
      H[(size_t)i * ldH + j] = acc;
    }
    __syncthreads();
  }
}

}  // namespace sapb
