// sapb_history.cu -- impulses carried across steps by contact identity.
//
// The previous-impulse warm start needs, for each of this step's contact
// slots, the impulse the same contact had at the end of the previous step.
// Slots are the contacts of a world in flat-buffer order, so when a contact
// appears or vanishes the later slots shift.  A contact is recognised by its
// key: the shape pair and the shape1 witness point in shape1's body frame
// (constant for a sphere centre or a box corner).  Per world (one CTA) the
// previous keys and this step's are staged in shared memory; a slot takes
// the impulse of the previous slot with the same pair whose point is the
// nearest to its own, provided that it is also the nearest of this step's
// slots to that previous contact (mutual nearest, searched within 64 slots
// of each side); then this step's keys replace the previous ones.  With an
// order of 2 or 3 the slots also carry the impulses of the steps before
// (the previous call's carried impulses and their predecessors, by the
// previous slots), and the start impulse is the polynomial through the last
// `order` impulses of the contact evaluated one step on: 2 g1 - g2 (linear),
// 3 g1 - 3 g2 + g3 (quadratic), g1 with one known, 0 for a new contact.  No
// counterpart in the reference, whose warm start is the previous velocity.
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "sapb_internal.h"

namespace sapb {
namespace {

constexpr int kHistMaxThreads = 128;  // a CTA per world: one warp per 32 slots, at most four
constexpr int kHistWindow = 64;
constexpr int kHistMaxOrder = 3;

struct Key {
  int s0, s1;
  double x, y, z;
};

__device__ __forceinline__ double dist2(const Key& a, const Key& b) {
  const double dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
  return dx * dx + dy * dy + dz * dz;
}

// rank_src (the free-motion launch's slot list, [W][C] flat indices in
// arrival order): ranked by flat index in place first and used as the slots'
// sources; NULL: the sources are H.contact_source.
__global__ void __launch_bounds__(kHistMaxThreads) history_kernel(const sapb_contact_history H, int32_t* rank_src) {
  const int kHistThreads = blockDim.x;
  extern __shared__ __align__(16) unsigned char smem[];
  const int C = H.max_contacts, e = blockIdx.x;
  Key* prev = reinterpret_cast<Key*>(smem);
  Key* cur = prev + C;
  const int order = H.order < 1 ? 1 : (H.order > kHistMaxOrder ? kHistMaxOrder : H.order);
  // order >= 2: the previous call's carried impulses (and order 3: the ones
  // before them) and known-impulse counts, staged before any slot is rewritten
  double* pg1 = reinterpret_cast<double*>(cur + C);
  double* pg2 = pg1 + 3 * C;
  int* pdepth = reinterpret_cast<int*>(pg2 + 3 * C);
  int* srcs = pdepth + C;  // arrival order [C], then ranked [C]
  int np = H.key_count[e];
  np = np < 0 ? 0 : (np > C ? C : np);
  int nc = H.contact_count[e];
  nc = nc < 0 ? 0 : (nc > C ? C : nc);
  const size_t base = (size_t)e * C;
  if (rank_src) {
    // the canonical slot order: this step's contacts by flat index (distinct)
    for (int c = threadIdx.x; c < nc; c += kHistThreads) srcs[c] = rank_src[base + c];
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += kHistThreads) {
      const int v = srcs[c];
      int rank = 0;
      for (int j = 0; j < nc; ++j) rank += srcs[j] < v ? 1 : 0;
      srcs[C + rank] = v;
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nc; c += kHistThreads) rank_src[base + c] = srcs[C + c];
  }
  for (int c = threadIdx.x; c < np; c += kHistThreads) {
    Key k;
    k.s0 = H.key_shape[2 * (base + c)];
    k.s1 = H.key_shape[2 * (base + c) + 1];
    k.x = H.key_point[3 * (base + c)];
    k.y = H.key_point[3 * (base + c) + 1];
    k.z = H.key_point[3 * (base + c) + 2];
    prev[c] = k;
    if (order >= 2) {
      const int d = H.has_history[base + c];
      pdepth[c] = d < 0 ? 0 : (d > order ? order : d);
      for (int r = 0; r < 3; ++r) {
        pg1[3 * c + r] = H.gamma_hist[3 * (base + c) + r];
        pg2[3 * c + r] = order >= 3 ? H.gamma_older[3 * (base + c) + r] : 0.0;
      }
    }
  }
  for (int c = threadIdx.x; c < nc; c += kHistThreads) {
    const int src = rank_src ? srcs[C + c] : H.contact_source[base + c];
    Key k{-2, -2, 0.0, 0.0, 0.0};
    if (src >= 0 && src < H.num_flat) {
      k.s0 = H.flat_shape0[src];
      k.s1 = H.flat_shape1[src];
      k.x = H.flat_point1[3 * (size_t)src];
      k.y = H.flat_point1[3 * (size_t)src + 1];
      k.z = H.flat_point1[3 * (size_t)src + 2];
    }
    cur[c] = k;
  }
  __syncthreads();
  for (int c = threadIdx.x; c < C; c += kHistThreads) {
    int best = -1;
    if (c < nc && cur[c].s0 != -2) {
      const Key k = cur[c];
      double bd = DBL_MAX;
      const int lo = c - kHistWindow > 0 ? c - kHistWindow : 0;
      const int hi = c + kHistWindow + 1 < np ? c + kHistWindow + 1 : np;
      for (int p = lo; p < hi; ++p) {
        if (prev[p].s0 != k.s0 || prev[p].s1 != k.s1) continue;
        const double d = dist2(k, prev[p]);
        if (d < bd) {
          bd = d;
          best = p;
        }
      }
      if (best >= 0) {  // mutual: this slot is the nearest of this step's to it
        const Key kp = prev[best];
        const int lo2 = best - kHistWindow > 0 ? best - kHistWindow : 0;
        const int hi2 = best + kHistWindow + 1 < nc ? best + kHistWindow + 1 : nc;
        for (int q = lo2; q < hi2; ++q) {
          if (q == c || cur[q].s0 != kp.s0 || cur[q].s1 != kp.s1) continue;
          const double d = dist2(kp, cur[q]);
          if (d < bd || (d == bd && q < c)) {
            best = -1;
            break;
          }
        }
      }
    }
    const size_t s = base + c;
    // g1: the last solve's impulse; g2, g3: the ones before (known when the
    // matched previous slot knew them)
    double g1[3] = {0.0, 0.0, 0.0}, g2[3] = {0.0, 0.0, 0.0}, g3[3] = {0.0, 0.0, 0.0};
    int depth = 0;
    if (best >= 0) {
      const size_t ps = base + best;
      for (int r = 0; r < 3; ++r) g1[r] = H.gamma_prev[3 * ps + r];
      depth = 1;
      if (order >= 2) {
        depth = pdepth[best] + 1 < order ? pdepth[best] + 1 : order;
        for (int r = 0; r < 3; ++r) {
          g2[r] = pg1[3 * best + r];
          g3[r] = pg2[3 * best + r];
        }
      }
    }
    for (int r = 0; r < 3; ++r) {
      H.gamma_hist[3 * s + r] = g1[r];
      if (order >= 3) H.gamma_older[3 * s + r] = depth >= 2 ? g2[r] : 0.0;
    }
    if (H.has_history) H.has_history[s] = depth;
    if (H.gamma_start) {
      for (int r = 0; r < 3; ++r) {
        double g = g1[r];  // depth 1 (0 for a new contact)
        if (depth == 2) g = 2.0 * g1[r] - g2[r];
        else if (depth == 3) g = 3.0 * g1[r] - 3.0 * g2[r] + g3[r];
        H.gamma_start[3 * s + r] = g;
      }
    }
  }
  __syncthreads();  // every slot has read the previous keys
  for (int c = threadIdx.x; c < nc; c += kHistThreads) {
    const size_t s = base + c;
    H.key_shape[2 * s] = cur[c].s0;
    H.key_shape[2 * s + 1] = cur[c].s1;
    H.key_point[3 * s] = cur[c].x;
    H.key_point[3 * s + 1] = cur[c].y;
    H.key_point[3 * s + 2] = cur[c].z;
  }
  if (threadIdx.x == 0) H.key_count[e] = nc;
}

}  // namespace
}  // namespace sapb

using namespace sapb;

namespace sapb {

int32_t history_launch(const sapb_contact_history* h, int32_t* rank_src, cudaStream_t stream) {
  if (!h || h->num_envs < 0 || h->max_contacts < 1 || h->num_flat < 0 || h->order < 0 || h->order > kHistMaxOrder ||
      (h->num_envs > 0 && (!h->contact_count || (!h->contact_source && !rank_src) || !h->key_shape ||
                           !h->key_point || !h->key_count || !h->gamma_prev || !h->gamma_hist ||
                           (h->order >= 2 && !h->has_history) || (h->order >= 3 && !h->gamma_older) ||
                           (h->num_flat > 0 && (!h->flat_shape0 || !h->flat_shape1 || !h->flat_point1))))) {
    set_last_error("sapb_contact_history_update: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (h->num_envs == 0) return SAPB_OK;
  const size_t smem = (sizeof(Key) * 2 + sizeof(double) * 6 + sizeof(int) * 3) * (size_t)h->max_contacts;
  if (smem > kMaxSmemPerBlock) {
    set_last_error("sapb_contact_history_update: %d slots per world exceed shared memory", h->max_contacts);
    return SAPB_ERR_UNSUPPORTED;
  }
  cudaError_t err = cudaFuncSetAttribute(history_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err == cudaSuccess) {
    int threads = (h->max_contacts + 31) / 32 * 32;
    if (threads > kHistMaxThreads) threads = kHistMaxThreads;
    history_kernel<<<h->num_envs, threads, smem, stream>>>(*h, rank_src);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) {
    set_last_error("sapb_contact_history_update: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

}  // namespace sapb

extern "C" int32_t sapb_contact_history_update(const sapb_contact_history* h, void* stream) {
  return history_launch(h, nullptr, static_cast<cudaStream_t>(stream));
}
