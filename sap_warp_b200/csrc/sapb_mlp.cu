// sapb_mlp.cu -- the learned warm start: a per-contact MLP 12 -> 128 -> 128 ->
// 128 -> 3 (GELU, tanh form) with BF16 weights and activations and FP32
// accumulation, run and trained by hand-written sm_100a kernels:
//
//   forward    one CTA per 128-row tile (persistent), the three hidden layers
//              as tcgen05.mma (M=128, N=128, K=16 slices) into a TMEM
//              accumulator, bias + GELU epilogue from TMEM back to shared
//              memory as the next layer's operand, the 128 -> 3 output layer
//              on the CUDA cores from the same registers.  The training
//              variant also saves the pre-activations (FP32) and activations
//              (BF16 tile images) and forms dL/dy of the mean squared error.
//   backward   per tile: dZ3 from dy, then per layer the weight gradient
//              dW = dZ^T [H | 1] (bias gradient from the ones column) and the
//              input gradient dH = dZ W, both tcgen05.mma with MN-major
//              operand descriptors over the same shared-memory images, the
//              weight gradients accumulating in TMEM across the CTA's tiles.
//   adam       fused Adam step on the FP32 master parameters that writes the
//              BF16 operand images the forward reads.
//
// plus the two domain kernels around it: per-contact features from the
// stage-2 problem, and the map from the network output (a correction, in
// SAP's unprojected impulse variable, to the previous step's impulses) to
// starting impulses gamma0 through SAP's regularized cone projection (the
// solve maps gamma0 to v0 = v* + A^-1 J^T gamma0).  The reference warm-starts from the previous
// step's velocity only (sim/solver_sap.py:1441-1451); this network has no
// counterpart there.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "sapb_device.cuh"
#include "sapb_internal.h"
#include "sapb_umma.cuh"

namespace sapb {
namespace mlp {

constexpr int kRows = 128, kHid = 128, kIn = SAPB_MLP_INPUTS_PADDED, kInUsed = SAPB_MLP_INPUTS,
              kOut = SAPB_MLP_OUTPUTS;
constexpr int kImg = kRows * kHid;  // elements of one hidden-activation tile image

// FP32 master parameters: W1[128][12] b1 W2[128][128] b2 W3[128][128] b3 W4[3][128] b4.
constexpr int kMW1 = 0, kMB1 = kMW1 + kHid * kInUsed, kMW2 = kMB1 + kHid, kMB2 = kMW2 + kHid * kHid,
              kMW3 = kMB2 + kHid, kMB3 = kMW3 + kHid * kHid, kMW4 = kMB3 + kHid, kMB4 = kMW4 + kOut * kHid,
              kParams = kMB4 + kOut;
// BF16 operand images of W1 (128 x 16, inputs padded with zeros), W2, W3
// (core-matrix images with 128 rows = output units) and W4 row-major.
constexpr int kPW1 = 0, kPW2 = kPW1 + kHid * kIn, kPW3 = kPW2 + kHid * kHid, kPW4 = kPW3 + kHid * kHid,
              kPacked = kPW4 + kOut * kHid;
// FP32 biases b1 b2 b3 b4.
constexpr int kB1 = 0, kB2 = kHid, kB3 = 2 * kHid, kB4 = 3 * kHid, kBias = kB4 + kOut;
static_assert(kParams == SAPB_MLP_PARAM_COUNT, "parameter count");
static_assert(kPacked == SAPB_MLP_PACKED_COUNT, "packed count");
static_assert(kBias == SAPB_MLP_BIAS_COUNT, "bias count");

constexpr uint32_t kPolls = 1u << 22;  // bounded mbarrier waits
constexpr int kThreads = 256;          // 8 warps: lane quadrant = warp & 3, column half = warp >> 2

__device__ int g_mlp_error;

// GELU, tanh form (Hendrycks & Gimpel, 2016), and its derivative.
constexpr float kGeluC = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float kGeluA = 0.044715f;
__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu(float z) {
  const float t = tanh_approx(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * z * (1.0f + t);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float t = tanh_approx(kGeluC * (z + kGeluA * z * z * z));
  return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * kGeluC * (1.0f + 3.0f * kGeluA * z * z);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t u) { return __uint_as_float(u << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t u) { return __uint_as_float(u & 0xFFFF0000u); }
__device__ __forceinline__ float bf16_to_float(uint16_t u) { return __uint_as_float((uint32_t)u << 16); }

__device__ __forceinline__ void copy_bytes(void* dst, const void* src, int bytes) {
  uint4* d = reinterpret_cast<uint4*>(dst);
  const uint4* s = reinterpret_cast<const uint4*>(src);
  for (int i = threadIdx.x; i < bytes / 16; i += blockDim.x) d[i] = __ldg(s + i);
}

// ---- forward ----------------------------------------------------------------
struct FwdParams {
  uint32_t polls;          // bound of each mbarrier wait (polls)
  int drop_first_commit;   // test hook: each CTA's first MMA commit is not issued
  const int32_t* tile_active;  // [tiles] 0: skip the tile (its outputs are not written); NULL: every tile
  const uint16_t* wp;
  const float* bias;
  const uint16_t* x;  // [rows][16] BF16
  int rows;
  float* y;           // [rows][3] (optional in training)
  const float* target;
  uint16_t* act;      // [tiles][3][kImg] activation images
  float* pre;         // [tiles][3][128 unit][128 row]
  float* dy;          // [rows][3]
  float* loss;        // [1]
  float dy_scale;
};

constexpr int kFsW1 = 0;
constexpr int kFsW2 = kFsW1 + kHid * kIn * 2;
constexpr int kFsW3 = kFsW2 + kImg * 2;
constexpr int kFsX = kFsW3 + kImg * 2;
constexpr int kFsH = kFsX + kRows * kIn * 2;
constexpr int kFsW4 = kFsH + kImg * 2;
constexpr int kFsB = kFsW4 + kOut * kHid * 4;
constexpr int kFsY = kFsB + 416 * 4;
constexpr int kFwdSmem = kFsY + 2 * kRows * kOut * 4;

template <bool kTrain>
__global__ void __launch_bounds__(kThreads, 2) mlp_forward_kernel(const FwdParams P) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  uint16_t* W1s = reinterpret_cast<uint16_t*>(sm + kFsW1);
  uint16_t* W2s = reinterpret_cast<uint16_t*>(sm + kFsW2);
  uint16_t* W3s = reinterpret_cast<uint16_t*>(sm + kFsW3);
  uint16_t* Xs = reinterpret_cast<uint16_t*>(sm + kFsX);
  uint16_t* Hs = reinterpret_cast<uint16_t*>(sm + kFsH);
  float* W4f = reinterpret_cast<float*>(sm + kFsW4);
  float* Bs = reinterpret_cast<float*>(sm + kFsB);
  float* Yp = reinterpret_cast<float*>(sm + kFsY);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = warp & 3, hf = warp >> 2;
  const int r = 32 * q + lane;  // tile row of this thread
  if (P.tile_active) {  // a CTA with no active tile returns before staging the weights (uniform)
    bool any = false;
    const int ntiles = (P.rows + kRows - 1) / kRows;
    for (int t = blockIdx.x; t < ntiles && !any; t += gridDim.x) any = P.tile_active[t] != 0;
    if (!any) return;
  }

  copy_bytes(W1s, P.wp + kPW1, kHid * kIn * 2);
  copy_bytes(W2s, P.wp + kPW2, kImg * 2);
  copy_bytes(W3s, P.wp + kPW3, kImg * 2);
  for (int i = tid; i < kOut * kHid; i += kThreads) W4f[i] = bf16_to_float(P.wp[kPW4 + i]);
  for (int i = tid; i < kBias; i += kThreads) Bs[i] = P.bias[i];
  if (warp == 0) {
    umma::tmem_alloc(&tbase, 128);
    umma::tmem_relinquish();
  }
  if (tid == 0) umma::mbar_init(&bar, 1);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t trow = tmem + ((uint32_t)(32 * q) << 16);
  const uint32_t aX = umma::smem_u32(Xs), aH = umma::smem_u32(Hs);
  const uint32_t aW[3] = {umma::smem_u32(W1s), umma::smem_u32(W2s), umma::smem_u32(W3s)};
  constexpr uint32_t kIdesc = umma::idesc_bf16(128, 128, false, false);

  uint32_t phase = 0;
  bool ok = true, outstanding = false;
  const int tiles = (P.rows + kRows - 1) / kRows;
  bool first_tile = true;
  for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    if (P.tile_active && P.tile_active[tile] == 0) continue;  // uniform over the CTA, before any barrier
    const int row0 = tile * kRows;
    const bool drop_here = first_tile;
    first_tile = false;
    {
      const int rr = tid >> 1, ch = tid & 1;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (row0 + rr < P.rows) v = __ldg(reinterpret_cast<const uint4*>(P.x + (size_t)(row0 + rr) * kIn) + ch);
      *reinterpret_cast<uint4*>(Xs + umma::core_off(rr, 8 * ch, kRows)) = v;
    }
    umma::fence_proxy_async();
    __syncthreads();
    float y0 = 0.f, y1 = 0.f, y2 = 0.f;
    for (int layer = 0; layer < 3; ++layer) {
      // the test hook leaves this layer's barrier phase without a commit, so
      // its bounded wait cannot complete (nothing is left in flight)
      const bool drop = P.drop_first_commit && drop_here && layer == 0;
      if (tid == 0 && !drop) {
        umma::fence_after_sync();
        // A = X or H (K-major, 128 rows), B = W (K-major, 128 output rows).
        if (layer == 0)
          umma::mma_chain(tmem, aX, 2048, 128, 4096, aW[0], 2048, 128, 4096, 1, kIdesc, 0);
        else
          umma::mma_chain(tmem, aH, 2048, 128, 4096, aW[layer], 2048, 128, 4096, 8, kIdesc, 0);
        umma::commit(&bar);
      }
      const bool got = umma::mbar_wait(&bar, phase, P.polls);
      phase ^= 1u;
      ok = __syncthreads_and(got) != 0;
      if (!ok) {
        outstanding = !drop;  // a commit was issued and not yet seen
        break;
      }
      umma::fence_after_sync();
      const float* b = Bs + kB1 + layer * kHid;
#pragma unroll 1
      for (int c = 0; c < 4; ++c) {
        const int col = 64 * hf + 16 * c;
        float z[16];
        umma::tmem_ld16(trow + col, z);
        uint32_t pk[8];
#pragma unroll
        for (int j = 0; j < 16; j += 2) {
          const float za = z[j] + b[col + j], zb = z[j + 1] + b[col + j + 1];
          if (kTrain) {
            float* pre = P.pre + (((size_t)tile * 3 + layer) * kHid + col + j) * kRows + r;
            pre[0] = za;
            pre[kRows] = zb;
          }
          pk[j / 2] = pack_bf16(gelu(za), gelu(zb));
          if (layer == 2) {
            const float ha = bf16_lo(pk[j / 2]), hb = bf16_hi(pk[j / 2]);
            y0 += W4f[col + j] * ha + W4f[col + j + 1] * hb;
            y1 += W4f[kHid + col + j] * ha + W4f[kHid + col + j + 1] * hb;
            y2 += W4f[2 * kHid + col + j] * ha + W4f[2 * kHid + col + j + 1] * hb;
          }
        }
        const uint4 lo = make_uint4(pk[0], pk[1], pk[2], pk[3]), hi = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        if (layer < 2) {
          *reinterpret_cast<uint4*>(Hs + umma::core_off(r, col, kRows)) = lo;
          *reinterpret_cast<uint4*>(Hs + umma::core_off(r, col + 8, kRows)) = hi;
        }
        if (kTrain) {
          uint16_t* img = P.act + ((size_t)tile * 3 + layer) * kImg;
          *reinterpret_cast<uint4*>(img + umma::core_off(r, col, kRows)) = lo;
          *reinterpret_cast<uint4*>(img + umma::core_off(r, col + 8, kRows)) = hi;
        }
      }
      if (layer == 2) {
        Yp[(hf * kRows + r) * 3 + 0] = y0;
        Yp[(hf * kRows + r) * 3 + 1] = y1;
        Yp[(hf * kRows + r) * 3 + 2] = y2;
      }
      umma::fence_before_sync();
      umma::fence_proxy_async();
      __syncthreads();
    }
    if (!ok) break;
    if (hf == 0) {
      const int gr = row0 + r;
      float se = 0.f;
      if (gr < P.rows) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const float y = Yp[r * 3 + j] + Yp[(kRows + r) * 3 + j] + Bs[kB4 + j];
          if (P.y) P.y[(size_t)gr * 3 + j] = y;
          if (kTrain) {
            const float d = y - P.target[(size_t)gr * 3 + j];
            P.dy[(size_t)gr * 3 + j] = d * P.dy_scale;
            se += d * d;
          }
        }
      }
      if (kTrain) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
        if (lane == 0) atomicAdd(P.loss, se);
      }
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(&g_mlp_error, 1);
    // the commit still outstanding, if any, before the accumulator is freed
    if (outstanding) umma::mbar_wait(&bar, phase ^ 1u, kPolls);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, 128);
  }
}

// ---- backward ---------------------------------------------------------------
struct BwdParams {
  uint32_t polls;  // bound of each mbarrier wait (polls)
  const uint16_t* wp;
  const uint16_t* x;
  int rows;
  const uint16_t* act;
  const float* pre;
  const float* dy;
  float* grad;  // master layout, accumulated
};

// Images with a trailing ones column block (column 128, resp. 16) so the
// weight-gradient MMA also yields the bias gradient.
constexpr int kOnesImg = kImg + kRows * 16;  // 128 rows x 144 columns
constexpr int kBsW2 = 0;
constexpr int kBsW3 = kBsW2 + kImg * 2;
constexpr int kBsHA = kBsW3 + kImg * 2;
constexpr int kBsHB = kBsHA + kOnesImg * 2;
constexpr int kBsD = kBsHB + kOnesImg * 2;
constexpr int kBsX = kBsD + kImg * 2;
constexpr int kBsY = kBsX + kRows * 32 * 2;
constexpr int kBsW4 = kBsY + kRows * 16 * 2;
constexpr int kBsDb4 = kBsW4 + kOut * kHid * 4;
constexpr int kBwdSmem = kBsDb4 + 16;

// TMEM columns of the backward accumulators.
constexpr uint32_t kTDH = 0, kTW3 = 128, kTW2 = 272, kTW1 = 416, kTW4 = 448, kTCols = 512;

__global__ void __launch_bounds__(kThreads, 1) mlp_backward_kernel(const BwdParams P) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  uint16_t* W2s = reinterpret_cast<uint16_t*>(sm + kBsW2);
  uint16_t* W3s = reinterpret_cast<uint16_t*>(sm + kBsW3);
  uint16_t* HA = reinterpret_cast<uint16_t*>(sm + kBsHA);
  uint16_t* HB = reinterpret_cast<uint16_t*>(sm + kBsHB);
  uint16_t* D = reinterpret_cast<uint16_t*>(sm + kBsD);
  uint16_t* Xs = reinterpret_cast<uint16_t*>(sm + kBsX);
  uint16_t* Ys = reinterpret_cast<uint16_t*>(sm + kBsY);
  float* W4f = reinterpret_cast<float*>(sm + kBsW4);
  float* db4 = reinterpret_cast<float*>(sm + kBsDb4);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int q = warp & 3, hf = warp >> 2;
  const int r = 32 * q + lane;

  copy_bytes(W2s, P.wp + kPW2, kImg * 2);
  copy_bytes(W3s, P.wp + kPW3, kImg * 2);
  for (int i = tid; i < kOut * kHid; i += kThreads) W4f[i] = bf16_to_float(P.wp[kPW4 + i]);
  for (int i = tid; i < kRows * 16; i += kThreads) {  // ones blocks, X and dy images
    HA[kImg + i] = 0;
    HB[kImg + i] = 0;
  }
  for (int i = tid; i < kRows * 32; i += kThreads) Xs[i] = 0;
  for (int i = tid; i < kRows * 16; i += kThreads) Ys[i] = 0;
  if (tid < 4) db4[tid] = 0.f;
  __syncthreads();
  if (tid < kRows) {
    const uint16_t one = 0x3F80u;
    HA[umma::core_off(tid, kHid, kRows)] = one;
    HB[umma::core_off(tid, kHid, kRows)] = one;
    Xs[umma::core_off(tid, kIn, kRows)] = one;
  }
  if (warp == 0) {
    umma::tmem_alloc(&tbase, kTCols);
    umma::tmem_relinquish();
  }
  if (tid == 0) umma::mbar_init(&bar, 1);
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tbase;
  const uint32_t lane_off = (uint32_t)(32 * q) << 16;
  const uint32_t aHA = umma::smem_u32(HA), aHB = umma::smem_u32(HB), aD = umma::smem_u32(D),
                 aX = umma::smem_u32(Xs), aY = umma::smem_u32(Ys), aW2 = umma::smem_u32(W2s),
                 aW3 = umma::smem_u32(W3s);
  // Operand forms over the 128-row images: K-major (rows = M) and MN-major
  // (columns = M or N, rows = K).
  constexpr uint32_t kK_LBO = 2048, kK_SBO = 128, kK_STEP = 4096;
  constexpr uint32_t kMN_LBO = 128, kMN_SBO = 2048, kMN_STEP = 256;

  uint32_t phase = 0;
  bool ok = true, any = false;
  const int tiles = (P.rows + kRows - 1) / kRows;
  // dZ of this thread's row and 64 columns from dH (registers) and the saved
  // pre-activation, written to D.
  auto write_dz = [&](int tile, int layer, int col, const float (&dh)[16], bool valid) {
    const float* pre = P.pre + (((size_t)tile * 3 + layer) * kHid + col) * kRows + r;
    uint32_t pk[8];
#pragma unroll
    for (int j = 0; j < 16; j += 2) {
      const float a = valid ? dh[j] * gelu_grad(pre[(size_t)j * kRows]) : 0.f;
      const float b = valid ? dh[j + 1] * gelu_grad(pre[(size_t)(j + 1) * kRows]) : 0.f;
      pk[j / 2] = pack_bf16(a, b);
    }
    *reinterpret_cast<uint4*>(D + umma::core_off(r, col, kRows)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(D + umma::core_off(r, col + 8, kRows)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
  };
  auto wait_mma = [&]() -> bool {
    const bool got = umma::mbar_wait(&bar, phase, P.polls);
    phase ^= 1u;
    const bool all = __syncthreads_and(got) != 0;
    if (all) umma::fence_after_sync();
    return all;
  };

  for (int tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    const int row0 = tile * kRows;
    const int gr = row0 + r;
    const bool valid = gr < P.rows;
    const uint16_t* img = P.act + (size_t)tile * 3 * kImg;
    // (1) H3 -> HA, H2 -> HB, dy -> Ys, dZ3 -> D
    copy_bytes(HA, img + 2 * kImg, kImg * 2);
    copy_bytes(HB, img + 1 * kImg, kImg * 2);
    float dyr[3] = {0.f, 0.f, 0.f};
    if (valid) {
#pragma unroll
      for (int j = 0; j < 3; ++j) dyr[j] = P.dy[(size_t)gr * 3 + j];
    }
    if (hf == 0) {
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        Ys[umma::core_off(r, j, kRows)] = (uint16_t)(pack_bf16(dyr[j], 0.f) & 0xFFFFu);
        float s = dyr[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) atomicAdd(&db4[j], s);
      }
    }
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      const int col = 64 * hf + 16 * c;
      float dh[16];
#pragma unroll
      for (int j = 0; j < 16; ++j)
        dh[j] = dyr[0] * W4f[col + j] + dyr[1] * W4f[kHid + col + j] + dyr[2] * W4f[2 * kHid + col + j];
      write_dz(tile, 2, col, dh, valid);
    }
    umma::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t acc = any ? 1u : 0u;
      umma::mma_chain(tmem + kTW4, aHA, kMN_LBO, kMN_SBO, kMN_STEP, aY, kMN_LBO, kMN_SBO, kMN_STEP, 8,
                      umma::idesc_bf16(128, 16, true, true), acc);
      umma::mma_chain(tmem + kTW3, aD, kMN_LBO, kMN_SBO, kMN_STEP, aHB, kMN_LBO, kMN_SBO, kMN_STEP, 8,
                      umma::idesc_bf16(128, 144, true, true), acc);
      umma::mma_chain(tmem + kTDH, aD, kK_LBO, kK_SBO, kK_STEP, aW3, kMN_LBO, kMN_SBO, kMN_STEP, 8,
                      umma::idesc_bf16(128, 128, false, true), 0);
      umma::commit(&bar);
    }
    if (!(ok = wait_mma())) break;
    // (2) dZ2 -> D, H1 -> HA
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      const int col = 64 * hf + 16 * c;
      float dh[16];
      umma::tmem_ld16(tmem + kTDH + lane_off + col, dh);
      write_dz(tile, 1, col, dh, valid);
    }
    copy_bytes(HA, img, kImg * 2);
    umma::fence_before_sync();
    umma::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      const uint32_t acc = any ? 1u : 0u;
      umma::mma_chain(tmem + kTW2, aD, kMN_LBO, kMN_SBO, kMN_STEP, aHA, kMN_LBO, kMN_SBO, kMN_STEP, 8,
                      umma::idesc_bf16(128, 144, true, true), acc);
      umma::mma_chain(tmem + kTDH, aD, kK_LBO, kK_SBO, kK_STEP, aW2, kMN_LBO, kMN_SBO, kMN_STEP, 8,
                      umma::idesc_bf16(128, 128, false, true), 0);
      umma::commit(&bar);
    }
    if (!(ok = wait_mma())) break;
    // (3) dZ1 -> D, X -> Xs
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
      const int col = 64 * hf + 16 * c;
      float dh[16];
      umma::tmem_ld16(tmem + kTDH + lane_off + col, dh);
      write_dz(tile, 0, col, dh, valid);
    }
    {
      const int rr = tid >> 1, ch = tid & 1;
      uint4 v = make_uint4(0u, 0u, 0u, 0u);
      if (row0 + rr < P.rows) v = __ldg(reinterpret_cast<const uint4*>(P.x + (size_t)(row0 + rr) * kIn) + ch);
      *reinterpret_cast<uint4*>(Xs + umma::core_off(rr, 8 * ch, kRows)) = v;
    }
    umma::fence_before_sync();
    umma::fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after_sync();
      umma::mma_chain(tmem + kTW1, aD, kMN_LBO, kMN_SBO, kMN_STEP, aX, kMN_LBO, kMN_SBO, kMN_STEP, 8,
                      umma::idesc_bf16(128, 32, true, true), any ? 1u : 0u);
      umma::commit(&bar);
    }
    if (!(ok = wait_mma())) break;
    any = true;
  }
  if (ok && any) {
    const int unit = r;  // TMEM lane = output unit of the weight gradients
    float v[16];
    for (int layer = 0; layer < 2; ++layer) {  // W3 / W2: 144 columns = 9 chunks
      const uint32_t t = tmem + (layer == 0 ? kTW3 : kTW2) + lane_off;
      const int mw = layer == 0 ? kMW3 : kMW2, mb = layer == 0 ? kMB3 : kMB2;
      for (int ch = hf ? 5 : 0; ch < (hf ? 9 : 5); ++ch) {
        umma::tmem_ld16(t + 16 * ch, v);
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = 16 * ch + j;
          if (col < kHid) atomicAdd(&P.grad[mw + unit * kHid + col], v[j]);
          else if (col == kHid) atomicAdd(&P.grad[mb + unit], v[j]);
        }
      }
    }
    umma::tmem_ld16(tmem + kTW1 + lane_off + 16 * hf, v);
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int col = 16 * hf + j;
      if (col < kInUsed) atomicAdd(&P.grad[kMW1 + unit * kInUsed + col], v[j]);
      else if (col == kIn) atomicAdd(&P.grad[kMB1 + unit], v[j]);
    }
    if (hf == 0) {
      umma::tmem_ld16(tmem + kTW4 + lane_off, v);  // lane = hidden unit k, column = output j
#pragma unroll
      for (int j = 0; j < kOut; ++j) atomicAdd(&P.grad[kMW4 + j * kHid + unit], v[j]);
    }
    if (tid < kOut) atomicAdd(&P.grad[kMB4 + tid], db4[tid]);
  }
  if (!ok) {
    if (tid == 0) atomicExch(&g_mlp_error, 1);
    umma::mbar_wait(&bar, phase ^ 1u, kPolls);
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    umma::fence_after_sync();
    umma::tmem_dealloc(tmem, kTCols);
  }
}

// ---- parameters: packing and Adam -------------------------------------------
__device__ __forceinline__ void packed_slot(int i, int* wslot, int* bslot) {
  *wslot = -1;
  *bslot = -1;
  if (i < kMB1) {
    *wslot = kPW1 + umma::core_off(i / kInUsed, i % kInUsed, kHid);
  } else if (i < kMW2) {
    *bslot = kB1 + (i - kMB1);
  } else if (i < kMB2) {
    const int k = i - kMW2;
    *wslot = kPW2 + umma::core_off(k / kHid, k % kHid, kHid);
  } else if (i < kMW3) {
    *bslot = kB2 + (i - kMB2);
  } else if (i < kMB3) {
    const int k = i - kMW3;
    *wslot = kPW3 + umma::core_off(k / kHid, k % kHid, kHid);
  } else if (i < kMW4) {
    *bslot = kB3 + (i - kMB3);
  } else if (i < kMB4) {
    *wslot = kPW4 + (i - kMW4);
  } else {
    *bslot = kB4 + (i - kMB4);
  }
}

__device__ __forceinline__ void store_packed(int i, float p, uint16_t* wp, float* bias) {
  int ws, bs;
  packed_slot(i, &ws, &bs);
  if (ws >= 0) wp[ws] = (uint16_t)(pack_bf16(p, 0.f) & 0xFFFFu);
  if (bs >= 0) bias[bs] = p;
}

__global__ void pack_kernel(const float* params, uint16_t* wp, float* bias) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x)
    store_packed(i, params[i], wp, bias);
}

struct AdamArgs {
  float lr, beta1, beta2, eps, weight_decay, c1, c2;  // c1 = 1/(1-beta1^t), c2 = 1/(1-beta2^t)
};

__global__ void adam_kernel(float* p, const float* g, float* m, float* v, AdamArgs a, uint16_t* wp, float* bias) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = a.beta1 * m[i] + (1.f - a.beta1) * gi;
    const float vi = a.beta2 * v[i] + (1.f - a.beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float pi = p[i];
    pi -= a.lr * (mi * a.c1 / (sqrtf(vi * a.c2) + a.eps) + a.weight_decay * pi);
    p[i] = pi;
    store_packed(i, pi, wp, bias);
  }
}

// ---- contact features and starting impulses ----------------------------------
struct FeatParams {
  sapb_contact_problem p;
  const double* normal_up;
  const double* gamma_prev;
  const double* vc_star;
  sapb_warmstart_norm norm;
  double tau_fallback;
  uint16_t* x;
  float* raw;
};

// One warp per slot when J_c v* is formed here from J and v*; one thread
// per slot (every lane its own slot) when vc_star supplies it.
__global__ void features_kernel(const FeatParams P) {
  const int n = P.p.dof_per_env, C = P.p.max_contacts;
  const long slots = (long)P.p.num_envs * C;
  const bool per_thread = P.vc_star != nullptr;
  const int lane = per_thread ? 0 : (threadIdx.x & 31);
  const long stride = per_thread ? (long)gridDim.x * blockDim.x : (long)gridDim.x * (blockDim.x / 32);
  const long first = per_thread ? (long)blockIdx.x * blockDim.x + threadIdx.x
                                : (long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  for (long s = first; s < slots; s += stride) {
    const int e = (int)(s / C), c = (int)(s - (long)e * C);
    int count = P.p.contact_count[e];
    count = count < 0 ? 0 : (count > C ? C : count);
    float f[kInUsed];
#pragma unroll
    for (int k = 0; k < kInUsed; ++k) f[k] = 0.f;
    const bool live = c < count;
    if (live) {
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      if (P.vc_star) {
        a0 = P.vc_star[3 * s];
        a1 = P.vc_star[3 * s + 1];
        a2 = P.vc_star[3 * s + 2];
      } else {
        const double* J = P.p.jacobian + (size_t)s * 3 * n;
        const double* vs = P.p.v_star + (size_t)e * n;
        for (int i = lane; i < n; i += 32) {
          const double v = vs[i];
          a0 += J[i] * v;
          a1 += J[n + i] * v;
          a2 += J[2 * n + i] * v;
        }
        for (int o = 16; o > 0; o >>= 1) {
          a0 += __shfl_xor_sync(0xffffffffu, a0, o);
          a1 += __shfl_xor_sync(0xffffffffu, a1, o);
          a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
      }
      const double w = fmax(P.p.w_eff[s], 1.0e-12);
      f[0] = (float)P.p.phi0[s];
      f[1] = (float)a0;
      f[2] = (float)a1;
      f[3] = (float)a2;
      f[4] = P.normal_up ? (float)P.normal_up[s] : 1.f;
      f[5] = (float)P.p.mu[s];
      f[6] = (float)log10(fmax(P.p.stiffness[s], 1.0e-30));
      f[7] = (float)(P.p.tau_d ? P.p.tau_d[s] : P.tau_fallback);
      f[8] = (float)P.p.dt[e];
      if (P.gamma_prev) {
        f[9] = (float)(w * P.gamma_prev[3 * s + 0]);
        f[10] = (float)(w * P.gamma_prev[3 * s + 1]);
        f[11] = (float)(w * P.gamma_prev[3 * s + 2]);
      }
    }
    if (lane == 0) {
      if (P.raw) {
#pragma unroll
        for (int k = 0; k < kInUsed; ++k) P.raw[(size_t)s * kInUsed + k] = f[k];
      }
      if (P.x) {
        uint32_t pk[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          float a = 0.f, b = 0.f;
          if (live && 2 * k < kInUsed) a = (f[2 * k] - P.norm.feature_mean[2 * k]) * P.norm.feature_inv_std[2 * k];
          if (live && 2 * k + 1 < kInUsed)
            b = (f[2 * k + 1] - P.norm.feature_mean[2 * k + 1]) * P.norm.feature_inv_std[2 * k + 1];
          pk[k] = pack_bf16(a, b);
        }
        uint4* dst = reinterpret_cast<uint4*>(P.x + (size_t)s * kIn);
        dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
      }
    }
  }
}

struct ImpulseParams {
  sapb_contact_problem p;
  const float* y;
  const double* gamma_prev;  // residual base (NULL: 0)
  const int32_t* has_history;  // [E*C] 1: the slot keeps gamma_prev (NULL: the network everywhere)
  sapb_warmstart_norm norm;
  double beta, sigma, tau_fallback;
  double* gamma0;
};

// The network predicts a correction u (velocity units) of the unprojected
// impulse y = -R^-1 (vc - vhat) of SAP's regularized projection; gamma0 is
// the projection of y0 = gamma_prev + u / w_eff, i.e. the impulse SAP assigns
// to the contact velocity vc = vhat - R y0 (sim/contact_solve.py:743-921).
// Separated contacts have y_n well below zero and project to exactly zero.
__global__ void impulses_kernel(const ImpulseParams P) {
  const int C = P.p.max_contacts;
  const long slots = (long)P.p.num_envs * C;
  for (long s = (long)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += (long)gridDim.x * blockDim.x) {
    const int e = (int)(s / C), c = (int)(s - (long)e * C);
    int count = P.p.contact_count[e];
    count = count < 0 ? 0 : (count > C ? C : count);
    double g[3] = {0.0, 0.0, 0.0};
    if (c < count && P.has_history && P.has_history[s] && P.gamma_prev) {
      g[0] = P.gamma_prev[3 * s];
      g[1] = P.gamma_prev[3 * s + 1];
      g[2] = P.gamma_prev[3 * s + 2];
    } else if (c < count) {
      const double w = fmax(P.p.w_eff[s], 1.0e-12);
      double y[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        y[j] = ((double)P.y[3 * s + j] * P.norm.output_scale[j] + P.norm.output_shift[j]) / w;
        if (P.gamma_prev) y[j] += P.gamma_prev[3 * s + j];
      }
      const double tau = P.p.tau_d ? P.p.tau_d[s] : P.tau_fallback;
      const ContactConst cc = make_contact_const(P.p.phi0[s], P.p.w_eff[s], P.p.mu[s], P.p.stiffness[s], tau, P.beta,
                                                 P.sigma, P.p.dt[e]);
      double cost;
      project_contact(cc, -cc.rt * y[0], -cc.rt * y[1], cc.vhat_n - cc.rn * y[2], g, &cost, nullptr);
    }
    P.gamma0[3 * s + 0] = g[0];
    P.gamma0[3 * s + 1] = g[1];
    P.gamma0[3 * s + 2] = g[2];
  }
}

// Tiles of kRows slot rows that hold a live contact without history (the
// rows the network must predict).
__global__ void active_tiles_kernel(const sapb_contact_problem p, const int32_t* has_history, int32_t* tile_active) {
  const int C = p.max_contacts;
  const long slots = (long)p.num_envs * C;
  const long tiles = (slots + kRows - 1) / kRows;
  for (long t = (long)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); t < tiles;
       t += (long)gridDim.x * (blockDim.x / 32)) {
    bool need = false;
    for (long s = t * kRows + (threadIdx.x & 31); s < (t + 1) * kRows && s < slots; s += 32) {
      const int e = (int)(s / C), c = (int)(s - (long)e * C);
      int count = p.contact_count[e];
      count = count < 0 ? 0 : (count > C ? C : count);
      if (c < count && !(has_history && has_history[s])) need = true;
    }
    need = __any_sync(0xffffffffu, need);
    if ((threadIdx.x & 31) == 0) tile_active[t] = need ? 1 : 0;
  }
}

// ---- launch helpers -----------------------------------------------------------
// Wait bound of the MLP kernels (polls of an mbarrier), and the test hook
// that drops each forward CTA's first commit; set by sapb_mlp_test_hooks.
static uint32_t g_host_polls = kPolls;
static int g_host_drop_first_commit = 0;

static int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

static int32_t cuda_status(cudaError_t err, const char* what) {
  if (err == cudaSuccess) return SAPB_OK;
  set_last_error("%s: %s", what, cudaGetErrorString(err));
  return SAPB_ERR_CUDA;
}

}  // namespace mlp
}  // namespace sapb

using namespace sapb;
using namespace sapb::mlp;

extern "C" {

int32_t sapb_mlp_param_count(void) { return kParams; }
int32_t sapb_mlp_packed_count(void) { return kPacked; }
int32_t sapb_mlp_bias_count(void) { return kBias; }

int32_t sapb_mlp_train_buffer_sizes(int32_t rows, int64_t* act_elems, int64_t* pre_elems) {
  if (rows < 0 || !act_elems || !pre_elems) {
    set_last_error("sapb_mlp_train_buffer_sizes: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const int64_t tiles = (rows + kRows - 1) / kRows;
  *act_elems = tiles * 3 * (int64_t)kImg;
  *pre_elems = tiles * 3 * (int64_t)kImg;
  return SAPB_OK;
}

int32_t sapb_mlp_pack(const float* params, uint16_t* packed, float* bias, void* stream) {
  if (!params || !packed || !bias) {
    set_last_error("sapb_mlp_pack: null pointer");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t err = cudaMemsetAsync(packed, 0, sizeof(uint16_t) * kPacked, s);
  if (err == cudaSuccess) {
    pack_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(params, packed, bias);
    err = cudaGetLastError();
  }
  return cuda_status(err, "sapb_mlp_pack");
}

static int32_t forward_common(const uint16_t* packed, const float* bias, const uint16_t* x, int32_t rows, float* y,
                              const float* target, const sapb_mlp_train_buffers* buf, void* stream, bool train,
                              const int32_t* tile_active = nullptr) {
  if (!packed || !bias || rows < 0 || (rows > 0 && !x) || (!train && rows > 0 && !y) ||
      (train && (!buf || !target || !buf->act || !buf->pre || !buf->dy || !buf->loss))) {
    set_last_error("sapb_mlp_forward: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (rows == 0) return SAPB_OK;
  if ((reinterpret_cast<uintptr_t>(x) & 15) != 0) {
    set_last_error("sapb_mlp_forward: features must be 16-byte aligned");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  FwdParams P;
  memset(&P, 0, sizeof(P));
  P.polls = g_host_polls;
  P.drop_first_commit = g_host_drop_first_commit;
  P.tile_active = tile_active;
  P.wp = packed;
  P.bias = bias;
  P.x = x;
  P.rows = rows;
  P.y = y;
  if (train) {
    P.target = target;
    P.act = buf->act;
    P.pre = buf->pre;
    P.dy = buf->dy;
    P.loss = buf->loss;
    P.dy_scale = 2.0f / (3.0f * (float)rows);
  }
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  auto kern = train ? mlp_forward_kernel<true> : mlp_forward_kernel<false>;
  cudaError_t err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
  if (err != cudaSuccess) return cuda_status(err, "sapb_mlp_forward");
  const int tiles = (rows + kRows - 1) / kRows;
  int grid = 2 * sm_count();
  if (grid > tiles) grid = tiles;
  kern<<<grid, kThreads, kFwdSmem, s>>>(P);
  return cuda_status(cudaGetLastError(), "sapb_mlp_forward");
}

int32_t sapb_mlp_forward(const uint16_t* packed, const float* bias, const uint16_t* x, int32_t rows, float* y,
                         void* stream) {
  return forward_common(packed, bias, x, rows, y, nullptr, nullptr, stream, false);
}

int32_t sapb_mlp_forward_tiles(const uint16_t* packed, const float* bias, const uint16_t* x, int32_t rows, float* y,
                               const int32_t* tile_active, void* stream) {
  return forward_common(packed, bias, x, rows, y, nullptr, nullptr, stream, false, tile_active);
}

int32_t sapb_warmstart_active_tiles(const sapb_contact_problem* problem, const int32_t* has_history,
                                    int32_t* tile_active, void* stream) {
  if (!problem || !tile_active || problem->num_envs < 0 || problem->max_contacts < 0 ||
      (problem->num_envs > 0 && !problem->contact_count)) {
    set_last_error("sapb_warmstart_active_tiles: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const long slots = (long)problem->num_envs * problem->max_contacts;
  if (slots == 0) return SAPB_OK;
  const long tiles = (slots + kRows - 1) / kRows;
  long blocks = (tiles + 7) / 8;
  if (blocks > 8L * sm_count()) blocks = 8L * sm_count();
  active_tiles_kernel<<<(int)blocks, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(*problem, has_history,
                                                                                      tile_active);
  return cuda_status(cudaGetLastError(), "sapb_warmstart_active_tiles");
}

int32_t sapb_mlp_forward_train(const uint16_t* packed, const float* bias, const uint16_t* x, const float* target,
                               int32_t rows, const sapb_mlp_train_buffers* buf, float* y, void* stream) {
  return forward_common(packed, bias, x, rows, y, target, buf, stream, true);
}

int32_t sapb_mlp_backward(const uint16_t* packed, const uint16_t* x, int32_t rows, const sapb_mlp_train_buffers* buf,
                          float* grad, void* stream) {
  if (!packed || rows < 0 || !buf || !grad || (rows > 0 && (!x || !buf->act || !buf->pre || !buf->dy))) {
    set_last_error("sapb_mlp_backward: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (rows == 0) return SAPB_OK;
  if ((reinterpret_cast<uintptr_t>(x) & 15) != 0 || (reinterpret_cast<uintptr_t>(buf->act) & 15) != 0) {
    set_last_error("sapb_mlp_backward: features and activations must be 16-byte aligned");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  BwdParams P;
  P.polls = g_host_polls;
  P.wp = packed;
  P.x = x;
  P.rows = rows;
  P.act = buf->act;
  P.pre = buf->pre;
  P.dy = buf->dy;
  P.grad = grad;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t err = cudaFuncSetAttribute(mlp_backward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kBwdSmem);
  if (err != cudaSuccess) return cuda_status(err, "sapb_mlp_backward");
  const int tiles = (rows + kRows - 1) / kRows;
  int grid = sm_count();
  if (grid > tiles) grid = tiles;
  mlp_backward_kernel<<<grid, kThreads, kBwdSmem, s>>>(P);
  return cuda_status(cudaGetLastError(), "sapb_mlp_backward");
}

int32_t sapb_mlp_adam(float* params, const float* grad, float* m, float* v, const sapb_adam_options* opt,
                      int32_t step, uint16_t* packed, float* bias, void* stream) {
  if (!params || !grad || !m || !v || !opt || step < 1 || !packed || !bias) {
    set_last_error("sapb_mlp_adam: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  AdamArgs a;
  a.lr = opt->lr;
  a.beta1 = opt->beta1;
  a.beta2 = opt->beta2;
  a.eps = opt->eps;
  a.weight_decay = opt->weight_decay;
  a.c1 = (float)(1.0 / (1.0 - std::pow((double)opt->beta1, (double)step)));
  a.c2 = (float)(1.0 / (1.0 - std::pow((double)opt->beta2, (double)step)));
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(params, grad, m, v, a, packed, bias);
  return cuda_status(cudaGetLastError(), "sapb_mlp_adam");
}

int32_t sapb_mlp_test_hooks(int32_t wait_polls, int32_t drop_first_commit) {
  if (wait_polls < 0) {
    set_last_error("sapb_mlp_test_hooks: wait_polls must be >= 0");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  g_host_polls = wait_polls == 0 ? kPolls : (uint32_t)wait_polls;
  g_host_drop_first_commit = drop_first_commit != 0;
  return SAPB_OK;
}

int32_t sapb_mlp_error(void* stream) {
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int flag = 0, zero = 0;
  cudaError_t err = cudaMemcpyFromSymbolAsync(&flag, g_mlp_error, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaMemcpyToSymbolAsync(g_mlp_error, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) return cuda_status(err, "sapb_mlp_error");
  return flag ? SAPB_ERR_TIMEOUT : SAPB_OK;
}

int32_t sapb_warmstart_features(const sapb_contact_problem* problem, const double* normal_up,
                                const double* gamma_prev, const double* vc_star,
                                const sapb_warmstart_norm* norm, double tau_fallback, uint16_t* features,
                                float* raw, void* stream) {
  if (!problem || (!features && !raw) || (features && !norm) || problem->num_envs < 0 || problem->dof_per_env < 1 ||
      problem->max_contacts < 0) {
    set_last_error("sapb_warmstart_features: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const long slots = (long)problem->num_envs * problem->max_contacts;
  if (slots == 0) return SAPB_OK;
  if (!problem->contact_count || !problem->jacobian || !problem->v_star || !problem->phi0 || !problem->w_eff ||
      !problem->mu || !problem->stiffness || !problem->dt) {
    set_last_error("sapb_warmstart_features: missing problem array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (features && (reinterpret_cast<uintptr_t>(features) & 15) != 0) {
    set_last_error("sapb_warmstart_features: features must be 16-byte aligned");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  FeatParams P;
  memset(&P, 0, sizeof(P));
  P.p = *problem;
  P.normal_up = normal_up;
  P.gamma_prev = gamma_prev;
  P.vc_star = vc_star;
  if (norm) P.norm = *norm;
  P.tau_fallback = tau_fallback;
  P.x = features;
  P.raw = raw;
  long blocks = vc_star ? (slots + 255) / 256 : (slots + 7) / 8;
  if (blocks > 8L * sm_count()) blocks = 8L * sm_count();
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  features_kernel<<<(int)blocks, 256, 0, s>>>(P);
  return cuda_status(cudaGetLastError(), "sapb_warmstart_features");
}

int32_t sapb_warmstart_impulses(const sapb_contact_problem* problem, const float* mlp_out,
                                const double* gamma_prev, const int32_t* has_history,
                                const sapb_warmstart_norm* norm, const sapb_solve_options* opts, double* gamma0,
                                void* stream) {
  if (!problem || !mlp_out || !norm || !opts || !gamma0 || problem->num_envs < 0 || problem->max_contacts < 0) {
    set_last_error("sapb_warmstart_impulses: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const long slots = (long)problem->num_envs * problem->max_contacts;
  if (slots == 0) return SAPB_OK;
  if (!problem->contact_count || !problem->w_eff || !problem->mu || !problem->phi0 || !problem->stiffness ||
      !problem->dt) {
    set_last_error("sapb_warmstart_impulses: missing problem array");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  ImpulseParams P;
  P.p = *problem;
  P.y = mlp_out;
  P.gamma_prev = gamma_prev;
  P.has_history = has_history;
  P.norm = *norm;
  P.beta = opts->contact_beta;
  P.sigma = opts->contact_sigma;
  P.tau_fallback = opts->contact_tau_d;
  P.gamma0 = gamma0;
  long blocks = (slots + 255) / 256;
  if (blocks > 8L * sm_count()) blocks = 8L * sm_count();
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  impulses_kernel<<<(int)blocks, 256, 0, s>>>(P);
  return cuda_status(cudaGetLastError(), "sapb_warmstart_impulses");
}

}  // extern "C"
