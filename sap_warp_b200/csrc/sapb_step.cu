// sapb_step.cu -- the whole SAP step behind one handle, for hosts that drive
// the step from C (SolverSAP.__init__ / .step, sim/solver_sap.py:749-968 and
// :1388-1494, as a C API): sapb_create allocates every work buffer once,
// sapb_step runs free motion + contact rows, the contact solve (with the
// previous-velocity, previous-impulse or learned warm start; dense or
// tree-blocked; equal or uneven worlds) and the position integration on the
// caller's stream without host synchronisation (so a caller may capture it
// in a CUDA graph), sapb_get_status copies the per-world solve statuses,
// sapb_destroy frees the buffers.
//
// Also the stable work-order sort (sapb_world_order): the persistent solve
// takes the worlds in the order of the previous step's Newton iterations,
// most first; one CTA sorts keys (iterations descending, world index
// ascending) by a bitonic network in shared memory.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "sapb_internal.h"

namespace sapb {
namespace {

constexpr int kOrderThreads = 1024;
constexpr int kOrderMaxWorlds = 32768;  // 2^15 keys of 4 bytes: 128 KB of shared memory
constexpr uint32_t kIndexBits = 16;     // world index in the low bits (< 2^16 after the check)

// Keys (0x7fff - min(iterations, 0x7fff)) << 16 | index sorted ascending:
// iterations descending, ties in index order (stable).  Padding keys
// 0xffffffff sort last.
__global__ void __launch_bounds__(kOrderThreads) world_order_kernel(const int32_t* iters, int32_t W, int32_t N,
                                                                    int32_t* order) {
  extern __shared__ uint32_t keys[];
  for (int i = threadIdx.x; i < N; i += kOrderThreads) {
    uint32_t key = 0xffffffffu;
    if (i < W) {
      int it = iters[i];
      it = it < 0 ? 0 : (it > 0x7fff ? 0x7fff : it);
      key = ((uint32_t)(0x7fff - it) << kIndexBits) | (uint32_t)i;
    }
    keys[i] = key;
  }
  __syncthreads();
  for (int k = 2; k <= N; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < N; i += kOrderThreads) {
        const int p = i ^ j;
        if (p > i) {
          const uint32_t a = keys[i], b = keys[p];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            keys[i] = b;
            keys[p] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < W; i += kOrderThreads) order[i] = (int32_t)(keys[i] & 0xffffu);
}

// The up component of each contact frame (R_WC[2][2]), the network's
// "normal" feature.
__global__ void frame_up_kernel(const double* frame, long long n, double* up) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    up[i] = frame[9 * i + 8];
}

template <typename T>
cudaError_t dev_alloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count);
}

}  // namespace
}  // namespace sapb

using namespace sapb;

struct sapb_handle {
  sapb_model_desc model;
  sapb_step_options opts;
  int32_t W, n, C, B, Q;
  // free motion + contact rows
  double *v_star, *vdot, *A, *J, *phi0, *w_eff, *mu, *stiffness, *tau_d;
  int32_t *count, *body0, *body1, *truncated;
  void* prep_ws;
  size_t prep_ws_bytes;
  // contact history (previous-impulse warm start): keys, carried impulses,
  // the impulses before them, the extrapolated start impulses
  int32_t *key_shape, *key_count, *has_history;
  double *key_point, *gamma_older, *gamma_start, *v_start;
  // solve
  double *v, *gamma, *gamma_prev, *cost, *grad_norm;
  int32_t *mode, *iters, *ls_iters, *converged, *status, *ws_accepted, *guess_flag, *order;
  int32_t *body_dof_start, *body_dof_count;
  void* solve_ws;
  size_t solve_ws_bytes;
  // tree-blocked layout (opts.prepare.tree_blocked): T trees (the
  // articulations) in blocks of NB DOFs, their first DOFs, A's tree blocks
  // and the tree of each contact side
  bool blk;
  int32_t T, NB;
  int32_t *tree_dof_start, *contact_tree;
  double* tree_mass;
  // uneven batches (model world offsets): the start velocities in the
  // solve's slots and each world's DOF count
  double* qd_slots;
  int32_t* dof_count;
  // learned start: the network, the contact frames and their up component,
  // the free-motion contact velocities, the factor of A (worlds with a new
  // contact), the features / outputs / active tiles, the network's impulses
  sapb_step_network net;
  double *frame, *normal_up, *vc_star, *factor, *gamma_cand, *gamma_zero;
  uint16_t* feat;
  float* mlp_y;
  int32_t* tiles;
};

extern "C" {

int32_t sapb_world_order(const int32_t* newton_iterations, int32_t num_envs, int32_t* order, void* stream) {
  if (num_envs < 0 || (num_envs > 0 && (!newton_iterations || !order))) {
    set_last_error("sapb_world_order: invalid argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (num_envs > kOrderMaxWorlds) {
    set_last_error("sapb_world_order: %d worlds above the supported %d", num_envs, kOrderMaxWorlds);
    return SAPB_ERR_UNSUPPORTED;
  }
  if (num_envs == 0) return SAPB_OK;
  int N = 1;
  while (N < num_envs) N <<= 1;
  const size_t smem = sizeof(uint32_t) * (size_t)N;
  cudaError_t err = cudaFuncSetAttribute(world_order_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (err == cudaSuccess) {
    world_order_kernel<<<1, kOrderThreads, smem, static_cast<cudaStream_t>(stream)>>>(newton_iterations, num_envs,
                                                                                       N, order);
    err = cudaGetLastError();
  }
  if (err != cudaSuccess) {
    set_last_error("sapb_world_order: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

void sapb_step_options_default(sapb_step_options* o) {
  if (!o) return;
  memset(o, 0, sizeof(*o));
  o->prepare.max_contacts = 128;
  o->prepare.contact_weight_mode = SAPB_WEIGHT_DIAG_DELASSUS;
  o->prepare.contact_point_mode = SAPB_POINT_MIDPOINT;
  o->prepare.fallback_mu = 0.1;
  o->prepare.fallback_stiffness = 1.0e10;
  o->prepare.fallback_tau_d = 0.0;
  o->prepare.tree_blocked = 0;
  sapb_solve_options_default(&o->solve, SAPB_LS_ARMIJO_DECAY);
  o->position_integration = SAPB_INTEGRATE_SAP_EULER;
  o->warm_start = SAPB_WARM_START_PREVIOUS_VELOCITY;
  o->work_order = SAPB_WORK_ORDER_PREVIOUS_ITERATIONS;
  o->impulse_history = 3;
}

void sapb_destroy(sapb_handle* h) {
  if (!h) return;
  void* ptrs[] = {h->v_star,    h->vdot,      h->A,     h->J,  h->phi0,     h->w_eff, h->mu,
                  h->stiffness, h->tau_d,     h->count, h->body0, h->body1, h->truncated, h->prep_ws,
                  h->v,         h->gamma,     h->gamma_prev, h->cost, h->grad_norm, h->mode, h->iters, h->ls_iters, h->converged, h->status,
                  h->ws_accepted, h->guess_flag, h->order, h->body_dof_start, h->body_dof_count, h->solve_ws,
                  h->key_shape, h->key_count, h->has_history, h->key_point,
                  h->gamma_older, h->gamma_start, h->v_start, h->tree_dof_start, h->contact_tree,
                  h->tree_mass, h->qd_slots, h->dof_count, h->frame, h->normal_up, h->vc_star,
                  h->factor, h->gamma_cand, h->gamma_zero, h->feat, h->mlp_y, h->tiles};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete h;
}

int32_t sapb_create(const sapb_model_desc* model, const sapb_step_options* opts, sapb_handle** out) {
  if (!model || !opts || !out) {
    set_last_error("sapb_create: null argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  const int32_t W = model->num_worlds, n = model->dofs_per_world, C = opts->prepare.max_contacts;
  const bool uneven = model->world_joint_start != nullptr;
  // totals (an uneven batch: from its offsets; dofs_per_world is the
  // largest world's, the solve's slot size)
  const int32_t B = model_bodies(*model), J = model_joints(*model), A = model_articulations(*model);
  int32_t Q = W * model->coords_per_world;
  if (W < 1 || n < 1 || C < 1 || model->bodies_per_world < 1 || J < 1 || A < 1 || !model->joint_child ||
      !model->joint_qd_start || !model->joint_dof_dim || !model->articulation_start) {
    set_last_error("sapb_create: invalid model description");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (uneven && (opts->prepare.tree_blocked || !model->world_body_start || !model->world_dof_start ||
                 !model->world_articulation_start || !model->body_world)) {
    set_last_error("sapb_create: an uneven batch needs all its world offsets and the dense layout");
    return SAPB_ERR_UNSUPPORTED;
  }
  if (opts->position_integration != SAPB_INTEGRATE_SAP_EULER && opts->position_integration != SAPB_INTEGRATE_MIDPOINT) {
    set_last_error("sapb_create: position_integration must be SAPB_INTEGRATE_SAP_EULER or _MIDPOINT");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (opts->warm_start != SAPB_WARM_START_PREVIOUS_VELOCITY && opts->warm_start != SAPB_WARM_START_PREVIOUS_IMPULSES &&
      opts->warm_start != SAPB_WARM_START_LEARNED) {
    set_last_error("sapb_create: warm_start must be SAPB_WARM_START_PREVIOUS_VELOCITY, _PREVIOUS_IMPULSES or _LEARNED");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (opts->warm_start == SAPB_WARM_START_LEARNED &&
      (!opts->network || !opts->network->packed || !opts->network->bias)) {
    set_last_error("sapb_create: the learned start needs opts->network with its device weights");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (opts->impulse_history < 0 || opts->impulse_history > 3) {
    set_last_error("sapb_create: impulse_history must be 0 (default), 1, 2 or 3");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (opts->work_order == SAPB_WORK_ORDER_PREVIOUS_ITERATIONS && W > kOrderMaxWorlds) {
    set_last_error("sapb_create: work_order by previous iterations supports at most %d worlds", kOrderMaxWorlds);
    return SAPB_ERR_UNSUPPORTED;
  }
  const bool blk = opts->prepare.tree_blocked != 0;
  const bool fp32 = opts->solve.hessian_precision == SAPB_FP32 || opts->solve.linear_solve_precision == SAPB_FP32;
  const size_t solve_smem =
      blk ? 0 : contact_solve_smem_bytes(n, C, fp32 ? SAPB_FP32 : SAPB_FP64, opts->solve.threads_per_cta);
  if (solve_smem > kMaxSmemPerBlock) {
    set_last_error("sapb_create: worlds of %d DOFs and %d contact slots exceed the on-chip solve", n, C);
    return SAPB_ERR_UNSUPPORTED;
  }
  // body -> world-local DOF range of its articulation (the reference's
  // _build_body_dof_maps, sim/contact_solve.py:3724-3758), from the model's
  // index arrays (copied to the host once)
  std::vector<int32_t> child(J), qd_start(J + 1), dim(2 * J), art(A + 1);
  cudaError_t err = cudaMemcpy(child.data(), model->joint_child, sizeof(int32_t) * J, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess)
    err = cudaMemcpy(qd_start.data(), model->joint_qd_start, sizeof(int32_t) * (J + 1), cudaMemcpyDeviceToHost);
  if (err == cudaSuccess)
    err = cudaMemcpy(dim.data(), model->joint_dof_dim, sizeof(int32_t) * 2 * J, cudaMemcpyDeviceToHost);
  if (err == cudaSuccess)
    err = cudaMemcpy(art.data(), model->articulation_start, sizeof(int32_t) * (A + 1), cudaMemcpyDeviceToHost);
  std::vector<int32_t> wbody(W + 1, 0), wdof(W + 1, 0);
  if (uneven) {
    if (err == cudaSuccess)
      err = cudaMemcpy(wbody.data(), model->world_body_start, sizeof(int32_t) * (W + 1), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
      err = cudaMemcpy(wdof.data(), model->world_dof_start, sizeof(int32_t) * (W + 1), cudaMemcpyDeviceToHost);
    if (err == cudaSuccess && model->joint_q_start)
      err = cudaMemcpy(&Q, model->joint_q_start + J, sizeof(int32_t), cudaMemcpyDeviceToHost);
  }
  if (err != cudaSuccess) {
    set_last_error("sapb_create: reading the model: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  // the world of a body and its first DOF
  auto world_of = [&](int b) {
    if (!uneven) return b / model->bodies_per_world;
    int e = 0;
    while (e + 1 < W && wbody[e + 1] <= b) ++e;
    return e;
  };
  auto dof0_of = [&](int e) { return uneven ? wdof[e] : e * n; };
  std::vector<int32_t> bstart(B, -1), bcount(B, 0);
  for (int a = 0; a < A; ++a) {
    int s0 = -1, tot = 0;
    for (int j = art[a]; j < art[a + 1] && j < J; ++j) {
      const int cnt = dim[2 * j] + dim[2 * j + 1];
      if (cnt > 0 && (s0 < 0 || qd_start[j] < s0)) s0 = qd_start[j];
      tot += cnt;
    }
    if (s0 < 0 || tot <= 0) continue;
    for (int j = art[a]; j < art[a + 1] && j < J; ++j) {
      const int b = child[j];
      if (b >= 0 && b < B) {
        bstart[b] = s0 - dof0_of(world_of(b));
        bcount[b] = tot;
      }
    }
  }
  // tree-blocked layout: the trees are world 0's articulations (every world
  // alike), each a contiguous DOF range within the block size
  const int32_t Aw = model->articulations_per_world;
  std::vector<int32_t> tds;
  int32_t NB = 0;
  if (blk) {
    tds.resize(Aw + 1);
    int largest = 0;
    bool ok = model->bodies_per_world <= 64 && Aw >= 1 && Aw <= 64;
    for (int t = 0; ok && t <= Aw; ++t) {
      tds[t] = t < Aw ? qd_start[art[t]] : n;
      if (t > 0) {
        ok = tds[t] >= tds[t - 1];
        largest = tds[t] - tds[t - 1] > largest ? tds[t] - tds[t - 1] : largest;
      }
    }
    ok = ok && tds[0] == 0;
    NB = opts->prepare.tree_dofs > 0 ? opts->prepare.tree_dofs : blocked_tree_block(largest);
    if (!ok || NB < 1 || blocked_tree_block(NB) != NB || largest > NB ||
        (Aw > 1 && blocked_fill_capacity(Aw, NB, C, fp32) < 1)) {
      set_last_error("sapb_create: the tree-blocked layout needs <= 64 bodies and articulations per world, each "
                     "articulation in one block of 6, 7 or 12 DOFs (largest %d, tree_dofs %d), and the worlds' "
                     "factor on chip", largest, opts->prepare.tree_dofs);
      return SAPB_ERR_UNSUPPORTED;
    }
  }
  sapb_handle* h = new sapb_handle;
  memset(h, 0, sizeof(*h));
  h->model = *model;
  h->opts = *opts;
  h->blk = blk;
  h->T = blk ? Aw : 0;
  h->NB = NB;
  if (blk) h->opts.prepare.tree_dofs = NB;
  if (h->opts.impulse_history == 0) h->opts.impulse_history = 3;
  h->W = W;
  h->n = n;
  h->C = C;
  h->B = B;
  h->Q = Q;
  const size_t Wn = (size_t)W * n, WC = (size_t)W * C;
  // the contact history runs for both candidate starts
  const bool cand = opts->warm_start != SAPB_WARM_START_PREVIOUS_VELOCITY;
  const bool learned = opts->warm_start == SAPB_WARM_START_LEARNED;
  if (learned) h->net = *opts->network;
  h->opts.network = nullptr;  // the handle keeps its own copy
  err = cudaSuccess;
  auto take = [&](cudaError_t e) {
    if (err == cudaSuccess) err = e;
  };
  take(dev_alloc(&h->v_star, Wn));
  take(dev_alloc(&h->vdot, Wn));
  if (blk) {
    take(dev_alloc(&h->tree_mass, (size_t)W * h->T * NB * NB));
    take(dev_alloc(&h->contact_tree, WC * 2));
    take(dev_alloc(&h->tree_dof_start, (size_t)h->T + 1));
    take(dev_alloc(&h->J, WC * 3 * 2 * NB));
  } else {
    take(dev_alloc(&h->A, Wn * n));
    take(dev_alloc(&h->J, WC * 3 * n));
  }
  take(dev_alloc(&h->phi0, WC));
  take(dev_alloc(&h->w_eff, WC));
  take(dev_alloc(&h->mu, WC));
  take(dev_alloc(&h->stiffness, WC));
  take(dev_alloc(&h->tau_d, WC));
  take(dev_alloc(&h->count, W));
  take(dev_alloc(&h->body0, WC));
  take(dev_alloc(&h->body1, WC));
  take(dev_alloc(&h->truncated, 1));
  if (cand) {
    if (!blk) take(dev_alloc(&h->v_start, Wn));  // the tree-blocked solve forms its candidate itself
    take(dev_alloc(&h->gamma_prev, WC * 3));
    take(dev_alloc(&h->key_shape, WC * 2));
    take(dev_alloc(&h->key_point, WC * 3));
    take(dev_alloc(&h->key_count, W));
    take(dev_alloc(&h->has_history, WC));
    take(dev_alloc(&h->gamma_older, WC * 3));
    take(dev_alloc(&h->gamma_start, WC * 3));
  }
  const size_t tiles = (WC + 127) / 128;
  if (learned) {
    take(dev_alloc(&h->frame, WC * 9));
    take(dev_alloc(&h->normal_up, WC));
    take(dev_alloc(&h->vc_star, WC * 3));
    if (!blk) take(dev_alloc(&h->factor, Wn * n));
    take(dev_alloc(&h->gamma_cand, WC * 3));
    take(dev_alloc(&h->gamma_zero, WC * 3));
    take(dev_alloc(&h->feat, WC * SAPB_MLP_INPUTS_PADDED));
    take(dev_alloc(&h->mlp_y, WC * SAPB_MLP_OUTPUTS));
    take(dev_alloc(&h->tiles, tiles));
  }
  take(dev_alloc(&h->v, Wn));
  take(dev_alloc(&h->gamma, WC * 3));
  take(dev_alloc(&h->cost, W));
  take(dev_alloc(&h->grad_norm, W));
  take(dev_alloc(&h->mode, WC));
  take(dev_alloc(&h->iters, W));
  take(dev_alloc(&h->ls_iters, W));
  take(dev_alloc(&h->converged, W));
  take(dev_alloc(&h->status, W));
  take(dev_alloc(&h->ws_accepted, W));
  take(dev_alloc(&h->guess_flag, 1));
  take(dev_alloc(&h->order, W));
  take(dev_alloc(&h->body_dof_start, B));
  take(dev_alloc(&h->body_dof_count, B));
  if (uneven) {
    take(dev_alloc(&h->qd_slots, Wn));
    take(dev_alloc(&h->dof_count, W));
  }
  h->prep_ws_bytes = sapb_prepare_workspace_size(model, C);
  h->solve_ws_bytes = blk ? sapb_blocked_solve_workspace_size(W, h->T, C) : sapb_contact_solve_workspace_size(W, n, C);
  if (err == cudaSuccess) err = cudaMalloc(&h->prep_ws, h->prep_ws_bytes > 0 ? h->prep_ws_bytes : 16);
  if (err == cudaSuccess) err = cudaMalloc(&h->solve_ws, h->solve_ws_bytes > 0 ? h->solve_ws_bytes : 16);
  if (err == cudaSuccess)
    err = cudaMemcpy(h->body_dof_start, bstart.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice);
  if (err == cudaSuccess)
    err = cudaMemcpy(h->body_dof_count, bcount.data(), sizeof(int32_t) * B, cudaMemcpyHostToDevice);
  if (err == cudaSuccess && blk)
    err = cudaMemcpy(h->tree_dof_start, tds.data(), sizeof(int32_t) * (h->T + 1), cudaMemcpyHostToDevice);
  if (err == cudaSuccess && uneven) {
    std::vector<int32_t> cnt(W);
    for (int e = 0; e < W; ++e) cnt[e] = wdof[e + 1] - wdof[e];
    err = cudaMemcpy(h->dof_count, cnt.data(), sizeof(int32_t) * W, cudaMemcpyHostToDevice);
  }
  if (err == cudaSuccess) err = cudaMemset(h->guess_flag, 0, sizeof(int32_t));
  if (err == cudaSuccess && cand) err = cudaMemset(h->gamma_prev, 0, sizeof(double) * WC * 3);
  if (err == cudaSuccess && cand) err = cudaMemset(h->key_count, 0, sizeof(int32_t) * W);
  if (err == cudaSuccess && cand) err = cudaMemset(h->has_history, 0, sizeof(int32_t) * WC);
  if (err == cudaSuccess && cand) err = cudaMemset(h->gamma_older, 0, sizeof(double) * WC * 3);
  if (err == cudaSuccess && cand) err = cudaMemset(h->gamma_start, 0, sizeof(double) * WC * 3);
  if (err == cudaSuccess) err = cudaMemset(h->iters, 0, sizeof(int32_t) * W);
  if (learned) {  // every learned buffer starts at zero (dead slots keep what they hold)
    if (err == cudaSuccess) err = cudaMemset(h->frame, 0, sizeof(double) * WC * 9);
    if (err == cudaSuccess) err = cudaMemset(h->normal_up, 0, sizeof(double) * WC);
    if (err == cudaSuccess) err = cudaMemset(h->vc_star, 0, sizeof(double) * WC * 3);
    if (err == cudaSuccess && h->factor) err = cudaMemset(h->factor, 0, sizeof(double) * Wn * n);
    if (err == cudaSuccess) err = cudaMemset(h->gamma_cand, 0, sizeof(double) * WC * 3);
    if (err == cudaSuccess) err = cudaMemset(h->gamma_zero, 0, sizeof(double) * WC * 3);
    if (err == cudaSuccess) err = cudaMemset(h->feat, 0, sizeof(uint16_t) * WC * SAPB_MLP_INPUTS_PADDED);
    if (err == cudaSuccess) err = cudaMemset(h->mlp_y, 0, sizeof(float) * WC * SAPB_MLP_OUTPUTS);
    if (err == cudaSuccess) err = cudaMemset(h->tiles, 0, sizeof(int32_t) * tiles);
  }
  if (err == cudaSuccess) {
    std::vector<int32_t> idx(W);
    for (int i = 0; i < W; ++i) idx[i] = i;
    err = cudaMemcpy(h->order, idx.data(), sizeof(int32_t) * W, cudaMemcpyHostToDevice);
  }
  if (err != cudaSuccess) {
    set_last_error("sapb_create: %s", cudaGetErrorString(err));
    sapb_destroy(h);
    return SAPB_ERR_CUDA;
  }
  *out = h;
  return SAPB_OK;
}

int32_t sapb_step(sapb_handle* h, const sapb_step_io* io, void* stream) {
  if (!h || !io || !io->in.joint_q || !io->in.joint_qd || !io->in.dt || !io->joint_q_out || !io->joint_qd_out) {
    set_last_error("sapb_step: null argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  if (io->joint_q_out == io->in.joint_q) {
    set_last_error("sapb_step: joint_q_out must not alias the input coordinates");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool cand = h->opts.warm_start != SAPB_WARM_START_PREVIOUS_VELOCITY;  // the contact history runs
  const bool learned = h->opts.warm_start == SAPB_WARM_START_LEARNED;
  const bool order = h->opts.work_order == SAPB_WORK_ORDER_PREVIOUS_ITERATIONS;
  // free motion and contact rows (sim/solver_sap.py:1415-1433)
  sapb_prepare_outputs po;
  memset(&po, 0, sizeof(po));
  po.v_star = h->v_star;
  po.vdot = h->vdot;
  po.dynamics_matrix = h->A;  // NULL in the tree-blocked layout
  po.tree_mass = h->tree_mass;
  po.contact_tree = h->contact_tree;
  po.jacobian = h->J;
  po.contact_count = h->count;
  po.phi0 = h->phi0;
  po.w_eff = h->w_eff;
  po.mu = h->mu;
  po.stiffness = h->stiffness;
  po.tau_d = h->tau_d;
  po.body0 = h->body0;
  po.body1 = h->body1;
  po.truncated_count = h->truncated;
  if (learned) {  // the network's inputs and, for its impulses, the factor of A where a contact is new
    po.frame = h->frame;
    po.vc_star = h->vc_star;
    po.dynamics_factor = h->factor;  // NULL in the tree-blocked layout
  }
  po.qd_slots = h->qd_slots;  // uneven batches: the start velocities in the solve's slots
  // previous impulses: the contact history runs inside the launch (the last
  // solves' impulses carried to this step's slots by contact identity and
  // extrapolated), and the free motion forms the start v* + A^-1 J^T gamma
  sapb_contact_history hist;
  memset(&hist, 0, sizeof(hist));
  if (cand) {
    hist.key_shape = h->key_shape;
    hist.key_point = h->key_point;
    hist.key_count = h->key_count;
    hist.gamma_prev = h->gamma;
    hist.gamma_hist = h->gamma_prev;
    hist.has_history = h->has_history;
    hist.order = h->opts.impulse_history;
    hist.gamma_older = h->gamma_older;
    hist.gamma_start = h->gamma_start;
    po.history = &hist;
    po.v_start = h->v_start;  // NULL in the tree-blocked layout
  }
  int32_t st = sapb_free_motion_contacts(&h->model, &io->in, &h->opts.prepare, &po, h->prep_ws, h->prep_ws_bytes,
                                         stream);
  if (st != SAPB_OK) return st;
  if (learned) {
    // the network's impulses (LearnedWarmStart.predict): features, the tiles
    // holding a new contact, the forward over them, the impulse map; the
    // history's impulses where a contact has them (tree-blocked: one set with
    // the history's start impulses; dense: zero there, the start velocity
    // already holding them)
    const long long slots = (long long)h->W * h->C;
    frame_up_kernel<<<(int)((slots + 255) / 256 < 4096 ? (slots + 255) / 256 : 4096), 256, 0, s>>>(h->frame, slots,
                                                                                                 h->normal_up);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_last_error("sapb_step: %s", cudaGetErrorString(e));
      return SAPB_ERR_CUDA;
    }
    sapb_contact_problem q;
    memset(&q, 0, sizeof(q));
    q.num_envs = h->W;
    q.dof_per_env = h->blk ? 2 * h->NB : h->n;
    q.max_contacts = h->C;
    q.contact_count = h->count;
    q.dynamics_matrix = h->A;
    q.jacobian = h->J;
    q.phi0 = h->phi0;
    q.w_eff = h->w_eff;
    q.mu = h->mu;
    q.stiffness = h->stiffness;
    q.tau_d = h->tau_d;
    q.v_star = h->v_star;
    q.v0 = h->v_star;
    q.dt = io->in.dt;
    const double* gprev = h->blk ? h->gamma_start : h->gamma_zero;
    st = sapb_warmstart_features(&q, h->normal_up, gprev, h->vc_star, &h->net.norm, h->net.feature_tau_d, h->feat,
                                 nullptr, stream);
    if (st == SAPB_OK) st = sapb_warmstart_active_tiles(&q, h->has_history, h->tiles, stream);
    if (st == SAPB_OK)
      st = sapb_mlp_forward_tiles(h->net.packed, h->net.bias, h->feat, (int32_t)slots, h->mlp_y, h->tiles, stream);
    if (st == SAPB_OK) {
      sapb_solve_options io_opts = h->opts.solve;
      io_opts.contact_tau_d = h->net.impulse_tau_d;
      st = sapb_warmstart_impulses(&q, h->mlp_y, gprev, h->has_history, &h->net.norm, &io_opts, h->gamma_cand,
                                   stream);
    }
    if (st != SAPB_OK) return st;
  }
  sapb_solve_outputs so;
  memset(&so, 0, sizeof(so));
  so.v = h->v;
  so.contact_gamma = h->gamma;
  so.contact_mode = h->mode;
  so.cost = h->cost;
  so.newton_iterations = h->iters;
  so.line_search_iterations = h->ls_iters;
  so.converged = h->converged;
  so.status = h->status;
  so.grad_norm = h->grad_norm;
  so.warm_start_accepted = h->ws_accepted;
  if (h->blk) {
    // the tree-blocked solve: the same Newton loop on A's tree blocks, the
    // history's start impulses as its candidate
    sapb_blocked_problem bp;
    memset(&bp, 0, sizeof(bp));
    bp.num_envs = h->W;
    bp.trees_per_env = h->T;
    bp.tree_dofs = h->NB;
    bp.max_contacts = h->C;
    bp.contact_count = h->count;
    bp.tree_mass = h->tree_mass;
    bp.jacobian = h->J;
    bp.contact_tree = h->contact_tree;
    bp.phi0 = h->phi0;
    bp.w_eff = h->w_eff;
    bp.mu = h->mu;
    bp.stiffness = h->stiffness;
    bp.tau_d = h->tau_d;
    bp.v_star = h->v_star;
    bp.v0 = io->in.joint_qd;
    bp.v_guess = h->v;
    bp.v_guess_active = h->guess_flag;
    bp.dt = io->in.dt;
    bp.world_order = order ? h->order : nullptr;
    bp.gamma0 = learned ? h->gamma_cand : (cand ? h->gamma_start : nullptr);
    bp.gamma0_count = cand ? 1 : 0;
    bp.tree_dof_start = h->tree_dof_start;
    bp.dofs_per_world = h->n;
    // the drive / limit terms at this step's coordinates
    sapb_dof_terms bdof;
    if (io->dof) {
      bdof = *io->dof;
      bdof.joint_q = io->in.joint_q;
      bdof.joint_coord_count = h->Q;
      bdof.world_dof_start = nullptr;
      bp.dof = &bdof;
    }
    st = sapb_blocked_contact_solve(&bp, &h->opts.solve, &so, h->solve_ws, h->solve_ws_bytes, stream);
  } else {
  // contact solve (sim/solver_sap.py:1434-1460), warm start from the last
  // solution once a step has run
  sapb_contact_problem p;
  memset(&p, 0, sizeof(p));
  p.num_envs = h->W;
  p.dof_per_env = h->n;
  p.max_contacts = h->C;
  p.num_bodies = h->B;
  p.contact_count = h->count;
  p.dynamics_matrix = h->A;
  p.jacobian = h->J;
  p.phi0 = h->phi0;
  p.w_eff = h->w_eff;
  p.mu = h->mu;
  p.stiffness = h->stiffness;
  p.tau_d = h->tau_d;
  p.body0 = h->body0;
  p.body1 = h->body1;
  p.body_dof_start = h->body_dof_start;
  p.body_dof_count = h->body_dof_count;
  p.v_star = h->v_star;
  p.v0 = h->qd_slots ? h->qd_slots : io->in.joint_qd;
  p.dof_count = h->dof_count;
  p.v_guess = h->v;
  p.v_guess_active = h->guess_flag;
  p.dt = io->in.dt;
  // the drive / limit terms act at this step's coordinates (the solve copies
  // the struct into its launch parameters)
  sapb_dof_terms dof_local;
  if (io->dof) {
    dof_local = *io->dof;
    dof_local.joint_q = io->in.joint_q;
    dof_local.joint_coord_count = h->Q;
    dof_local.world_dof_start = h->model.world_dof_start;  // uneven: the per-DOF arrays in global order
    p.dof = &dof_local;
  }
  if (learned) {
    // the network's impulses on new contacts through the factor of A, over
    // the history's start velocity
    p.gamma0 = h->gamma_cand;
    p.gamma0_count = 1;
    p.gamma0_base = h->v_start;
    p.dynamics_factor = h->factor;
  } else if (cand) {
    p.v_candidates = h->v_start;
    p.v_candidate_count = 1;
  }
  p.world_order = order ? h->order : nullptr;
  st = sapb_contact_solve(&p, &h->opts.solve, &so, h->solve_ws, h->solve_ws_bytes, stream);
  }
  if (st != SAPB_OK) return st;
  if (order) {
    st = sapb_world_order(h->iters, h->W, h->order, stream);
    if (st != SAPB_OK) return st;
  }
  // the tail in one launch: position integration (sim/solver_sap.py:1267-1386;
  // fixed joints keep their coordinates) and the new SAP-order velocities
  sapb_step_tail tail;
  memset(&tail, 0, sizeof(tail));
  tail.joint_q_in = io->in.joint_q;
  tail.v_prev = io->in.joint_qd;
  tail.v_new = h->v;
  tail.dt = io->in.dt;
  tail.mode = h->opts.position_integration;
  tail.joint_q_out = io->joint_q_out;
  tail.joint_qd_out = io->joint_qd_out;
  st = sapb_step_tail_launch(&h->model, &tail, stream);
  if (st != SAPB_OK) return st;
  // nonzero: warm start from this solution; the next step's history reads
  // this solve's impulses (h->gamma) before its own solve rewrites them
  const cudaError_t err = cudaMemsetAsync(h->guess_flag, 1, sizeof(int32_t), s);
  if (err != cudaSuccess) {
    set_last_error("sapb_step: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

int32_t sapb_get_status(const sapb_handle* h, int32_t* status, int32_t* converged, int32_t* newton_iterations,
                        void* stream) {
  if (!h) {
    set_last_error("sapb_get_status: null handle");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t bytes = sizeof(int32_t) * (size_t)h->W;
  cudaError_t err = cudaSuccess;
  if (status) err = cudaMemcpyAsync(status, h->status, bytes, cudaMemcpyDefault, s);
  if (err == cudaSuccess && converged) err = cudaMemcpyAsync(converged, h->converged, bytes, cudaMemcpyDefault, s);
  if (err == cudaSuccess && newton_iterations)
    err = cudaMemcpyAsync(newton_iterations, h->iters, bytes, cudaMemcpyDefault, s);
  if (err != cudaSuccess) {
    set_last_error("sapb_get_status: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

int32_t sapb_step_solve_outputs(const sapb_handle* h, sapb_solve_outputs* out) {
  if (!h || !out) {
    set_last_error("sapb_step_solve_outputs: null argument");
    return SAPB_ERR_INVALID_ARGUMENT;
  }
  memset(out, 0, sizeof(*out));
  out->v = h->v;
  out->contact_gamma = h->gamma;
  out->contact_mode = h->mode;
  out->cost = h->cost;
  out->newton_iterations = h->iters;
  out->line_search_iterations = h->ls_iters;
  out->converged = h->converged;
  out->status = h->status;
  out->grad_norm = h->grad_norm;
  out->warm_start_accepted = h->ws_accepted;
  return SAPB_OK;
}

}  // extern "C"
