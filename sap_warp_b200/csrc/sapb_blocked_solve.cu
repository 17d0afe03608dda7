// sapb_blocked_solve.cu -- host side of the tree-blocked solve (block
// sizes, on-chip capacity, launch; kernels in sapb_blocked_solve.cuh,
// instantiated in sapb_blocked_nb*.cu) and the dense -> blocked gather.
#include "sapb_blocked_solve.cuh"

namespace sapb {

int32_t blocked_tree_block(int tree_dofs) {
  if (tree_dofs < 0) return 0;
  if (tree_dofs <= 6) return 6;
  if (tree_dofs <= 7) return 7;
  if (tree_dofs <= 12) return 12;
  return 0;
}

int32_t blocked_fill_capacity(int T, int NB, int C, bool fp32) {
  if (NB < 1 || blocked_tree_block(NB) != NB || T < 1 || T > kBMaxTrees || C < 0) return 0;
  return fp32 ? blocked_capacity<float>(T, NB, C) : blocked_capacity<double>(T, NB, C);
}

int32_t blocked_solve_launch(const sapb_blocked_problem* p, const sapb_solve_options* o,
                             const sapb_solve_outputs* out, void* workspace, cudaStream_t stream) {
  BlockedParams P;
  memset(&P, 0, sizeof(P));
  P.p = *p;
  P.o = *o;
  P.out = *out;
  P.use_guess_flag_ptr_valid = (p->v_guess && p->v_guess_active) ? 1 : 0;
  P.queue = reinterpret_cast<int32_t*>(workspace);
  P.nd = p->dofs_per_world > 0 ? p->dofs_per_world : p->trees_per_env * p->tree_dofs;
  if (p->dof) P.dof = *p->dof;
  if (p->num_envs == 0) return SAPB_OK;
  const bool fp32 = o->hessian_precision == SAPB_FP32 || o->linear_solve_precision == SAPB_FP32;
  const bool terms = P.dof.has_pd || P.dof.has_limits;
  // the on-chip factor capacity, less the drive / limit vectors' room
  P.capacity = blocked_fill_capacity(p->trees_per_env, p->tree_dofs, p->max_contacts, fp32);
  if (terms && P.capacity > 0)
    P.capacity = fp32 ? blocked_capacity<float>(p->trees_per_env, p->tree_dofs, p->max_contacts, true)
                      : blocked_capacity<double>(p->trees_per_env, p->tree_dofs, p->max_contacts, true);
  if (P.capacity < 1 && p->trees_per_env > 1) {
    set_last_error("blocked contact solve: a world of %d trees and %d contact slots does not fit on chip",
                   p->trees_per_env, p->max_contacts);
    return SAPB_ERR_UNSUPPORTED;
  }
  // threads per world: as asked, else 128 for worlds of up to 128 padded
  // DOFs (a few small trees: more worlds in flight between block barriers)
  // and 256 beyond
  int threads = o->threads_per_cta;
  if (threads != 128 && threads != 256) threads = p->trees_per_env * p->tree_dofs <= 128 ? 128 : 256;
  cudaError_t err;
  switch (p->tree_dofs) {
    case 6:
      err = launch_blocked<6>(P, fp32, threads, stream);
      break;
    case 7:
      err = launch_blocked<7>(P, fp32, threads, stream);
      break;
    default:
      err = launch_blocked<12>(P, fp32, threads, stream);
      break;
  }
  if (err != cudaSuccess) {
    set_last_error("blocked contact solve launch: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

// ---- dense -> blocked gather -------------------------------------------------

// The tree holding world DOF s (-1: none): tree t holds tds[t] .. tds[t+1]-1,
// or t * NB .. with tds NULL.
__device__ inline int tree_of_dof(const int32_t* tds, int T, int NB, int s) {
  if (s < 0) return -1;
  if (!tds) return s / NB < T ? s / NB : -1;
  for (int t = 0; t < T; ++t)
    if (s >= tds[t] && s < tds[t + 1]) return t;
  return -1;
}

__global__ void dense_to_blocked_kernel(sapb_contact_problem d, int T, int NB, const int32_t* tds,
                                        double* tree_mass, double* jac, int32_t* contact_tree) {
  const int n = d.dof_per_env, C = d.max_contacts;
  const size_t E = (size_t)d.num_envs;
  const size_t nA = E * T * NB * NB, nJ = E * C * 3 * 2 * NB, nT = E * C;
  const size_t total = nA + nJ + nT;
  auto tstart = [&](int t) { return tds ? tds[t] : t * NB; };
  auto tcount = [&](int t) {  // clamped to NB and to the world's DOFs
    const int s0 = tstart(t);
    int c = tds ? tds[t + 1] - s0 : NB;
    if (c > NB) c = NB;
    if (s0 < 0 || c < 0) return 0;
    return s0 + c > n ? (n > s0 ? n - s0 : 0) : c;
  };
  auto body_tree = [&](const int* bodies, size_t ec) {
    if (!bodies || bodies[ec] < 0 || bodies[ec] >= d.num_bodies) return -1;
    return tree_of_dof(tds, T, NB, d.body_dof_start[bodies[ec]]);
  };
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < total; k += (size_t)gridDim.x * blockDim.x) {
    if (k < nA) {
      const size_t e = k / ((size_t)T * NB * NB);
      const int r = (int)(k - e * T * NB * NB);
      const int t = r / (NB * NB), a = (r / NB) % NB, b = r % NB;
      const int s0 = tstart(t), nt = tcount(t);
      // a tree's own block, the identity in its padding
      tree_mass[k] = (a < nt && b < nt) ? d.dynamics_matrix[(e * n + s0 + a) * n + s0 + b] : (a == b ? 1.0 : 0.0);
    } else if (k < nA + nJ) {
      const size_t q = k - nA;
      const size_t row = q / (2 * NB);  // (e, c, r)
      const int col = (int)(q - row * 2 * NB);
      const size_t ec = row / 3;
      const int side = col / NB, a = col % NB;
      const int tt = body_tree(side == 0 ? d.body0 : d.body1, ec);
      const int to = body_tree(side == 0 ? d.body1 : d.body0, ec);
      double v = 0.0;
      // a contact whose two sides lie on one tree keeps its (summed) columns on side 0
      if (tt >= 0 && a < tcount(tt) && !(side == 1 && tt == to)) v = d.jacobian[row * n + tstart(tt) + a];
      jac[q] = v;
    } else {
      const size_t ec = k - nA - nJ;
      const int t0 = body_tree(d.body0, ec);
      int t1 = body_tree(d.body1, ec);
      if (t1 == t0) t1 = -1;
      contact_tree[2 * ec] = t0;
      contact_tree[2 * ec + 1] = t1;
    }
  }
}

int32_t dense_to_blocked_launch(const sapb_contact_problem* d, int T, int NB, const int32_t* tree_dof_start,
                                double* tree_mass, double* jac, int32_t* contact_tree, cudaStream_t stream) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  dense_to_blocked_kernel<<<sms * 4, 256, 0, stream>>>(*d, T, NB, tree_dof_start, tree_mass, jac, contact_tree);
  const cudaError_t err = cudaGetLastError();
  if (err != cudaSuccess) {
    set_last_error("dense to blocked gather: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return SAPB_OK;
}

}  // namespace sapb

