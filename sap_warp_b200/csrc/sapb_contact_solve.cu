// sapb_contact_solve.cu -- host side of the fused contact solve: shared-
// memory size, occupancy query and the dispatch to the DOF specialisations
// (kernels in sapb_contact_solve.cuh, instantiated in sapb_solve_n*.cu).
#include "sapb_contact_solve.cuh"

namespace sapb {

size_t contact_solve_smem_bytes(int n, int C, int hessian_precision, int threads) {
  return make_layout(n, C, hessian_precision == SAPB_FP32 ? 4 : 8, (threads > 0 ? threads : 128) / 32).total;
}

// Resident CTAs per SM of the kernel a problem of this shape launches: the
// same dispatch with num_envs = 0, which stops at the occupancy query.
static cudaError_t solve_dispatch(const SolveParams& P, bool fp32, cudaStream_t stream, int* blocks_out);

int32_t contact_solve_occupancy(int n, int C, int hessian_precision, int variant, int threads) {
  if (n < 1 || C < 0) return SAPB_ERR_INVALID_ARGUMENT;
  const bool fp32 = hessian_precision == SAPB_FP32;
  if (contact_solve_smem_bytes(n, C, fp32 ? SAPB_FP32 : SAPB_FP64, threads) > kMaxSmemPerBlock)
    return SAPB_ERR_UNSUPPORTED;
  SolveParams P;
  memset(&P, 0, sizeof(P));
  P.p.dof_per_env = n;
  P.p.max_contacts = C;
  P.o.line_search_variant = variant;
  P.o.threads_per_cta = threads;
  int per_sm = 0;
  const cudaError_t err = solve_dispatch(P, fp32, nullptr, &per_sm);
  if (err != cudaSuccess) {
    set_last_error("contact solve occupancy: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  return per_sm;
}

template <int NS>
static int widths_of(int32_t* out, int capacity) {
  int k = 0;
  for (; k < LdltBlocks<NS>::kCount && k < capacity; ++k) out[k] = LdltBlocks<NS>::kW[k];
  return LdltBlocks<NS>::kCount;
}

int ldlt_block_widths(int n, int32_t* out, int capacity) {
  switch (n) {
    case 35: return widths_of<35>(out, capacity);
    case 18: return widths_of<18>(out, capacity);
    case 13: return widths_of<13>(out, capacity);
    case 6: return widths_of<6>(out, capacity);
    default: return widths_of<0>(out, capacity);
  }
}

static cudaError_t solve_dispatch(const SolveParams& P, bool fp32, cudaStream_t stream, int* blocks_out) {
  // Kernels specialised on the DOF count of the common trees (humanoid 35,
  // quadruped 18, arm + box 13, single free body 6); a generic one otherwise
  // and for per-world DOF counts; the generic one with eight warps per world
  // on request.
  if (P.o.threads_per_cta == 256)
    return fp32 ? launch_solve_wide<true>(P, stream, blocks_out) : launch_solve_wide<false>(P, stream, blocks_out);
  if (P.p.dof_count) return launch_solve_ns<0>(P, fp32, stream, blocks_out);
  switch (P.p.dof_per_env) {
#define SAPB_DISPATCH_N(NV) \
  case NV:                  \
    return launch_solve_ns<NV>(P, fp32, stream, blocks_out);
    SAPB_DISPATCH_N(35)
    SAPB_DISPATCH_N(18)
    SAPB_DISPATCH_N(13)
    SAPB_DISPATCH_N(6)
#undef SAPB_DISPATCH_N
    default:
      return launch_solve_ns<0>(P, fp32, stream, blocks_out);
  }
}

int32_t contact_solve_launch(const sapb_contact_problem* p, const sapb_solve_options* o, const sapb_solve_outputs* out,
                             void* workspace, size_t workspace_bytes, cudaStream_t stream) {
  SolveParams P;
  memset(&P, 0, sizeof(P));
  P.p = *p;
  if (p->dof) P.dof = *p->dof;
  P.o = *o;
  P.out = *out;
  P.use_guess_flag_ptr_valid = (p->v_guess && p->v_guess_active) ? 1 : 0;
  P.queue = reinterpret_cast<int32_t*>(workspace);
  if (p->num_envs == 0) return SAPB_OK;
  // If either the Hessian or the linear-solve precision is FP32, both the
  // J^T G J assembly and the LDL^T factorization run in FP32; the gradient,
  // costs, line search and convergence test stay FP64 in every variant.
  const bool fp32 = o->hessian_precision == SAPB_FP32 || o->linear_solve_precision == SAPB_FP32;
  const size_t smem =
      contact_solve_smem_bytes(p->dof_per_env, p->max_contacts, fp32 ? SAPB_FP32 : SAPB_FP64, o->threads_per_cta);
  if (smem > kMaxSmemPerBlock) {
    set_last_error("contact solve: world too large for the on-chip path (shared memory %zu > %zu bytes)", smem,
                   (size_t)kMaxSmemPerBlock);
    return SAPB_ERR_UNSUPPORTED;
  }
  const cudaError_t err = solve_dispatch(P, fp32, stream, nullptr);
  if (err != cudaSuccess) {
    set_last_error("contact solve launch: %s", cudaGetErrorString(err));
    return SAPB_ERR_CUDA;
  }
  (void)workspace_bytes;
  return SAPB_OK;
}

}  // namespace sapb

