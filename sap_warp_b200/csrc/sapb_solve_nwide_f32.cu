// Contact-solve kernels sized at run time with 256 threads per world (eight warps); FP32 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_wide<true>(const SolveParams&, cudaStream_t, int*);
}  // namespace sapb
