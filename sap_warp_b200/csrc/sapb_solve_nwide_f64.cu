// Contact-solve kernels sized at run time with 256 threads per world (eight warps); FP64 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_wide<false>(const SolveParams&, cudaStream_t, int*);
}  // namespace sapb
