// The runtime-size contact-solve kernel with 128 threads per world, monotone_decay line search; FP32 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_ls<128, float, 4, 0, SAPB_LS_MONOTONE_DECAY, LdltBlocks<0>::kW[0]>(const SolveParams&, cudaStream_t,
                                                                                      int*);
}  // namespace sapb
