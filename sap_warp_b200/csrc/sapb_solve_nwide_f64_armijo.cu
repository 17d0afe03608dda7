// The runtime-size contact-solve kernel with 256 threads per world, armijo_decay line search; FP64 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_ls<256, double, 1, 0, SAPB_LS_ARMIJO_DECAY, LdltBlocks<0>::kW[0]>(const SolveParams&, cudaStream_t,
                                                                                      int*);
}  // namespace sapb
