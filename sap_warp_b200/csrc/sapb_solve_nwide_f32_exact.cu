// The runtime-size contact-solve kernel with 256 threads per world, exact_root line search; FP32 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_ls<256, float, 2, 0, SAPB_LS_EXACT_ROOT, LdltBlocks<0>::kW[0]>(const SolveParams&, cudaStream_t,
                                                                                      int*);
}  // namespace sapb
