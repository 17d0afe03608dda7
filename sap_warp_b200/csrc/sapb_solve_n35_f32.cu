// Contact-solve kernels specialised on 35 DOFs per world; FP32 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_np<35, true>(const SolveParams&, cudaStream_t, int*);
}  // namespace sapb
