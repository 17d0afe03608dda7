// Contact-solve kernels specialised on 6 DOFs per world; FP64 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_np<6, false>(const SolveParams&, cudaStream_t, int*);
}  // namespace sapb
