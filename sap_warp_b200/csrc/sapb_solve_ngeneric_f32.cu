// Contact-solve kernels sized at run time (n <= 60; with per-world DOF counts each world runs the code of its size class); FP32 Hessian and factor.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_np<0, true>(const SolveParams&, cudaStream_t, int*);
}  // namespace sapb
