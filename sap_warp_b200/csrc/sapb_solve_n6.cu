// Contact-solve kernels specialised on 6 DOFs per world.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_ns<6>(const SolveParams&, bool, cudaStream_t, int*);
}  // namespace sapb
