// Contact-solve kernels specialised on 18 DOFs per world.
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_ns<18>(const SolveParams&, bool, cudaStream_t, int*);
}  // namespace sapb
