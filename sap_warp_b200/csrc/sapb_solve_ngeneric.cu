// Contact-solve kernels specialised on the DOF count at run time (n <= 60).
#include "sapb_contact_solve.cuh"

namespace sapb {
template cudaError_t launch_solve_ns<0>(const SolveParams&, bool, cudaStream_t, int*);
}  // namespace sapb
