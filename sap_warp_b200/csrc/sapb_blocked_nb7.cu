// Tree-blocked solve kernels for blocks of 7 DOFs (both Hessian precisions, 128 and 256 threads, every line search).
#include "sapb_blocked_solve.cuh"

namespace sapb {
namespace blk {
template cudaError_t launch_blocked<7>(const BlockedParams&, bool, int, cudaStream_t);
}  // namespace blk
}  // namespace sapb
