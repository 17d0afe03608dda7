// Tree-blocked solve kernels for blocks of 6 DOFs (both Hessian precisions, 128 and 256 threads, every line search).
#include "sapb_blocked_solve.cuh"

namespace sapb {
namespace blk {
template cudaError_t launch_blocked<6>(const BlockedParams&, bool, int, cudaStream_t);
}  // namespace blk
}  // namespace sapb
