// sapb_internal.h -- declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/sapb.h"

namespace sapb {

// Dynamic shared memory a block may opt into on sm_100 (227 KB) minus the
// kernels' static shared memory.
constexpr size_t kMaxSmemPerBlock = 227 * 1024 - 1024;

void set_last_error(const char* fmt, ...);

size_t contact_solve_smem_bytes(int n, int C, int hessian_precision);
int32_t contact_solve_launch(const sapb_contact_problem* p, const sapb_solve_options* o, const sapb_solve_outputs* out,
                             void* workspace, size_t workspace_bytes, cudaStream_t stream);

}  // namespace sapb
