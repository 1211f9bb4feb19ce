// Split-TF32 trailing-update GEMM on the 5th-generation tensor cores.
//   C[2M x N] (fp32, column-major, ldc) -= A[2M x K] * B[N x K]^T
// A and B are K-major fp32 operands prepared by the LU panel kernels
// (realified complex rows with the hi/lo TF32 split laid out along K).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace sieb200 {

struct GemmTC;

int gemm_tc_create(GemmTC** out);
void gemm_tc_destroy(GemmTC* g);
// Returns a SIEB200_* status; the kernel's bounded waits report through an
// error word checked on the next synchronization (gemm_tc_check).
// max_ctas > 0 caps the persistent kernel's grid, leaving the other SMs to
// concurrent work on other streams.
// layout 0: A and B are one K sweep; layout 1: [hi | lo] halves along K,
// C -= A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T (persistent kernel).
// shift0 > 0 leaves the first shift0 columns of the first 128 rows (one row
// tile) untouched: those rows take columns [shift0, N), the others [0, N)
// (the trailing update of a block LU whose next diagonal block is factored
// concurrently).
int gemm_tc_sub(GemmTC* g, cudaStream_t stream, float* C, int64_t ldc, const float* A,
                const float* B, int64_t M2, int64_t N, int K, int max_ctas = 0, int layout = 0,
                int64_t shift0 = 0);
int gemm_tc_check(GemmTC* g, cudaStream_t stream);
// Selects the implementation: 3 = persistent tcgen05 kernel whose epilogue
// adds -acc to C by TMA reduction (default), 2 = persistent kernel that
// loads, subtracts and stores the C tile by TMA, 1 = one CTA per tile
// tcgen05 kernel, 0 = SIMT on the same packed operands (checking path).
// SIEB200_GEMM_MODE=<0..3> in the environment overrides the default;
// SIEB200_GEMM_C_SLOTS=1 moves C in one 128-column slot instead of four
// 32-column ones.
void gemm_tc_set_mode(GemmTC* g, int mode);

}  // namespace sieb200
