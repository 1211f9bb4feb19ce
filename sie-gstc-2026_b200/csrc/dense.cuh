// Dense solver object shared by dense.cu (cuSOLVER reference path) and
// mixed.cu (own FP64 LU and split-FP32 tensor-core LU + GMRES refinement).
#pragma once

#include "common.cuh"

namespace sieb200 {

struct DenseSolver {
    sieb200_ctx* ctx = nullptr;
    int64_t n = 0;
    int method = 0;
    double* A = nullptr;  // FP64 matrix (cuSOLVER/own FP64: factors in place; mixed: original)
    int64_t lda = 0;
    bool factored = false;
    DeviceBuffer ipiv, work;
    // Own LU state (mixed.cu).
    DeviceBuffer lu;       // factors: complex64 (mixed) or complex128 (own FP64), n x n
    DeviceBuffer perm;     // row permutation, LAPACK-style swaps
    DeviceBuffer panel;    // panel / tournament workspace
    DeviceBuffer gemm_a, gemm_b;  // split-TF32 operand staging
    DeviceBuffer krylov;   // GMRES basis and small dense work
    DeviceBuffer vec;      // residual / work vectors
    DeviceBuffer flags;    // triangular-solve progress flags and error word
    DeviceBuffer gemv_scratch;
    DeviceBuffer couple;   // triangular-solve coupling products (mixed)
    void* gemm_state = nullptr;
    // Cap on the SMs of the persistent trailing GEMM (0: all but one); a
    // sweep running several systems concurrently gives each its share.
    int sm_cap = 0;

    int factorize(double* A, int64_t lda);
    int solve(int64_t nrhs, double* B, int64_t ldb, bool adjoint, double tol, int maxit, int* iters);
};

int mixed_factorize(DenseSolver* s);
int gmres_c64_prepare(DenseSolver* s);
int mixed_solve(DenseSolver* s, int64_t nrhs, double* B, int64_t ldb, bool adjoint, double tol,
                int maxit, int* iters);
void mixed_release(DenseSolver* s);

int gemv_device(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec, const cplx* x,
                double beta, cplx* y, DeviceBuffer& scratch);
// y = A^H x (+ beta y), A complex128 column-major.
int gemv_h_device(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, const cplx* x, double beta,
                  cplx* y);
// Same product with its partial sums in a fixed device array (no allocation).
// Measured FP64 FMA throughput of the device (TFLOP/s; FMA = 2 flops).
int fp64_fma_rate(sieb200_ctx* ctx, double* tflops);
int fp64_mma_rate(sieb200_ctx* ctx, double* tflops);
int gemv_device_static_scratch(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec,
                               const cplx* x, double beta, cplx* y);
void destroy_cusolver(sieb200_ctx* ctx);
// C = alpha A X + beta C, FP64 complex column-major (hand-written SIMT kernel,
// block_solve.cu).
int zgemm_device(cudaStream_t stream, int64_t m, int64_t nc, int64_t kdim, const cplx* A, int64_t lda,
                 const cplx* X, int64_t ldx, cplx* C, int64_t ldc, cplx alpha, cplx beta);

}  // namespace sieb200

struct sieb200_dense_solver {
    sieb200::DenseSolver impl;
};
