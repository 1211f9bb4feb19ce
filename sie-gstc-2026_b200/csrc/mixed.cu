// Own LU factorizations (FP64 and split-FP32 tensor-core) and GMRES-based
// iterative refinement. Filled in by the blocked-LU implementation.

#include "dense.cuh"

namespace sieb200 {

int mixed_factorize(DenseSolver* s) {
    (void)s;
    set_error("own LU factorization is not built into this library yet");
    return SIEB200_INVALID_ARG;
}

int mixed_solve(DenseSolver* s, int64_t nrhs, double* B, int64_t ldb, bool adjoint, double tol,
                int maxit, int* iters) {
    (void)s; (void)nrhs; (void)B; (void)ldb; (void)adjoint; (void)tol; (void)maxit; (void)iters;
    set_error("own LU solve is not built into this library yet");
    return SIEB200_INVALID_ARG;
}

void mixed_release(DenseSolver* s) { (void)s; }

}  // namespace sieb200
