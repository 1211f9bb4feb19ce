// Internal state of the mixed-precision dense solver (mixed.cu) shared with
// its multi-right-hand-side block solve (block_solve.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "dense.cuh"
#include "gemm_tc.cuh"
#include "sm100.cuh"

namespace sieb200 {

constexpr int NB = 64;  // LU block size (complex columns)

// Forward declaration: packed operands of the multi-right-hand-side solve.
struct BlockSolveState;

struct MixedState {
    int64_t n = 0, np = 0, ldw = 0, nbl = 0;
    float2* W = nullptr;        // factors, np x np, ld = ldw
    float2* Linv = nullptr;     // inverse unit-lower diagonal blocks, NB x NB each (col-major)
    float2* Uinv = nullptr;     // inverse upper diagonal blocks
    float* Apack[2] = {nullptr, nullptr};  // split realified L21: (2*np) x (6*NB), K-major; by step parity
    float* Bpack = nullptr;     // split U12 columns: np x (6*NB), K-major
    float2* panel = nullptr;    // NB x np scratch for U12 / np x NB for L21
    double* diag = nullptr;     // butterfly diagonals: U (level1 a,b; level2 e,f) and V, 4*np each
    unsigned* err = nullptr;    // error word (nonzero = failure code)
    unsigned* tri_flags = nullptr;   // per block progress flags (2 * nbl) + 2 tickets
    cplx* vecs = nullptr;       // FP64 work vectors
    int use_tc = 1;
    int hilo = 1;               // split [hi | lo] packs, three products per GEMM k-block
    int pair = 0;               // trailing update every second block step (K = 2 x 384)
    int pair_min = 0;           // pair schedule for steps whose paired GEMM is at least this wide
    int ovl_min = 0;            // overlap the next panels with GEMMs at least this wide (0: off)
    int ovl_sms = 20;           // SMs the overlapped GEMMs leave to the panels
    int lcol = 1;               // single steps: the next block column below its diagonal block takes the
                                // step's update from the panels (0), the GEMM (1, TF32) or col_update_kernel
                                // (FP32) on the third stream (2) or ahead of the GEMM (3)
    int lo_rn = 0;              // split packs: lo parts rounded to the nearest TF32 (else truncated by the MMA)
    int diag_split = 1;         // diagonal blocks take their update in a 16-CTA kernel ahead of the LU kernel
    int diag_panels = 0;        // diagonal-block elimination synchronised per panel of 8 steps, not per step
    int diag_rec = 0;           // diagonal block by 2 x 2 recursion over 32 x 32 warp-level factorizations
    int diag_compact = 0;       // diagonal-block elimination in one code path (runtime row half)
    int head_max = 0;           // single steps: panels whose trailing width is at most this split into a
                                // head (the next block's rows and columns) on the lookahead stream and the
                                // rest on the context stream (0: one panels launch)
    int head_smem = 0;          // dynamic shared memory of a head launch (bytes)
    GemmTC* gemm = nullptr;
    CUtensorMap tmW;                       // W for the triangular solves' tile loads
    const void* tm_base = nullptr;
    int tm_rows = 0;                       // rows per box of tmW / tmWH
    int64_t tm_np = 0;
    // Conjugate-transpose solves (W^H = U^H L^H): W^H and the conjugate
    // transposes of the diagonal-block inverses, built on first use after a
    // factorization (in the solver's panel workspace).
    cplx* dinv = nullptr;               // GMRES_C64: inverse diagonal of Z
    bool adj_ready = false;
    bool couple_ready[2] = {false, false};  // trsv_fold_kernel's products (forward, adjoint)
    float2* WH = nullptr;
    float2* LinvH = nullptr;
    float2* UinvH = nullptr;
    CUtensorMap tmWH;
    cudaStream_t side = nullptr;           // high-priority stream of the lookahead panel
    cudaEvent_t ev_cols = nullptr, ev_diag = nullptr, ev_pan = nullptr;
    cudaStream_t side2 = nullptr;          // third stream: the next block column's update beside the GEMM
    cudaEvent_t ev_lcol = nullptr;
    cudaEvent_t ev_gemm = nullptr, ev_head = nullptr;  // split panels: trailing GEMM done; head done
    // The factorization's launches as one CUDA graph (both streams and the
    // event edges between them), captured on the second call with an
    // unchanged key and replayed while it stays so; not while the profiler
    // is on (its per-kernel events run eagerly).
    struct GraphKey {
        const void* A = nullptr;
        int64_t lda = -1, n = -1;
        const void* W = nullptr;
        const void* pack = nullptr;
        int use_tc = -1, sms = -1;
        int64_t ovl = -1;
        int64_t head = -1;
        bool operator==(const GraphKey& o) const {
            return A == o.A && lda == o.lda && n == o.n && W == o.W && pack == o.pack && use_tc == o.use_tc &&
                   sms == o.sms && ovl == o.ovl && head == o.head;
        }
    };
    // Two graphs (for example one per buffer of a caller that uploads the
    // next system while this one is solved); the two keys seen last decide
    // what is worth capturing.
    struct Graph {
        GraphKey key;
        cudaGraphExec_t exec = nullptr;
        long long launches = 0;  // kernels per replay
        uint64_t used = 0;
    };
    Graph graphs[2];
    GraphKey seen[2];
    uint64_t tick = 0;
    // Multi-right-hand-side solve (block_solve.cu), built on first use after
    // a factorization.
    BlockSolveState* block = nullptr;
    // Own FP64 LU (SIEB200_SOLVER_LU_FP64): the same butterfly transform and
    // blocked schedule in complex128, factors in W64 (np x np, ld ldw).
    double2* W64 = nullptr;
    double2* Linv64 = nullptr;
    double2* Uinv64 = nullptr;
};

// Index quadruple of a depth-2 butterfly: {i, i+q, i+2q, i+3q}, q = np/4.
// Transposed application T^T = L1^T L2^T (first the two level-2 blocks, then
// level 1) of a butterfly with diagonals d = [a (h), b (h), e (h), f (h)],
// h = np/2: level-2 block s pairs (s h + i, s h + i + q) with e[s q + i],
// f[s q + i]; level 1 pairs (i', i' + h) with a[i'], b[i'].
template <class T>
__device__ __forceinline__ void bfly_T4(T x[4], const double* d, int64_t np, int64_t i) {
    const int64_t h = np / 2, q = np / 4;
    const double r = 0.70710678118654752440;
    const double* a = d;
    const double* b = d + h;
    const double* e = d + 2 * h;
    const double* f = d + 3 * h;
    // level-2 transpose: halves s = 0 (x0,x1) and s = 1 (x2,x3)
    T z[4];
    z[0] = (x[0] + x[1]) * (e[i] * r);
    z[1] = (x[0] - x[1]) * (f[i] * r);
    z[2] = (x[2] + x[3]) * (e[q + i] * r);
    z[3] = (x[2] - x[3]) * (f[q + i] * r);
    // level-1 transpose: pairs (i, i+h) -> (z0, z2), (i+q, i+q+h) -> (z1, z3)
    x[0] = (z[0] + z[2]) * (a[i] * r);
    x[2] = (z[0] - z[2]) * (b[i] * r);
    x[1] = (z[1] + z[3]) * (a[i + q] * r);
    x[3] = (z[1] - z[3]) * (b[i + q] * r);
}

// Forward application T = L2 L1 (level 1, then level 2).
template <class T>
__device__ __forceinline__ void bfly_N4(T x[4], const double* d, int64_t np, int64_t i) {
    const int64_t h = np / 2, q = np / 4;
    const double r = 0.70710678118654752440;
    const double* a = d;
    const double* b = d + h;
    const double* e = d + 2 * h;
    const double* f = d + 3 * h;
    T z[4];
    z[0] = (x[0] * a[i] + x[2] * b[i]) * r;
    z[2] = (x[0] * a[i] - x[2] * b[i]) * r;
    z[1] = (x[1] * a[i + q] + x[3] * b[i + q]) * r;
    z[3] = (x[1] * a[i + q] - x[3] * b[i + q]) * r;
    x[0] = (z[0] * e[i] + z[1] * f[i]) * r;
    x[1] = (z[0] * e[i] - z[1] * f[i]) * r;
    x[2] = (z[2] * e[q + i] + z[3] * f[q + i]) * r;
    x[3] = (z[2] * e[q + i] - z[3] * f[q + i]) * r;
}

__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t y;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(y) : "f"(x));
    return __uint_as_float(y);
}
// The remainder x - hi of the split: rounded to the nearest TF32 (rn != 0),
// or left in FP32, whose last 13 mantissa bits the tensor core ignores.
__device__ __forceinline__ float tf32_lo(float x, float hi, int rn) {
    const float l = x - hi;
    return rn ? tf32_hi(l) : l;
}

// The FGMRES cycles stop once the Arnoldi residual estimate is at most
// this fraction of tol * ||b||; the restart then checks the true FP64
// residual against tol * ||b|| itself (SIEB200_GMRES_EST_FACTOR, in (0, 1]).
double gmres_est_factor();

// Multi-right-hand-side solve with the mixed factors (block_solve.cu).
int block_solve(DenseSolver* s, MixedState* st, int64_t nrhs, double* B, int64_t ldb, double tol, int maxit,
                int* iters);
// Frees the block-solve workspaces (on release of the solver).
void block_solve_release(MixedState* st);
// Marks the packed factors stale (a new factorization was enqueued).
void block_solve_invalidate(MixedState* st);

}  // namespace sieb200
