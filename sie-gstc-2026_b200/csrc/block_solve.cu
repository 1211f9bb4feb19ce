// Multi-right-hand-side solve with the mixed factors: what cusolverDnZgetrs
// does for nrhs columns at once (include/sie_mom/cuda/dense_lu_solver.cuh:122-166,
// called with nrhs = case count by src/sie_mom/solvers/gstc_sie.cu:694-697),
// here as a batched FGMRES in FP64 whose preconditioner applies the
// split-FP32 factors to all columns together.
//
// Preconditioner M^{-1} R = V U^{-1} L^{-1} U^T R for an n x nrhs block R:
//   * the butterflies U^T and V column by column (FP64 in, complex64 Y);
//   * blocked triangular solves on Y in place: per 64-row block k the
//     diagonal block is applied through its explicit inverse (one small
//     kernel, which also packs the solved block as the tensor-core B operand),
//     then the rest of Y takes the block's contribution as one split-TF32
//     tcgen05 GEMM, Y[rows] -= L[rows, k] X_k (lower) or U[rows, k] X_k
//     (upper), with FP32 accumulation: 3 products hi*hi + hi*lo + lo*hi
//     of K = 128 (the realified complex columns) from split [hi | lo]
//     operands, each read once per tile;
//   * the GEMM's A operands (realified split rows of every L21 and every
//     column block of U above the diagonal) are packed from the factors once
//     per factorization, 32 np^2 bytes (48 np^2 with the three-product
//     layout [hi | hi | lo], SIEB200_BLOCK_HILO=0); when they do not fit, the
//     caller solves column by column instead.
// FGMRES: every column keeps its own Krylov space (classical Gram-Schmidt
// twice, Givens rotations on the host), but the columns advance in lockstep,
// so each iteration is one multi-column preconditioner application and one
// FP64 complex GEMM Z * [z_1 .. z_nrhs] (the hand-written zgemm_kernel
// below); a column whose residual estimate reaches the tolerance stops
// contributing (its direction is zero from then on).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "mixed.cuh"

namespace sieb200 {

struct BlockSolveState {
    int64_t np = 0, nbl = 0, ldy = 0;
    int nrhs_cap = 0;
    int kw = 0;           // pack width: KH (split [hi | lo], default) or K3 (SIEB200_BLOCK_HILO=0)
    DeviceBuffer packs;   // L packs | U packs (fp32)
    DeviceBuffer work;    // Y (np x nrhs c64) | Xpack (nrhs x 384 fp32)
    DeviceBuffer krylov;  // FP64 FGMRES vectors
    float* Lp = nullptr;
    float* Up = nullptr;
    float2* Y = nullptr;
    float* Xpack = nullptr;
    bool packed = false;  // packs match the current factors
    // The triangular solves on Y as one CUDA graph (captured on the second
    // application with an unchanged key).
    struct Key {
        const void* Y = nullptr;
        const void* packs = nullptr;
        const void* W = nullptr;
        int64_t np = 0;
        int nrhs = 0, kw = 0;
        bool operator==(const Key& o) const {
            return Y == o.Y && packs == o.packs && W == o.W && np == o.np && nrhs == o.nrhs && kw == o.kw;
        }
    };
    Key graph_key, seen_key;
    cudaGraphExec_t graph = nullptr;
    long long graph_launches = 0;
    // lookahead triangular solves: side-stream fork/join and per-step events
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_x[2] = {nullptr, nullptr}, ev_b[2] = {nullptr, nullptr};
};

namespace {

constexpr int K3 = 6 * NB;  // three-product packs: [hi | hi | lo] (A) or [hi | lo | hi] (B) of 2 NB reals
constexpr int KH = 4 * NB;  // split packs: [hi | lo] of 2 NB reals (A and B)

__host__ __device__ inline int64_t lower_pack_rows_before(int64_t k, int64_t np) {
    // sum over j < k of (np - NB (j + 1)): rows below diagonal block j
    return k * np - (int64_t)NB * k * (k + 1) / 2;
}
__host__ __device__ inline int64_t upper_pack_rows_before(int64_t k) {
    // sum over j < k of NB j: rows above diagonal block j
    return (int64_t)NB * k * (k - 1) / 2;
}

// Packs the GEMM A operands of both triangular solves from W: for block
// column k (grid.y), the split realified rows of L[s0:np, k] (grid.z = 0) or
// of U[0:k0, k] (grid.z = 1), 32 rows per CTA (grid.x), staged through
// shared memory so that both the column reads and the K-major row writes
// are coalesced. Row 2r: [Re, -Im] per column, row 2r + 1: [Im, Re];
// layout [hi | lo] along K (kw = KH) or [hi | hi | lo] (kw = K3); columns
// beyond the block's width are zero.
__global__ void __launch_bounds__(256) pack_factors_kernel(const float2* __restrict__ W, int64_t ldw, int64_t np,
                                                           float* __restrict__ Lp, float* __restrict__ Up,
                                                           int kw, int lo_rn) {
    __shared__ float2 tile[32][NB + 1];
    const int64_t k = blockIdx.y;
    const int64_t k0 = k * NB;
    const int kb = (int)(np - k0 < NB ? np - k0 : NB);
    const bool upper = blockIdx.z == 1;
    const int64_t r_begin = upper ? 0 : k0 + kb;
    const int64_t r_end = upper ? k0 : np;
    const int64_t rb = r_begin + (int64_t)blockIdx.x * 32;
    if (rb >= r_end) return;
    float* base = upper ? Up + 2 * upper_pack_rows_before(k) * kw : Lp + 2 * lower_pack_rows_before(k, np) * kw;
    const int tid = threadIdx.x;
    for (int e = tid; e < 32 * NB; e += blockDim.x) {
        const int r = e % 32, c = e / 32;
        const int64_t gr = rb + r;
        tile[r][c] = (gr < r_end && c < kb) ? W[gr + (k0 + c) * ldw] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int e = tid; e < 32 * 2 * NB; e += blockDim.x) {
        const int rr = e / (2 * NB), kk = e % (2 * NB);
        const int64_t gr = rb + rr;
        if (gr >= r_end) continue;
        const int c = kk >> 1, h = kk & 1;
        const float2 v = tile[rr][c];
        const float v0 = h == 0 ? v.x : -v.y;
        const float v1 = h == 0 ? v.y : v.x;
        const float h0 = tf32_hi(v0), h1 = tf32_hi(v1);
        float* row0 = base + (2 * (gr - r_begin)) * kw;
        float* row1 = row0 + kw;
        const float l0 = tf32_lo(v0, h0, lo_rn), l1 = tf32_lo(v1, h1, lo_rn);
        if (kw == KH) {
            row0[kk] = h0; row0[2 * NB + kk] = l0;
            row1[kk] = h1; row1[2 * NB + kk] = l1;
        } else {
            row0[kk] = h0; row0[2 * NB + kk] = h0; row0[4 * NB + kk] = l0;
            row1[kk] = h1; row1[2 * NB + kk] = h1; row1[4 * NB + kk] = l1;
        }
    }
}

// Y (np x nrhs, complex64, ldy) = U^T [R; 0] for the n x nrhs FP64 block R.
__global__ void rbt_block_T_kernel(const cplx* __restrict__ R, int64_t ldr, int64_t n, int64_t np,
                                   const double* __restrict__ d, float2* __restrict__ Y, int64_t ldy) {
    const int64_t q = np / 4;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (i >= q) return;
    const cplx* r = R + c * ldr;
    cplx v[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int64_t row = i + s * q;
        v[s] = row < n ? r[row] : cx(0, 0);
    }
    bfly_T4(v, d, np, i);
    float2* y = Y + c * ldy;
#pragma unroll
    for (int s = 0; s < 4; ++s) y[i + s * q] = make_float2((float)v[s].re, (float)v[s].im);
}

// Z (n x nrhs, FP64, ldz) = V Y (first n rows kept).
__global__ void rbt_block_N_kernel(const float2* __restrict__ Y, int64_t ldy, int64_t n, int64_t np,
                                   const double* __restrict__ d, cplx* __restrict__ Z, int64_t ldz) {
    const int64_t q = np / 4;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (i >= q) return;
    const float2* y = Y + c * ldy;
    cplx v[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const float2 t = y[i + s * q];
        v[s] = cx(t.x, t.y);
    }
    bfly_N4(v, d, np, i);
    cplx* z = Z + c * ldz;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int64_t row = i + s * q;
        if (row < n) z[row] = v[s];
    }
}

// Diagonal block k of a triangular solve on Y: X_k = Inv_k Y_k for 16
// columns per CTA (FP64 accumulation of the complex64 values), written back
// into Y and packed as the GEMM's B operand: column j of Xpack is
// [Re, Im] per row, split [hi | lo | hi] along K. Rows beyond the block's
// width are zero in Xpack (the inverse is padded with the identity).
// With Fb != null the block first takes the previous step's update itself,
// Y_k -= F X_prev (F the 64 x 64 factor block between the two, column-major
// with leading dimension ldf; X_prev the previous block's solved rows of Y,
// kbp of them): the trailing GEMM of the previous step skips this block, so
// that this kernel and that GEMM run side by side.
constexpr int DA_COLS = 16;
constexpr int kSmemDiagApply = (2 * NB * (NB + 1) + 2 * DA_COLS * NB) * (int)sizeof(float2);
__global__ void __launch_bounds__(256) diag_apply_kernel(float2* __restrict__ Y, int64_t ldy, int64_t k0, int kb,
                                                         int nrhs, const float2* __restrict__ Inv,
                                                         float* __restrict__ Xpack,
                                                         const float2* __restrict__ Fb, int64_t ldf,
                                                         const float2* __restrict__ Xprev, int kbp, int kw,
                                                         int lo_rn) {
    extern __shared__ __align__(16) float2 da_smem[];
    float2(*inv)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(da_smem);              // [row][col]
    float2(*fb)[NB + 1] = inv + NB;                                                    // [row][col]
    float2(*ys)[NB] = reinterpret_cast<float2(*)[NB]>(da_smem + 2 * NB * (NB + 1));   // [col][row]
    float2(*xp)[NB] = ys + DA_COLS;                                                    // [col][row]
    const int tid = threadIdx.x;
    const int c0 = blockIdx.x * DA_COLS;
    for (int e = tid; e < NB * NB; e += blockDim.x) inv[e % NB][e / NB] = Inv[e];  // Inv[r + c NB]
    for (int e = tid; e < DA_COLS * NB; e += blockDim.x) {
        const int r = e % NB, c = e / NB;
        ys[c][r] = (c0 + c < nrhs && r < kb) ? Y[(k0 + r) + (int64_t)(c0 + c) * ldy] : make_float2(0.f, 0.f);
    }
    if (Fb) {
        for (int e = tid; e < NB * NB; e += blockDim.x) {
            const int r = e % NB, c = e / NB;
            fb[r][c] = (r < kb && c < kbp) ? Fb[r + (int64_t)c * ldf] : make_float2(0.f, 0.f);
        }
        for (int e = tid; e < DA_COLS * NB; e += blockDim.x) {
            const int r = e % NB, c = e / NB;
            xp[c][r] = (c0 + c < nrhs && r < kbp) ? Xprev[r + (int64_t)(c0 + c) * ldy] : make_float2(0.f, 0.f);
        }
    }
    __syncthreads();
    const int c = tid / 16;         // column of this thread
    const int r0 = (tid % 16) * 4;  // its four rows
    if (Fb) {
        double fr[4] = {0, 0, 0, 0}, fi[4] = {0, 0, 0, 0};
        for (int kk = 0; kk < NB; ++kk) {
            const float2 x = xp[c][kk];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float2 a = fb[r0 + u][kk];
                fr[u] += (double)a.x * x.x - (double)a.y * x.y;
                fi[u] += (double)a.x * x.y + (double)a.y * x.x;
            }
        }
        // each thread owns rows r0 .. r0+3 of column c of ys
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float2 y = ys[c][r0 + u];
            ys[c][r0 + u] = make_float2((float)((double)y.x - fr[u]), (float)((double)y.y - fi[u]));
        }
        __syncthreads();
    }
    double ar[4] = {0, 0, 0, 0}, ai[4] = {0, 0, 0, 0};
    for (int kk = 0; kk < NB; ++kk) {
        const float2 y = ys[c][kk];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const float2 a = inv[r0 + u][kk];
            ar[u] += (double)a.x * y.x - (double)a.y * y.y;
            ai[u] += (double)a.x * y.y + (double)a.y * y.x;
        }
    }
    const int gc = c0 + c;
    if (gc >= nrhs) return;
    float* col = Xpack + (int64_t)gc * kw;  // [hi | lo] (KH) or [hi | lo | hi] (K3)
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int r = r0 + u;
        const bool in = r < kb;
        const float vx = in ? (float)ar[u] : 0.f, vy = in ? (float)ai[u] : 0.f;
        if (in) Y[(k0 + r) + (int64_t)gc * ldy] = make_float2(vx, vy);
        const float h0 = tf32_hi(vx), h1 = tf32_hi(vy);
        col[2 * r] = h0; col[2 * r + 1] = h1;
        col[2 * NB + 2 * r] = tf32_lo(vx, h0, lo_rn); col[2 * NB + 2 * r + 1] = tf32_lo(vy, h1, lo_rn);
        if (kw == K3) { col[4 * NB + 2 * r] = h0; col[4 * NB + 2 * r + 1] = h1; }
    }
}

// ------------------------------------------------------------ FP64 ZGEMM
// C (m x nc, ldc) = alpha A (m x kdim, lda) X (kdim x nc, ldx) + beta C, all
// complex128 column-major (beta = 0: C is not read). CTA tile 128 x 32 with
// K steps of 8 staged in shared memory (the next step's tiles are loaded
// into registers while the current one is multiplied); each of the 128
// threads accumulates an 8 x 4 block of complex products with FP64 FMAs.
constexpr int ZG_BM = 128, ZG_BN = 32, ZG_BK = 8, ZG_THREADS = 128;
constexpr int ZG_LA = ZG_BM * ZG_BK / ZG_THREADS;  // A entries per thread per K step
constexpr int ZG_LX = ZG_BK * ZG_BN / ZG_THREADS;  // X entries per thread

__global__ void __launch_bounds__(ZG_THREADS) zgemm_kernel(int64_t m, int64_t nc, int64_t kdim,
                                                           const double2* __restrict__ A, int64_t lda,
                                                           const double2* __restrict__ X, int64_t ldx,
                                                           double2* __restrict__ C, int64_t ldc, double2 alpha,
                                                           double2 beta) {
    __shared__ double2 As[2][ZG_BK][ZG_BM];
    __shared__ double2 Xs[2][ZG_BK][ZG_BN + 1];
    const int tid = threadIdx.x;
    const int64_t row0 = (int64_t)blockIdx.x * ZG_BM;
    const int64_t col0 = (int64_t)blockIdx.y * ZG_BN;
    const int tx = tid % 8, ty = tid / 8;  // columns 4 tx .. +3, rows 8 ty .. +7
    double2 acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
    double2 ra[ZG_LA], rx[ZG_LX];
    // A tile: 128 rows x 8 columns, row fastest; X tile: 8 rows x 32 columns.
    auto load = [&](int64_t k0) {
#pragma unroll
        for (int u = 0; u < ZG_LA; ++u) {
            const int e = tid + u * ZG_THREADS;
            const int r = e % ZG_BM, kk = e / ZG_BM;
            const int64_t gr = row0 + r, gk = k0 + kk;
            ra[u] = (gr < m && gk < kdim) ? A[gr + gk * lda] : make_double2(0.0, 0.0);
        }
#pragma unroll
        for (int u = 0; u < ZG_LX; ++u) {
            const int e = tid + u * ZG_THREADS;
            const int kk = e % ZG_BK, c = e / ZG_BK;
            const int64_t gk = k0 + kk, gc = col0 + c;
            rx[u] = (gk < kdim && gc < nc) ? X[gk + gc * ldx] : make_double2(0.0, 0.0);
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int u = 0; u < ZG_LA; ++u) {
            const int e = tid + u * ZG_THREADS;
            As[buf][e / ZG_BM][e % ZG_BM] = ra[u];
        }
#pragma unroll
        for (int u = 0; u < ZG_LX; ++u) {
            const int e = tid + u * ZG_THREADS;
            Xs[buf][e % ZG_BK][e / ZG_BK] = rx[u];
        }
    };
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (int64_t k0 = 0; k0 < kdim; k0 += ZG_BK) {
        const bool more = k0 + ZG_BK < kdim;
        if (more) load(k0 + ZG_BK);
#pragma unroll
        for (int kk = 0; kk < ZG_BK; ++kk) {
            double2 a[8], x[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[buf][kk][8 * ty + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) x[j] = Xs[buf][kk][4 * tx + j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc[i][j].x = fma(a[i].x, x[j].x, fma(-a[i].y, x[j].y, acc[i][j].x));
                    acc[i][j].y = fma(a[i].x, x[j].y, fma(a[i].y, x[j].x, acc[i][j].y));
                }
        }
        if (more) {
            store(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int64_t gc = col0 + 4 * tx + j;
        if (gc >= nc) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int64_t gr = row0 + 8 * ty + i;
            if (gr >= m) continue;
            const double2 v = acc[i][j];
            double2 out = make_double2(alpha.x * v.x - alpha.y * v.y, alpha.x * v.y + alpha.y * v.x);
            if (beta.x != 0.0 || beta.y != 0.0) {
                const double2 c = C[gr + gc * ldc];
                out.x += beta.x * c.x - beta.y * c.y;
                out.y += beta.x * c.y + beta.y * c.x;
            }
            C[gr + gc * ldc] = out;
        }
    }
}

// ------------------------------------------------ batched Krylov kernels
// h[i nrhs + c] = sum_r conj(V_i(r, c)) W(r, c) for i < nv: one CTA per
// (i, c), fixed-order reduction (bit-reproducible). V_i = V + i * ldv_blk.
__global__ void __launch_bounds__(256) bdot_kernel(int64_t n, int nrhs, const cplx* __restrict__ V,
                                                   int64_t ldv_blk, int64_t ldv, const cplx* __restrict__ W,
                                                   int64_t ldw, cplx* __restrict__ h) {
    __shared__ double sre[8], sim[8];
    const int i = blockIdx.y, c = blockIdx.x;
    const cplx* v = V + (int64_t)i * ldv_blk + (int64_t)c * ldv;
    const cplx* w = W + (int64_t)c * ldw;
    double re = 0.0, im = 0.0;
    for (int64_t r = threadIdx.x; r < n; r += blockDim.x) {
        const cplx a = v[r], b = w[r];
        re += a.re * b.re + a.im * b.im;
        im += a.re * b.im - a.im * b.re;
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) {
        sre[threadIdx.x >> 5] = re;
        sim[threadIdx.x >> 5] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            a += sre[k];
            b += sim[k];
        }
        h[(int64_t)i * nrhs + c] = cx(a, b);
    }
}

// W(:, c) -= sum_{i < nv} V_i(:, c) h[i nrhs + c]
__global__ void baxpy_kernel(int64_t n, int nrhs, int nv, const cplx* __restrict__ V, int64_t ldv_blk, int64_t ldv,
                             const cplx* __restrict__ h, cplx* __restrict__ W, int64_t ldw) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n) return;
    cplx acc = W[r + (int64_t)c * ldw];
    for (int i = 0; i < nv; ++i) {
        const cplx v = V[(int64_t)i * ldv_blk + (int64_t)c * ldv + r];
        const cplx s = h[(int64_t)i * nrhs + c];
        acc = acc - v * s;
    }
    W[r + (int64_t)c * ldw] = acc;
}

// Y(:, c) = X(:, c) * s[c]  (s real)
__global__ void bscale_kernel(int64_t n, const cplx* __restrict__ X, int64_t ldx, const double* __restrict__ s,
                              cplx* __restrict__ Y, int64_t ldy) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n) return;
    Y[r + (int64_t)c * ldy] = X[r + (int64_t)c * ldx] * s[c];
}

// X(:, c) += sum_{i < nv} Zd_i(:, c) y[i nrhs + c]
__global__ void bcombo_kernel(int64_t n, int nrhs, int nv, const cplx* __restrict__ Zd, int64_t ldz_blk,
                              int64_t ldz, const cplx* __restrict__ y, cplx* __restrict__ X, int64_t ldx) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n) return;
    cplx acc = X[r + (int64_t)c * ldx];
    for (int i = 0; i < nv; ++i) acc += Zd[(int64_t)i * ldz_blk + (int64_t)c * ldz + r] * y[(int64_t)i * nrhs + c];
    X[r + (int64_t)c * ldx] = acc;
}

__global__ void bcopy_kernel(int64_t n, const cplx* __restrict__ X, int64_t ldx, cplx* __restrict__ Y, int64_t ldy) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= n) return;
    Y[r + (int64_t)c * ldy] = X[r + (int64_t)c * ldx];
}

// The same product on the FP64 tensor cores (mma.sync m8n8k4 .f64, 256 FMAs
// per warp instruction): CTA tile 64 x 64 complex, four warps of 32 x 32,
// K stages of 16 complex columns brought by cp.async (16 bytes per complex
// entry, zero-filled outside the operands) into a 3-deep ring. Each 8 x 8
// output block keeps its real and imaginary parts in two accumulators:
//   Re += Ar Br + (-Ai) Bi,  Im += Ar Bi + Ai Br,
// four MMAs per block and k-step of 4. Fragments (PTX m8n8k4 .f64 layout):
// lane l holds A(l / 4, l % 4), B(l % 4, l / 4) and D(l / 4, 2 (l % 4) + {0, 1}).
// Shared layouts: A as [k][row] with rows padded to 66 (conflict-free
// 16-byte fragment loads), X as [col][k] with k padded to 20.
constexpr int ZD_BM = 64, ZD_BN = 64, ZD_BK = 16, ZD_THREADS = 128, ZD_STAGES = 3;
constexpr int ZD_ALD = ZD_BM + 2, ZD_XLD = ZD_BK + 4;
constexpr int ZD_STAGE_A = ZD_BK * ZD_ALD, ZD_STAGE_X = ZD_BN * ZD_XLD;  // complex entries
constexpr int kSmemZgemmDmma = ZD_STAGES * (ZD_STAGE_A + ZD_STAGE_X) * 16;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool in) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(ZD_THREADS, 2) zgemm_dmma_kernel(int64_t m, int64_t nc, int64_t kdim,
                                                                   const double2* __restrict__ A, int64_t lda,
                                                                   const double2* __restrict__ X, int64_t ldx,
                                                                   double2* __restrict__ C, int64_t ldc,
                                                                   double2 alpha, double2 beta) {
    extern __shared__ __align__(16) double2 zd_smem[];
    double2* As = zd_smem;                                // [stage][k][ZD_ALD]
    double2* Xs = zd_smem + ZD_STAGES * ZD_STAGE_A;       // [stage][col][ZD_XLD]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t row0 = (int64_t)blockIdx.x * ZD_BM, col0 = (int64_t)blockIdx.y * ZD_BN;
    const int wr = (warp & 1) * 32, wc = (warp >> 1) * 32;  // warp tile origin in the CTA tile
    const int nk = (int)((kdim + ZD_BK - 1) / ZD_BK);

    auto issue = [&](int kt) {
        const int st = kt % ZD_STAGES;
        const int64_t k0 = (int64_t)kt * ZD_BK;
        const uint32_t sa = (uint32_t)__cvta_generic_to_shared(As + st * ZD_STAGE_A);
        const uint32_t sx = (uint32_t)__cvta_generic_to_shared(Xs + st * ZD_STAGE_X);
#pragma unroll
        for (int u = 0; u < ZD_BM * ZD_BK / ZD_THREADS; ++u) {  // A: rows fastest
            const int e = tid + u * ZD_THREADS;
            const int r = e % ZD_BM, kk = e / ZD_BM;
            const int64_t gr = row0 + r, gk = k0 + kk;
            const bool in = gr < m && gk < kdim;
            cp_async16(sa + (uint32_t)(kk * ZD_ALD + r) * 16u, in ? (const void*)(A + gr + gk * lda) : (const void*)A,
                       in);
        }
#pragma unroll
        for (int u = 0; u < ZD_BN * ZD_BK / ZD_THREADS; ++u) {  // X: k fastest
            const int e = tid + u * ZD_THREADS;
            const int kk = e % ZD_BK, c = e / ZD_BK;
            const int64_t gk = k0 + kk, gc = col0 + c;
            const bool in = gk < kdim && gc < nc;
            cp_async16(sx + (uint32_t)(c * ZD_XLD + kk) * 16u, in ? (const void*)(X + gk + gc * ldx) : (const void*)X,
                       in);
        }
    };

    double re[4][4][2], im[4][4][2];  // [row block][col block][fragment pair]
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) re[i][j][0] = re[i][j][1] = im[i][j][0] = im[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < ZD_STAGES - 1; ++s) {
        if (s < nk) issue(s);
        cp_async_commit();
    }
    const int fr = lane >> 2, fk = lane & 3;
    for (int kt = 0; kt < nk; ++kt) {
        cp_async_wait<ZD_STAGES - 2>();
        __syncthreads();  // stage kt is in; stage kt - 1 is no longer read
        if (kt + ZD_STAGES - 1 < nk) issue(kt + ZD_STAGES - 1);
        cp_async_commit();
        const double2* as = As + (kt % ZD_STAGES) * ZD_STAGE_A;
        const double2* xs = Xs + (kt % ZD_STAGES) * ZD_STAGE_X;
#pragma unroll
        for (int k4 = 0; k4 < ZD_BK; k4 += 4) {
            double2 af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = as[(k4 + fk) * ZD_ALD + wr + 8 * i + fr];
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = xs[(wc + 8 * j + fr) * ZD_XLD + k4 + fk];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const double nai = -af[i].y;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    dmma(re[i][j][0], re[i][j][1], af[i].x, bf[j].x);
                    dmma(re[i][j][0], re[i][j][1], nai, bf[j].y);
                    dmma(im[i][j][0], im[i][j][1], af[i].x, bf[j].y);
                    dmma(im[i][j][0], im[i][j][1], af[i].y, bf[j].x);
                }
            }
        }
    }
    cp_async_wait<0>();
    const bool use_beta = beta.x != 0.0 || beta.y != 0.0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t gr = row0 + wr + 8 * i + fr;
        if (gr >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int64_t gc = col0 + wc + 8 * j + 2 * fk + h;
                if (gc >= nc) continue;
                const double vr = re[i][j][h], vi = im[i][j][h];
                double2 out = make_double2(alpha.x * vr - alpha.y * vi, alpha.x * vi + alpha.y * vr);
                if (use_beta) {
                    const double2 c = C[gr + gc * ldc];
                    out.x += beta.x * c.x - beta.y * c.y;
                    out.y += beta.x * c.y + beta.y * c.x;
                }
                C[gr + gc * ldc] = out;
            }
        }
    }
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// C = alpha A X + beta C (FP64 complex, column-major). Exposed for the
// residual of the batched refinement and its tests.
int zgemm_device(cudaStream_t stream, int64_t m, int64_t nc, int64_t kdim, const cplx* A, int64_t lda,
                 const cplx* X, int64_t ldx, cplx* C, int64_t ldc, cplx alpha, cplx beta) {
    if (m <= 0 || nc <= 0) return SIEB200_OK;
    SIEB_CHECK(nc < 65536ll * ZG_BN && m < (1ll << 40), SIEB200_INVALID_ARG, "zgemm: size out of range");
    // The tensor-core kernel needs 16-byte aligned operands (cp.async of one
    // complex entry); SIEB200_ZGEMM_DMMA=0 selects the FMA kernel.
    const char* dm_env = getenv("SIEB200_ZGEMM_DMMA");
    const bool aligned = ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(X) |
                           reinterpret_cast<uintptr_t>(C)) & 15) == 0;
    if (!(dm_env && dm_env[0] == '0') && aligned && nc < 65536ll * ZD_BN) {
        static bool attr_set[64] = {};
        int dev = 0;
        SIEB_TRY_CUDA(cudaGetDevice(&dev));
        if (!attr_set[dev & 63]) {
            SIEB_TRY_CUDA(cudaFuncSetAttribute(zgemm_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               kSmemZgemmDmma));
            attr_set[dev & 63] = true;
        }
        const dim3 grid(nblk(m, ZD_BM), nblk(nc, ZD_BN));
        zgemm_dmma_kernel<<<grid, ZD_THREADS, kSmemZgemmDmma, stream>>>(
            m, nc, kdim, reinterpret_cast<const double2*>(A), lda, reinterpret_cast<const double2*>(X), ldx,
            reinterpret_cast<double2*>(C), ldc, make_double2(alpha.re, alpha.im), make_double2(beta.re, beta.im));
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        return SIEB200_OK;
    }
    const dim3 grid(nblk(m, ZG_BM), nblk(nc, ZG_BN));
    zgemm_kernel<<<grid, ZG_THREADS, 0, stream>>>(m, nc, kdim, reinterpret_cast<const double2*>(A), lda,
                                                  reinterpret_cast<const double2*>(X), ldx,
                                                  reinterpret_cast<double2*>(C), ldc,
                                                  make_double2(alpha.re, alpha.im), make_double2(beta.re, beta.im));
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

void block_solve_release(MixedState* st) {
    if (!st || !st->block) return;
    BlockSolveState* bs = st->block;
    if (bs->graph) cudaGraphExecDestroy(bs->graph);
    for (cudaEvent_t e : {bs->ev_fork, bs->ev_join, bs->ev_x[0], bs->ev_x[1], bs->ev_b[0], bs->ev_b[1]})
        if (e) cudaEventDestroy(e);
    delete st->block;
    st->block = nullptr;
}

// Sizes and carves the packs and the Y / Xpack workspace; false when the
// packs would not fit in the device's free memory (the caller falls back).
static int prepare(DenseSolver* s, MixedState* st, int nrhs, bool* fits) {
    *fits = true;
    if (!st->block) st->block = new BlockSolveState();
    BlockSolveState* bs = st->block;
    const int64_t np = st->np, nbl = st->nbl;
    const int64_t l_rows = lower_pack_rows_before(nbl - 1, np);  // every L21 (the last block has none)
    const int64_t u_rows = upper_pack_rows_before(nbl);
    const char* hilo_env = getenv("SIEB200_BLOCK_HILO");
    const int kw = (hilo_env && hilo_env[0] == '0') ? K3 : KH;
    if (kw != bs->kw) bs->packed = false;
    bs->kw = kw;
    const size_t bL = sizeof(float) * 2 * (size_t)l_rows * kw;
    const size_t bU = sizeof(float) * 2 * (size_t)u_rows * kw;
    const size_t need = ((bL + 255) / 256) * 256 + bU;
    if (bs->packs.bytes < need) {
        size_t free_b = 0, total_b = 0;
        SIEB_TRY_CUDA(cudaMemGetInfo(&free_b, &total_b));
        const size_t margin = (size_t)2 << 30;
        if (need + margin > free_b + bs->packs.bytes) {
            *fits = false;
            return SIEB200_OK;
        }
        bs->packs.release();
        SIEB_RETURN_IF(bs->packs.reserve(need));
        bs->packed = false;
    }
    bs->Lp = bs->packs.as<float>();
    bs->Up = reinterpret_cast<float*>(bs->packs.as<char>() + ((bL + 255) / 256) * 256);
    const int64_t ldy = ((np + 31) / 32) * 32;
    const size_t bY = ((sizeof(float2) * (size_t)ldy * nrhs + 255) / 256) * 256;
    SIEB_RETURN_IF(bs->work.reserve(bY + 2 * sizeof(float) * (size_t)nrhs * kw));  // two Xpack buffers
    if (!bs->ev_fork) {
        for (cudaEvent_t* e : {&bs->ev_fork, &bs->ev_join, &bs->ev_x[0], &bs->ev_x[1], &bs->ev_b[0], &bs->ev_b[1]})
            SIEB_TRY_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        SIEB_TRY_CUDA(cudaFuncSetAttribute(diag_apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kSmemDiagApply));
    }
    bs->Y = bs->work.as<float2>();
    bs->Xpack = reinterpret_cast<float*>(bs->work.as<char>() + bY);
    bs->ldy = ldy;
    bs->np = np;
    bs->nbl = nbl;
    // The packs are built once per factorization (which clears `packed`).
    if (!bs->packed) {
        const dim3 grid(nblk(np, 32), (unsigned)nbl, 2);
        pack_factors_kernel<<<grid, 256, 0, s->ctx->stream>>>(st->W, st->ldw, np, bs->Lp, bs->Up, kw, st->lo_rn);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        bs->packed = true;
    }
    bs->nrhs_cap = nrhs;
    return SIEB200_OK;
}

// The two blocked triangular solves on Y (np x nrhs) in place.
// Lookahead (optional): the trailing GEMM of step k skips the next block,
// whose diagonal kernel takes step k's update itself (the fold), so the
// diagonal kernel of step k + 1 runs on the side stream beside the trailing
// GEMM of step k, which leaves it a few SMs; the diagonal kernel of step k
// waits for the trailing GEMM of step k - 2 (the last one that reaches its
// block and the last reader of its Xpack buffer, double-buffered by step).
// The default is one stream, every GEMM over all rows below: on the config-3
// system (N = 17280, 64 columns) the lookahead measured 18.8 against 16.7 ms
// per application (the diagonal kernels with the fold and the cross-stream
// hand-offs are slower than the GEMMs they overlap); SIEB200_BLOCK_LOOKAHEAD=1
// selects it.
static int enqueue_triangular(DenseSolver* s, MixedState* st, BlockSolveState* bs, int nrhs) {
    cudaStream_t stream = s->ctx->stream;
    const int64_t np = st->np, nbl = st->nbl;
    const unsigned gda = nblk(nrhs, DA_COLS);
    const char* la_env = getenv("SIEB200_BLOCK_LOOKAHEAD");
    const bool la = la_env && la_env[0] == '1' && st->side != nullptr;
    const int kw = bs->kw, layout = kw == KH ? 1 : 0;
    float* Xbuf[2] = {bs->Xpack, bs->Xpack + (size_t)nrhs * kw};
    if (!la) {
        for (int64_t k = 0; k < nbl; ++k) {
            const int64_t k0 = k * NB;
            const int kb = (int)std::min<int64_t>(NB, np - k0);
            diag_apply_kernel<<<gda, 256, kSmemDiagApply, stream>>>(bs->Y, bs->ldy, k0, kb, nrhs,
                                                                     st->Linv + (size_t)k * NB * NB, Xbuf[0],
                                                                     nullptr, 0, nullptr, 0, kw, st->lo_rn);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
            const int64_t s0 = k0 + kb;
            if (s0 < np) {
                const float* A = bs->Lp + 2 * lower_pack_rows_before(k, np) * kw;
                SIEB_RETURN_IF(gemm_tc_sub(st->gemm, stream, reinterpret_cast<float*>(bs->Y + s0), 2 * bs->ldy, A,
                                           Xbuf[0], 2 * (np - s0), nrhs, kw, 0, layout));
            }
        }
        for (int64_t k = nbl - 1; k >= 0; --k) {
            const int64_t k0 = k * NB;
            const int kb = (int)std::min<int64_t>(NB, np - k0);
            diag_apply_kernel<<<gda, 256, kSmemDiagApply, stream>>>(bs->Y, bs->ldy, k0, kb, nrhs,
                                                                     st->Uinv + (size_t)k * NB * NB, Xbuf[0],
                                                                     nullptr, 0, nullptr, 0, kw, st->lo_rn);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
            if (k0 > 0) {
                const float* A = bs->Up + 2 * upper_pack_rows_before(k) * kw;
                SIEB_RETURN_IF(gemm_tc_sub(st->gemm, stream, reinterpret_cast<float*>(bs->Y), 2 * bs->ldy, A,
                                           Xbuf[0], 2 * k0, nrhs, kw, 0, layout));
            }
        }
        return SIEB200_OK;
    }
    cudaStream_t side = st->side;
    const int cap = std::max(1, s->ctx->sm_count - 4);  // SMs left to the diagonal kernels
    SIEB_TRY_CUDA(cudaEventRecord(bs->ev_fork, stream));
    SIEB_TRY_CUDA(cudaStreamWaitEvent(side, bs->ev_fork, 0));
    for (int pass = 0; pass < 2; ++pass) {  // 0: L (forward), 1: U (backward)
        for (int64_t t = 0; t < nbl; ++t) {
            const int64_t k = pass == 0 ? t : nbl - 1 - t;
            const int64_t k0 = k * NB;
            const int kb = (int)std::min<int64_t>(NB, np - k0);
            float* Xk = Xbuf[t & 1];
            if (t >= 2) SIEB_TRY_CUDA(cudaStreamWaitEvent(side, bs->ev_b[t & 1], 0));
            // the previous step's update of this block, folded in
            const float2* Fb = nullptr;
            const float2* Xprev = nullptr;
            int kbp = 0;
            if (t >= 1) {
                const int64_t kprev = pass == 0 ? k - 1 : k + 1;
                const int64_t p0 = kprev * NB;
                Fb = st->W + k0 + p0 * st->ldw;
                Xprev = bs->Y + p0;
                kbp = (int)std::min<int64_t>(NB, np - p0);
            }
            diag_apply_kernel<<<gda, 256, kSmemDiagApply, side>>>(
                bs->Y, bs->ldy, k0, kb, nrhs, (pass == 0 ? st->Linv : st->Uinv) + (size_t)k * NB * NB, Xk, Fb,
                st->ldw, Xprev, kbp, kw, st->lo_rn);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
            SIEB_TRY_CUDA(cudaEventRecord(bs->ev_x[t & 1], side));
            // trailing update of every block but the next one
            const float* A;
            float* C;
            int64_t rows;
            if (pass == 0) {
                const int64_t s0 = k0 + kb, n1 = std::min<int64_t>(NB, np - s0);
                rows = np - s0 - n1;
                A = bs->Lp + 2 * (lower_pack_rows_before(k, np) + n1) * kw;
                C = reinterpret_cast<float*>(bs->Y + s0 + n1);
            } else {
                rows = k0 - NB;  // rows above the previous block
                A = bs->Up + 2 * upper_pack_rows_before(k) * kw;
                C = reinterpret_cast<float*>(bs->Y);
            }
            if (rows > 0) {
                SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, bs->ev_x[t & 1], 0));
                SIEB_RETURN_IF(gemm_tc_sub(st->gemm, stream, C, 2 * bs->ldy, A, Xk, 2 * rows, nrhs, kw, cap, layout));
            }
            // recorded every step, so that the wait two steps later sees
            // this step's GEMM (or, without one, everything before it)
            SIEB_TRY_CUDA(cudaEventRecord(bs->ev_b[t & 1], stream));
        }
        // the second pass starts from the whole first one
        SIEB_TRY_CUDA(cudaEventRecord(bs->ev_join, side));
        SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, bs->ev_join, 0));
        SIEB_TRY_CUDA(cudaEventRecord(bs->ev_fork, stream));
        SIEB_TRY_CUDA(cudaStreamWaitEvent(side, bs->ev_fork, 0));
    }
    SIEB_TRY_CUDA(cudaEventRecord(bs->ev_join, side));
    SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, bs->ev_join, 0));
    return SIEB200_OK;
}

// Z = M^{-1} R for n x nrhs FP64 blocks (ld n).
static int apply_block_precond(DenseSolver* s, MixedState* st, BlockSolveState* bs, const cplx* R, cplx* Z,
                               int nrhs) {
    sieb200_ctx* ctx = s->ctx;
    cudaStream_t stream = ctx->stream;
    const int64_t n = st->n, np = st->np, q = np / 4;
    rbt_block_T_kernel<<<dim3(nblk(q, 256), (unsigned)nrhs), 256, 0, stream>>>(R, n, n, np, st->diag, bs->Y,
                                                                                 bs->ldy);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    cudaEvent_t ev;
    ctx->prof.begin(stream, 5, 2.0 * 3.0 * 8.0 * (double)np * (double)np / 2.0 * nrhs,
                    2.0 * (4.0 * 2.0 * bs->kw * (double)np * (double)np / (2.0 * NB)), &ev);
    BlockSolveState::Key key;
    key.Y = bs->Y; key.packs = bs->packs.ptr; key.W = st->W; key.np = np; key.nrhs = nrhs; key.kw = bs->kw;
    const char* no_graphs = getenv("SIEB200_NO_GRAPHS");
    const bool graphs = !ctx->prof.enabled && !(no_graphs && no_graphs[0] == '1');
    if (graphs && bs->graph && bs->graph_key == key) {
        SIEB_TRY_CUDA(cudaGraphLaunch(bs->graph, stream));
        note_launches(bs->graph_launches);
    } else if (graphs && bs->seen_key == key) {
        if (bs->graph) cudaGraphExecDestroy(bs->graph);
        bs->graph = nullptr;
        const long long l0 = launch_count();
        SIEB_TRY_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_triangular(s, st, bs, nrhs);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(stream, &g);
        if (rc == SIEB200_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&bs->graph, g, 0);
        if (g) cudaGraphDestroy(g);
        if (rc != SIEB200_OK) return rc;
        if (ce != cudaSuccess) {
            cudaGetLastError();
            bs->graph = nullptr;
            set_error(std::string("capturing the block triangular solves failed: ") + cudaGetErrorString(ce));
            return SIEB200_CUDA_ERROR;
        }
        bs->graph_key = key;
        bs->graph_launches = launch_count() - l0;
        SIEB_TRY_CUDA(cudaGraphLaunch(bs->graph, stream));
    } else {
        bs->seen_key = key;
        SIEB_RETURN_IF(enqueue_triangular(s, st, bs, nrhs));
    }
    ctx->prof.end(stream, ev);
    rbt_block_N_kernel<<<dim3(nblk(q, 256), (unsigned)nrhs), 256, 0, stream>>>(bs->Y, bs->ldy, n, np,
                                                                                 st->diag + 4 * np, Z, n);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

static int fetch(cudaStream_t stream, void* host, const void* dev, size_t bytes) {
    SIEB_TRY_CUDA(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
    return SIEB200_OK;
}

int block_solve(DenseSolver* s, MixedState* st, int64_t nrhs64, double* Bd, int64_t ldb, double tol, int maxit,
                int* iters) {
    sieb200_ctx* ctx = s->ctx;
    cudaStream_t stream = ctx->stream;
    const int nrhs = (int)nrhs64;
    const int64_t n = st->n;
    bool fits = true;
    SIEB_RETURN_IF(prepare(s, st, nrhs, &fits));
    if (!fits) return -1;
    BlockSolveState* bs = st->block;
    // Restart length: the iteration budget up to 50 directions per column.
    const int m = std::max(1, std::min(maxit, 50));
    // X, R, W (n x nrhs each); V (m+1 blocks), Zd (m blocks); h, y, scales
    const size_t blk = (size_t)n * nrhs;
    const size_t small = (size_t)(m + 2) * nrhs;
    const size_t need = sizeof(cplx) * (blk * (3 + (m + 1) + m) + 2 * small) + sizeof(double) * nrhs + 1024;
    SIEB_RETURN_IF(bs->krylov.reserve(need));
    cplx* X = bs->krylov.as<cplx>();
    cplx* R = X + blk;
    cplx* W = R + blk;
    cplx* V = W + blk;
    cplx* Zd = V + (m + 1) * blk;
    cplx* hd = Zd + m * blk;
    cplx* yd = hd + small;
    double* sd = reinterpret_cast<double*>(yd + small);
    cplx* B = reinterpret_cast<cplx*>(Bd);
    const dim3 gv(nblk(n, 256), (unsigned)nrhs);
    // right-hand sides into R (ld n), their norms
    bcopy_kernel<<<gv, 256, 0, stream>>>(n, B, ldb, R, n);
    SIEB_NOTE_LAUNCH();
    std::vector<cplx> hh((size_t)(m + 2) * nrhs);
    bdot_kernel<<<dim3((unsigned)nrhs, 1), 256, 0, stream>>>(n, nrhs, R, 0, n, R, n, hd);
    SIEB_NOTE_LAUNCH();
    SIEB_RETURN_IF(fetch(stream, hh.data(), hd, sizeof(cplx) * nrhs));
    std::vector<double> bnorm(nrhs);
    const double est_factor = gmres_est_factor();
    for (int c = 0; c < nrhs; ++c) {
        bnorm[c] = std::sqrt(std::max(hh[c].re, 0.0));
        SIEB_CHECK(bnorm[c] > 0 && std::isfinite(bnorm[c]), SIEB200_INVALID_ARG,
                   "right-hand side norm must be finite and nonzero");
    }
    SIEB_TRY_CUDA(cudaMemsetAsync(X, 0, sizeof(cplx) * blk, stream));
    int total = 0;
    std::vector<cplx> H((size_t)(m + 1) * m * nrhs), g((size_t)(m + 1) * nrhs), cs((size_t)m * nrhs),
        sn((size_t)m * nrhs);
    std::vector<double> beta(nrhs), scale(nrhs);
    std::vector<int> active(nrhs), used(nrhs);
    for (int outer = 0; outer < 1000; ++outer) {
        if (outer > 0) {
            // R = B - Z X
            bcopy_kernel<<<gv, 256, 0, stream>>>(n, B, ldb, R, n);
            SIEB_NOTE_LAUNCH();
            cudaEvent_t ev;
            ctx->prof.begin(stream, 2, 8.0 * (double)n * n * nrhs, 16.0 * (double)n * n, &ev);
            SIEB_RETURN_IF(zgemm_device(stream, n, nrhs, n, reinterpret_cast<const cplx*>(s->A), s->lda, X, n, R, n,
                                        cx(-1, 0), cx(1, 0)));
            ctx->prof.end(stream, ev);
        }
        bdot_kernel<<<dim3((unsigned)nrhs, 1), 256, 0, stream>>>(n, nrhs, R, 0, n, R, n, hd);
        SIEB_NOTE_LAUNCH();
        SIEB_RETURN_IF(fetch(stream, hh.data(), hd, sizeof(cplx) * nrhs));
        int n_active = 0;
        for (int c = 0; c < nrhs; ++c) {
            beta[c] = std::sqrt(std::max(hh[c].re, 0.0));
            if (!std::isfinite(beta[c])) {
                set_error("GMRES refinement produced a non-finite residual");
                return SIEB200_NONFINITE;
            }
            active[c] = beta[c] > tol * bnorm[c];
            n_active += active[c];
            scale[c] = active[c] ? 1.0 / beta[c] : 0.0;
            used[c] = 0;
        }
        if (n_active == 0) break;
        if (total >= maxit) {
            if (iters) *iters = total;
            set_error("GMRES refinement did not reach the tolerance within max_iterations");
            return SIEB200_NOT_CONVERGED;
        }
        SIEB_TRY_CUDA(cudaMemcpyAsync(sd, scale.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, stream));
        bscale_kernel<<<gv, 256, 0, stream>>>(n, R, n, sd, V, n);
        SIEB_NOTE_LAUNCH();
        std::fill(g.begin(), g.end(), cx(0, 0));
        for (int c = 0; c < nrhs; ++c) g[(size_t)c * (m + 1)] = cx(active[c] ? beta[c] : 0.0, 0);
        int j = 0;
        for (; j < m && total < maxit; ++j, ++total) {
            cplx* vj = V + (size_t)j * blk;
            cplx* zj = Zd + (size_t)j * blk;
            SIEB_RETURN_IF(apply_block_precond(s, st, bs, vj, zj, nrhs));
            cudaEvent_t ev;
            ctx->prof.begin(stream, 2, 8.0 * (double)n * n * nrhs, 16.0 * (double)n * n, &ev);
            SIEB_RETURN_IF(zgemm_device(stream, n, nrhs, n, reinterpret_cast<const cplx*>(s->A), s->lda, zj, n, W, n,
                                        cx(1, 0), cx(0, 0)));
            ctx->prof.end(stream, ev);
            // CGS2
            std::vector<cplx> hsum((size_t)(j + 1) * nrhs, cx(0, 0));
            for (int pass = 0; pass < 2; ++pass) {
                bdot_kernel<<<dim3((unsigned)nrhs, (unsigned)(j + 1)), 256, 0, stream>>>(n, nrhs, V, (int64_t)blk, n,
                                                                                      W, n, hd);
                SIEB_NOTE_LAUNCH();
                baxpy_kernel<<<gv, 256, 0, stream>>>(n, nrhs, j + 1, V, (int64_t)blk, n, hd, W, n);
                SIEB_NOTE_LAUNCH();
                SIEB_TRY_CUDA(cudaGetLastError());
                SIEB_RETURN_IF(fetch(stream, hh.data(), hd, sizeof(cplx) * (j + 1) * nrhs));
                for (size_t e = 0; e < (size_t)(j + 1) * nrhs; ++e) hsum[e] += hh[e];
            }
            bdot_kernel<<<dim3((unsigned)nrhs, 1), 256, 0, stream>>>(n, nrhs, W, 0, n, W, n, hd);
            SIEB_NOTE_LAUNCH();
            SIEB_RETURN_IF(fetch(stream, hh.data(), hd, sizeof(cplx) * nrhs));
            int still = 0;
            for (int c = 0; c < nrhs; ++c) {
                const double hn = std::sqrt(std::max(hh[c].re, 0.0));
                scale[c] = 0.0;
                if (!active[c]) continue;
                cplx* Hc = &H[(size_t)c * (m + 1) * m];
                cplx* gc = &g[(size_t)c * (m + 1)];
                cplx* csc = &cs[(size_t)c * m];
                cplx* snc = &sn[(size_t)c * m];
                for (int i = 0; i <= j; ++i) Hc[(size_t)i * m + j] = hsum[(size_t)i * nrhs + c];
                for (int i = 0; i < j; ++i) {
                    const cplx a = Hc[(size_t)i * m + j], bb = Hc[(size_t)(i + 1) * m + j];
                    const cplx conj_s = cx(snc[i].re, -snc[i].im);
                    const cplx t1 = cx(csc[i].re * a.re + (snc[i] * bb).re, csc[i].re * a.im + (snc[i] * bb).im);
                    const cplx t2 = cx(-(conj_s * a).re + csc[i].re * bb.re, -(conj_s * a).im + csc[i].re * bb.im);
                    Hc[(size_t)i * m + j] = t1;
                    Hc[(size_t)(i + 1) * m + j] = t2;
                }
                const cplx a = Hc[(size_t)j * m + j];
                const double an = std::hypot(a.re, a.im), den = std::hypot(an, hn);
                if (den == 0.0) { csc[j] = cx(1, 0); snc[j] = cx(0, 0); }
                else if (an == 0.0) { csc[j] = cx(0, 0); snc[j] = cx(1, 0); }
                else {
                    csc[j] = cx(an / den, 0);
                    snc[j] = cx(a.re / an * hn / den, a.im / an * hn / den);
                }
                Hc[(size_t)j * m + j] = cx(csc[j].re * a.re + snc[j].re * hn, csc[j].re * a.im + snc[j].im * hn);
                const cplx gj = gc[j];
                const cplx conj_s = cx(snc[j].re, -snc[j].im);
                gc[j] = cx(csc[j].re * gj.re, csc[j].re * gj.im);
                gc[j + 1] = cx(-(conj_s * gj).re, -(conj_s * gj).im);
                used[c] = j + 1;
                const double est = std::hypot(gc[j + 1].re, gc[j + 1].im);
                if (est <= est_factor * tol * bnorm[c] || hn == 0.0) {
                    active[c] = 0;  // converged within this cycle: no further directions
                } else {
                    scale[c] = 1.0 / hn;
                    ++still;
                }
            }
            if (still == 0 || j + 1 == m) { ++j; ++total; break; }
            SIEB_TRY_CUDA(cudaMemcpyAsync(sd, scale.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, stream));
            bscale_kernel<<<gv, 256, 0, stream>>>(n, W, n, sd, V + (size_t)(j + 1) * blk, n);
            SIEB_NOTE_LAUNCH();
        }
        // y_c = H_c^{-1} g_c (upper triangular, used[c] x used[c]); X += Zd y
        const int jmax = *std::max_element(used.begin(), used.end());
        std::vector<cplx> ycol((size_t)jmax * nrhs, cx(0, 0));
        for (int c = 0; c < nrhs; ++c) {
            const int jc = used[c];
            const cplx* Hc = &H[(size_t)c * (m + 1) * m];
            const cplx* gc = &g[(size_t)c * (m + 1)];
            std::vector<cplx> y(jc);
            for (int i = jc - 1; i >= 0; --i) {
                cplx sacc = gc[i];
                for (int k = i + 1; k < jc; ++k) sacc = sacc - Hc[(size_t)i * m + k] * y[k];
                const cplx d = Hc[(size_t)i * m + i];
                const double dd = d.re * d.re + d.im * d.im;
                y[i] = dd > 0 ? cx((sacc.re * d.re + sacc.im * d.im) / dd, (sacc.im * d.re - sacc.re * d.im) / dd)
                              : cx(0, 0);
            }
            for (int i = 0; i < jc; ++i) ycol[(size_t)i * nrhs + c] = y[i];
        }
        if (jmax > 0) {
            SIEB_TRY_CUDA(cudaMemcpyAsync(yd, ycol.data(), sizeof(cplx) * ycol.size(), cudaMemcpyHostToDevice, stream));
            bcombo_kernel<<<gv, 256, 0, stream>>>(n, nrhs, jmax, Zd, (int64_t)blk, n, yd, X, n);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
        }
        SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
        SIEB_RETURN_IF(gemm_tc_check(st->gemm, stream));
    }
    bcopy_kernel<<<gv, 256, 0, stream>>>(n, X, n, B, ldb);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    if (iters) *iters = total;
    return SIEB200_OK;
}

// Marks the packs stale after a new factorization.
void block_solve_invalidate(MixedState* st) {
    if (st && st->block) st->block->packed = false;
}

}  // namespace sieb200
