// Mixed-precision dense solver: randomized butterfly transform + blocked LU
// without pivoting in complex64 with split-TF32 tensor-core trailing updates,
// wrapped in FP64 restarted GMRES (right preconditioned) against the intact
// complex128 system. Replaces the cusolverDnZgetrf/Zgetrs path of
// include/sie_mom/cuda/dense_lu_solver.cuh:42-166 for the solves/s metric.
//
// Method (published): Parker's random butterfly transform makes Gaussian
// elimination without pivoting safe with high probability; Baboulin,
// Dongarra et al. ("Accelerating linear system solutions using randomization
// techniques", ACM TOMS 2013) pair it with iterative refinement. Here:
//   W = U^T A V  (depth-2 recursive butterflies, random diagonals exp(r/10),
//                 r uniform in [-1/2, 1/2], fixed seed), A padded to a
//                 multiple of 4 with an identity block,
//   W = L U      (no pivoting, block size NB; diagonal blocks factored and
//                 inverted in one CTA each; panels by explicit block inverses;
//                 trailing update on the tensor cores, or SIMT for checking),
//   M^{-1} r = V U^{-1} L^{-1} U^T r  (single-kernel blocked triangular
//                 solves with progress flags, FP64 arithmetic on c64 factors),
//   GMRES(m) in FP64 on A M^{-1} until ||b - A x|| <= tol ||b||.
// Every spin-wait is bounded: on timeout the kernel records an error word and
// returns; the host reports SIEB200_TIMEOUT.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "mixed.cuh"

namespace sieb200 {

namespace {

// Dynamic shared memory of the block kernels (two NB x (NB+1) complex64
// tiles, or one plus a 32-row slab).
constexpr int kSmemDiag = (2 * NB * (NB + 1) + NB * NB / 4) * (int)sizeof(float2);
constexpr int kSmemPanel = (NB * (NB + 4) + 2 * 32 * (NB + 1)) * (int)sizeof(float2);
// Upper bound of a split panels head's dynamic shared memory: asking for
// more than kSmemPanel keeps the other panels' CTAs (kSmemPanel each) off
// the head's SMs (228 KB per SM).
constexpr int kSmemPanelHeadMax = 200 * 1024;
// Panel CTAs: 256 threads; a 32-row (32-column) slab of NB entries and an
// NB x NB inverse are 8 and 16 entries per thread.
constexpr int kPanelThreads = 256;
constexpr int kPanelSlab = 32 * NB / kPanelThreads;
constexpr int kPanelInv = NB * NB / kPanelThreads;
static_assert(NB == 64 && kPanelThreads == 256, "panel threads: 16 x 16, four columns (rows) of 64 each");
// The diagonal-block kernel stages the previous step's two 64 x 64 factor
// blocks; its size also keeps it off SMs that hold a trailing-GEMM CTA.
constexpr int kSmemDiagUpd = 2 * NB * (NB + 1) * (int)sizeof(float2);
constexpr int kDiagThreads = 256;  // diagonal-block kernel: 8 warps of NB / 8 columns
// The same two kernels in complex128 (own FP64 LU).
constexpr int kSmemPanel64 = (NB * (NB + 4) + 2 * 32 * (NB + 1)) * (int)sizeof(double2);
constexpr int kSmemDiagUpd64 = 2 * NB * (NB + 1) * (int)sizeof(double2);


// SIEB200_DIAG_SPLIT=0 folds the diagonal blocks' updates back into the LU
// kernel.
static int diag_split_env() {
    const char* e = getenv("SIEB200_DIAG_SPLIT");
    return (e && e[0] == '0') ? 0 : 1;
}

// SIEB200_DIAG_PANELS=1: the diagonal-block elimination with one named
// barrier per panel instead of one block barrier per step (measured ~2 us
// per launch slower in the N = 6000 factorization).
static int diag_panels_env() {
    const char* e = getenv("SIEB200_DIAG_PANELS");
    return (e && e[0] == '1') ? 1 : 0;
}

// SIEB200_DIAG_COMPACT=1: diag_steps_compact instead of the fully unrolled
// elimination (11 % faster alone under ncu, 31.2 against 35.0 us, but the
// factorization measured 6.05 against 5.98 ms at N = 6016 in situ).
static int diag_compact_env() {
    const char* e = getenv("SIEB200_DIAG_COMPACT");
    return (e && e[0] == '1') ? 1 : 0;
}

static void drop_graphs(MixedState* st) {
    for (auto& g : st->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = MixedState::Graph();
    }
}

// ------------------------------------------------------------ butterflies
__device__ __forceinline__ double rbt_value(uint64_t seed, int64_t i) {
    // splitmix64 -> uniform r in [-1/2, 1/2] -> exp(r / 10)
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    const double u = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
    return exp(u / 10.0);
}

__global__ void rbt_init_kernel(double* diag, int64_t np, uint64_t seed) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 8 * np) return;
    diag[i] = rbt_value(seed, i);
}

// W = U^T A_pad V, read A (c128, n x n, lda) once, write W (c64).
template <class T>
__global__ void rbt_matrix_kernel(const cplx* __restrict__ A, int64_t lda, int64_t n, int64_t np,
                                  const double* __restrict__ du, const double* __restrict__ dv,
                                  T* __restrict__ W, int64_t ldw) {
    const int64_t q = np / 4;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t j = blockIdx.y;
    if (i >= q || j >= q) return;
    cplx blk[4][4];  // [row s][col t]
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        const int64_t c = j + t * q;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int64_t r = i + s * q;
            cplx v;
            if (r < n && c < n) v = A[r + c * lda];
            else v = cx(r == c ? 1.0 : 0.0, 0.0);
            blk[s][t] = v;
        }
    }
    // rows: U^T on each column
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        cplx x[4] = {blk[0][t], blk[1][t], blk[2][t], blk[3][t]};
        bfly_T4(x, du, np, i);
#pragma unroll
        for (int s = 0; s < 4; ++s) blk[s][t] = x[s];
    }
    // columns: (row) * V = (V^T row^T)^T
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        cplx x[4] = {blk[s][0], blk[s][1], blk[s][2], blk[s][3]};
        bfly_T4(x, dv, np, j);
#pragma unroll
        for (int t = 0; t < 4; ++t) blk[s][t] = x[t];
    }
#pragma unroll
    for (int t = 0; t < 4; ++t)
#pragma unroll
        for (int s = 0; s < 4; ++s)
            W[(i + s * q) + (j + t * q) * ldw] = T{(decltype(T::x))blk[s][t].re, (decltype(T::x))blk[s][t].im};
}

// y = U^T x_pad (vector); x has n entries (rest treated as 0).
__global__ void rbt_vec_T_kernel(const cplx* __restrict__ x, int64_t n, int64_t np,
                                 const double* __restrict__ d, cplx* __restrict__ y) {
    const int64_t q = np / 4;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q) return;
    cplx v[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int64_t r = i + s * q;
        v[s] = r < n ? x[r] : cx(0, 0);
    }
    bfly_T4(v, d, np, i);
#pragma unroll
    for (int s = 0; s < 4; ++s) y[i + s * q] = v[s];
}

// x = V y (first n entries kept).
__global__ void rbt_vec_N_kernel(const cplx* __restrict__ y, int64_t n, int64_t np,
                                 const double* __restrict__ d, cplx* __restrict__ x) {
    const int64_t q = np / 4;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= q) return;
    cplx v[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) v[s] = y[i + s * q];
    bfly_N4(v, d, np, i);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int64_t r = i + s * q;
        if (r < n) x[r] = v[s];
    }
}

// ------------------------------------------------------------ block LU
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cnegf(float2 a) { return make_float2(-a.x, -a.y); }
// a - c x with fused multiply-adds.
__device__ __forceinline__ float2 cfmsf(float2 a, float2 c, float2 x) {
    return make_float2(fmaf(-c.x, x.x, fmaf(c.y, x.y, a.x)), fmaf(-c.x, x.y, fmaf(-c.y, x.x, a.y)));
}
__device__ __forceinline__ float2 shfl_c(float2 v, int src) {
    return make_float2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// The same helpers for complex128, so that the block kernels below run in
// either precision (complex64 for the mixed LU, complex128 for the own FP64
// LU).
__device__ __forceinline__ double2 cmulf(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cnegf(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 cfmsf(double2 a, double2 c, double2 x) {
    return make_double2(fma(-c.x, x.x, fma(c.y, x.y, a.x)), fma(-c.x, x.y, fma(-c.y, x.x, a.y)));
}
__device__ __forceinline__ double2 shfl_c(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
template <class T> struct RealOf;
template <> struct RealOf<float2> { using type = float; };
template <> struct RealOf<double2> { using type = double; };
template <class T> __device__ __forceinline__ T cmk(double x, double y);
template <> __device__ __forceinline__ float2 cmk<float2>(double x, double y) { return make_float2((float)x, (float)y); }
template <> __device__ __forceinline__ double2 cmk<double2>(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float rcp_rn(float x) { return __frcp_rn(x); }
__device__ __forceinline__ double rcp_rn(double x) { return __drcp_rn(x); }
// |pivot|^2 below this counts as a zero pivot.
__device__ __forceinline__ float tiny_pivot(float) { return 1e-30f; }
__device__ __forceinline__ double tiny_pivot(double) { return 1e-280; }

// Diagonal block: LU without pivoting and both triangular inverses in one
// pass of NB rank-1 steps over registers. Warp w holds columns
// [kDiagCols w, kDiagCols (w+1)), lane l rows l and l+32. Step j takes the
// coefficient column c_j = col_j / p_j (p_j the pivot, entry j zeroed) from
// the warp that owns column j and applies  a(r, c) -= c_j(r) a(j, c)  to
// every column c != j, restricted to rows r > j when c < j. Per column c
// this is, in turn,
//   * for j < c: the elimination itself (rows > j) and, in rows r < j, the
//     accumulation of S(r, c) = -p_r inv(U~)(r, c), where U = D U~ (U~
//     unit upper): the rows of the transposed elimination scaled by -p_r,
//     which leaves row j of U in place at step j;
//   * at j = c: the column becomes -l_c below the pivot (E_c = I - l_c e_c^T);
//   * for j > c: inv(L) = E_{NB-1} ... E_0 accumulated below the diagonal.
// So the register ends as [inv(L) strictly below | p_c | S strictly above],
// with inv(U)(r, c) = -S(r, c) / (p_r p_c) and 1/p_c on the diagonal. The
// block is padded to NB x NB with the identity (kb < NB only at the end).
// A zero or non-finite pivot sets the error word and continues with a zero
// reciprocal. The diagonal block of W itself is only read: everything after
// the factorization takes the diagonal blocks from Linv / Uinv.
constexpr int kDiagWarps = kDiagThreads / 32;
constexpr int kDiagCols = NB / kDiagWarps;
static_assert(kDiagCols % 2 == 0 && 32 % kDiagCols == 0, "diag column split");

// Steps j = kDiagCols bp + u, u = 0 .. kDiagCols-1, all in row half H.
template <class T, int H>
__device__ __forceinline__ void diag_steps(T (&a)[kDiagCols][2], int bp, int w, int lane,
                                           T (*cbuf)[NB], T* rcps, unsigned* err) {
    using R = typename RealOf<T>::type;
    constexpr int CW = kDiagCols;
#pragma unroll
    for (int u = 0; u < CW; ++u) {
        const int j = CW * bp + u, jl = j & 31, buf = u & 1;
        const bool g0 = lane > j, g1 = lane + 32 > j;  // rows below the pivot
        const T z = cmk<T>(0.f, 0.f);
        T ca0, ca1;
        if (w == bp) {  // publish c_j, then update this warp's other columns
            const T piv = shfl_c(a[u][H], jl);
            const R pm = piv.x * piv.x + piv.y * piv.y;
            const bool bad = !(pm > tiny_pivot(pm)) || !isfinite(pm);
            if (bad && lane == 0) atomicCAS(err, 0u, 1u);
            const R inv = bad ? R(0) : rcp_rn(pm);
            const T rcp = cmk<T>(piv.x * inv, -piv.y * inv);
            ca0 = cmulf(a[u][0], rcp);
            ca1 = cmulf(a[u][1], rcp);
            if (lane == jl) {
                if (H) ca1 = z;
                else ca0 = z;
            }
            cbuf[buf][lane] = ca0;
            cbuf[buf][lane + 32] = ca1;
            if (lane == 0) rcps[j] = rcp;
            a[u][0] = g0 ? cnegf(ca0) : a[u][0];
            a[u][1] = g1 ? cnegf(ca1) : a[u][1];
            const T cl0 = g0 ? ca0 : z, cl1 = g1 ? ca1 : z;
#pragma unroll
            for (int v = 0; v < CW; ++v) {
                if (v == u) continue;
                const T x = shfl_c(a[v][H], jl);
                if (v < u) {
                    if (H == 0) a[v][0] = cfmsf(a[v][0], cl0, x);
                    a[v][1] = cfmsf(a[v][1], cl1, x);
                } else {
                    a[v][0] = cfmsf(a[v][0], ca0, x);
                    a[v][1] = cfmsf(a[v][1], ca1, x);
                }
            }
        }
        __syncthreads();
        if (w != bp) {
            ca0 = cbuf[buf][lane];
            ca1 = cbuf[buf][lane + 32];
            if (w < bp) {  // columns left of the pivot: rows below j only
                const T cl0 = g0 ? ca0 : z, cl1 = g1 ? ca1 : z;
#pragma unroll
                for (int v = 0; v < CW; ++v) {
                    const T x = shfl_c(a[v][H], jl);
                    if (H == 0) a[v][0] = cfmsf(a[v][0], cl0, x);
                    a[v][1] = cfmsf(a[v][1], cl1, x);
                }
            } else {
#pragma unroll
                for (int v = 0; v < CW; ++v) {
                    const T x = shfl_c(a[v][H], jl);
                    a[v][0] = cfmsf(a[v][0], ca0, x);
                    a[v][1] = cfmsf(a[v][1], ca1, x);
                }
            }
        }
    }
}

// diag_steps with the row half H a runtime value and the two non-owner
// cases (columns left or right of the pivot block) in one code path through
// warp-uniform selects: the same FMAs on the same values in the same order
// (same results), in about a third of the instructions of the unrolled
// code, whose fetch was the kernel's top stall (no_instruction).
template <class T>
__device__ __forceinline__ void diag_steps_compact(T (&a)[kDiagCols][2], int bp, int H, int w, int lane,
                                                   T (*cbuf)[NB], T* rcps, unsigned* err) {
    using R = typename RealOf<T>::type;
    constexpr int CW = kDiagCols;
    const bool left = w < bp;   // this warp's columns lie left of the pivot block
    const bool keep0 = H != 0;  // rows 0..31 are above every pivot of this half
#pragma unroll
    for (int u = 0; u < CW; ++u) {
        const int j = CW * bp + u, jl = j & 31, buf = u & 1;
        const bool g0 = lane > j, g1 = lane + 32 > j;  // rows below the pivot
        const T z = cmk<T>(0.f, 0.f);
        if (w == bp) {  // publish c_j, then update this warp's other columns
            const T piv = shfl_c(keep0 ? a[u][1] : a[u][0], jl);
            const R pm = piv.x * piv.x + piv.y * piv.y;
            const bool bad = !(pm > tiny_pivot(pm)) || !isfinite(pm);
            if (bad && lane == 0) atomicCAS(err, 0u, 1u);
            const R inv = bad ? R(0) : rcp_rn(pm);
            const T rcp = cmk<T>(piv.x * inv, -piv.y * inv);
            T ca0 = cmulf(a[u][0], rcp);
            T ca1 = cmulf(a[u][1], rcp);
            if (lane == jl) {
                if (keep0) ca1 = z;
                else ca0 = z;
            }
            cbuf[buf][lane] = ca0;
            cbuf[buf][lane + 32] = ca1;
            if (lane == 0) rcps[j] = rcp;
            a[u][0] = g0 ? cnegf(ca0) : a[u][0];
            a[u][1] = g1 ? cnegf(ca1) : a[u][1];
            const T cl0 = g0 ? ca0 : z, cl1 = g1 ? ca1 : z;
#pragma unroll
            for (int v = 0; v < CW; ++v) {
                if (v == u) continue;
                const T x = shfl_c(keep0 ? a[v][1] : a[v][0], jl);
                if (v < u) {
                    a[v][0] = keep0 ? a[v][0] : cfmsf(a[v][0], cl0, x);
                    a[v][1] = cfmsf(a[v][1], cl1, x);
                } else {
                    a[v][0] = cfmsf(a[v][0], ca0, x);
                    a[v][1] = cfmsf(a[v][1], ca1, x);
                }
            }
        }
        __syncthreads();
        if (w != bp) {
            const T ca0 = cbuf[buf][lane], ca1 = cbuf[buf][lane + 32];
            // left of the pivot block: rows below j only, and nothing in
            // rows 0..31 once the pivots are in the lower half
            const T k0 = left ? (g0 ? ca0 : z) : ca0;
            const T k1 = left ? (g1 ? ca1 : z) : ca1;
            const bool skip0 = left && keep0;
#pragma unroll
            for (int v = 0; v < CW; ++v) {
                const T x = shfl_c(keep0 ? a[v][1] : a[v][0], jl);
                a[v][0] = skip0 ? a[v][0] : cfmsf(a[v][0], k0, x);
                a[v][1] = cfmsf(a[v][1], k1, x);
            }
        }
    }
}

// The same steps, one panel of kDiagCols columns at a time: the warp that// The same steps, one panel of kDiagCols columns at a time: the warp that
// owns columns [kDiagCols p, kDiagCols (p+1)) runs the panel's steps alone
// (its own columns only, through shuffles), leaving each coefficient column
// c_j in cbuf[j], and signals named barrier 1 + p without waiting on it
// (bar.arrive); every other warp waits there (bar.sync) and then applies the
// panel's steps to its columns. So while the others apply panel p, the warp
// owning panel p + 1 applies it to its own columns and goes on to factor
// them: one barrier per panel instead of one per step, and no warp waits for
// a panel's update of columns other than its own. Each column takes the
// same updates in the same order as in diag_steps (same results). cbuf
// holds all NB coefficient columns ([j][row]); every barrier id is used
// once, and warp p arrives at its barrier only after passing those of
// panels 0 .. p-1, whose owners arrive unconditionally: no wait can hang.
__device__ __forceinline__ void named_bar_arrive(int id, int threads) {
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(threads) : "memory");
}
__device__ __forceinline__ void named_bar_sync(int id, int threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

template <class T, int H>
__device__ __forceinline__ void diag_panel(T (&a)[kDiagCols][2], int p, int w, int lane, T (*cbuf)[NB],
                                           T* rcps, unsigned* err) {
    using R = typename RealOf<T>::type;
    constexpr int CW = kDiagCols;
    const T z = cmk<T>(0.f, 0.f);
    if (w == p) {
#pragma unroll
        for (int u = 0; u < CW; ++u) {
            const int j = CW * p + u, jl = j & 31;
            const bool g0 = lane > j, g1 = lane + 32 > j;
            const T piv = shfl_c(a[u][H], jl);
            const R pm = piv.x * piv.x + piv.y * piv.y;
            const bool bad = !(pm > tiny_pivot(pm)) || !isfinite(pm);
            if (bad && lane == 0) atomicCAS(err, 0u, 1u);
            const R inv = bad ? R(0) : rcp_rn(pm);
            const T rcp = cmk<T>(piv.x * inv, -piv.y * inv);
            T ca0 = cmulf(a[u][0], rcp);
            T ca1 = cmulf(a[u][1], rcp);
            if (lane == jl) {
                if (H) ca1 = z;
                else ca0 = z;
            }
            cbuf[j][lane] = ca0;
            cbuf[j][lane + 32] = ca1;
            if (lane == 0) rcps[j] = rcp;
            a[u][0] = g0 ? cnegf(ca0) : a[u][0];
            a[u][1] = g1 ? cnegf(ca1) : a[u][1];
            const T cl0 = g0 ? ca0 : z, cl1 = g1 ? ca1 : z;
#pragma unroll
            for (int v = 0; v < CW; ++v) {
                if (v == u) continue;
                const T x = shfl_c(a[v][H], jl);
                if (v < u) {
                    if (H == 0) a[v][0] = cfmsf(a[v][0], cl0, x);
                    a[v][1] = cfmsf(a[v][1], cl1, x);
                } else {
                    a[v][0] = cfmsf(a[v][0], ca0, x);
                    a[v][1] = cfmsf(a[v][1], ca1, x);
                }
            }
        }
        __syncwarp();
        named_bar_arrive(1 + p, kDiagThreads);
    } else {
        named_bar_sync(1 + p, kDiagThreads);
#pragma unroll
        for (int u = 0; u < CW; ++u) {
            const int j = CW * p + u, jl = j & 31;
            const bool g0 = lane > j, g1 = lane + 32 > j;
            const T ca0 = cbuf[j][lane], ca1 = cbuf[j][lane + 32];
            if (w < p) {  // columns left of the pivot: rows below j only
                const T cl0 = g0 ? ca0 : z, cl1 = g1 ? ca1 : z;
#pragma unroll
                for (int v = 0; v < CW; ++v) {
                    const T x = shfl_c(a[v][H], jl);
                    if (H == 0) a[v][0] = cfmsf(a[v][0], cl0, x);
                    a[v][1] = cfmsf(a[v][1], cl1, x);
                }
            } else {
#pragma unroll
                for (int v = 0; v < CW; ++v) {
                    const T x = shfl_c(a[v][H], jl);
                    a[v][0] = cfmsf(a[v][0], ca0, x);
                    a[v][1] = cfmsf(a[v][1], ca1, x);
                }
            }
        }
    }
}

// ---- diagonal block by 2 x 2 recursion over 32 x 32 blocks ----
// LU without pivoting of A = [A11 A12; A21 A22] and both inverses:
//   A11 = L11 U11 (one warp), U12 = inv(L11) A12, L21 = A21 inv(U11),
//   A22 - L21 U12 = L22 U22 (one warp),
//   inv(L) = [inv(L11) 0; -inv(L22) L21 inv(L11)  inv(L22)],
//   inv(U) = [inv(U11)  -inv(U11) U12 inv(U22); 0 inv(U22)].
// Each 32 x 32 factorization is the one-pass scheme of diag_steps run by a
// single warp, lane r holding row r: no block barrier per step, and the
// coupling products run on all eight warps from shared memory (the two
// that need only the first block, L21 inv(L11) and inv(U11) U12, beside the
// second factorization).
constexpr int RB = NB / 2;       // 32
constexpr int kRecLd = RB + 1;   // row stride of the 32 x 32 shared-memory blocks (float2)
constexpr int kSmemDiagRec = (NB * (NB + 1) + 8 * RB * kRecLd + 2 * RB) * (int)sizeof(float2);

// One warp: LU and both inverses of the 32 x 32 block whose row `lane` is
// in a[0..31] (column c in a[c]), 32 rank-1 steps as in diag_steps: step j
// takes c_j = col_j / p_j (entry j zeroed) and applies
// a(r, c) -= c_j(r) a(j, c) to every column c != j, rows r > j only when
// c < j; column j becomes -c_j below the pivot. a(j, c) comes from lane j
// by shuffle. The steps run in groups of four over a register window that
// is rotated by four columns after each group (a[u] holds the group's
// column j0 + u, a[c] column (j0 + c) mod 32), so that every register index
// is static while the group loop stays rolled (the fully unrolled 32 steps
// would be ~9 k instructions of straight-line code). Ends with a[c] = column
// c: inv(L)(r, c) below the diagonal, the pivot p_r on it, S(r, c) =
// -p_r inv(U~)(r, c) above; rcps[j] = 1 / p_j (lane 0 writes).
__device__ __forceinline__ void leaf32(float2 (&a)[RB], int lane, float2* rcps, unsigned* err) {
    const float2 z = make_float2(0.f, 0.f);
#pragma unroll 1
    for (int j0 = 0; j0 < RB; j0 += 4) {
        const int rlim = RB - j0;  // a[c] holds a column right of the pivot iff u < c < rlim
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int j = j0 + u;
            const float2 piv = shfl_c(a[u], j);
            const float pm = piv.x * piv.x + piv.y * piv.y;
            const bool bad = !(pm > tiny_pivot(pm)) || !isfinite(pm);
            if (bad && lane == 0) atomicCAS(err, 0u, 1u);
            const float inv = bad ? 0.f : rcp_rn(pm);
            const float2 rcp = make_float2(piv.x * inv, -piv.y * inv);
            float2 cj = cmulf(a[u], rcp);
            if (lane == j) cj = z;
            const float2 cl = lane > j ? cj : z;
#pragma unroll
            for (int c = 0; c < RB; ++c) {
                if (c == u) continue;
                const float2 x = shfl_c(a[c], j);
                const float2 k = (c > u && c < rlim) ? cj : cl;
                a[c] = cfmsf(a[c], k, x);
            }
            a[u] = lane > j ? cnegf(cj) : a[u];
            if (lane == 0) rcps[j] = rcp;
        }
        const float2 t0 = a[0], t1 = a[1], t2 = a[2], t3 = a[3];
#pragma unroll
        for (int c = 0; c < RB - 4; ++c) a[c] = a[c + 4];
        a[RB - 4] = t0;
        a[RB - 3] = t1;
        a[RB - 2] = t2;
        a[RB - 1] = t3;
    }
    __syncwarp();
}

// Z = X Y (MODE 0), Z = -X Y (MODE 1) or Z -= X Y (MODE 2) for 32 x 32
// complex64 blocks in shared memory (row-major, strides ldx / ldy / ldz),
// by NT threads (t = 0 .. NT-1): thread t forms the entries of row t % 32
// in columns t / 32 + (NT / 32) i, k ascending, FP32 FMAs.
template <int NT, int MODE>
__device__ __forceinline__ void mm32(const float2* X, int ldx, const float2* Y, int ldy, float2* Z, int ldz,
                                     int t) {
    constexpr int E = RB * RB / NT;   // entries per thread
    constexpr int CS = NT / RB;       // column stride between them
    const int r = t % RB, c0 = t / RB;
    float2 acc[E];
#pragma unroll
    for (int i = 0; i < E; ++i) acc[i] = MODE == 2 ? Z[r * ldz + c0 + CS * i] : make_float2(0.f, 0.f);
    for (int k = 0; k < RB; ++k) {
        const float2 x = X[r * ldx + k];
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const float2 y = Y[k * ldy + c0 + CS * i];
            if (MODE == 2) acc[i] = cfmsf(acc[i], x, y);
            else acc[i] = make_float2(fmaf(x.x, y.x, fmaf(-x.y, y.y, acc[i].x)), fmaf(x.x, y.y, fmaf(x.y, y.x, acc[i].y)));
        }
    }
#pragma unroll
    for (int i = 0; i < E; ++i) Z[r * ldz + c0 + CS * i] = MODE == 1 ? cnegf(acc[i]) : acc[i];
}

// Writes the 32 x 32 inverses of the block leaf32 left in a (lane r = row
// r): IL = inv(L) (unit diagonal), IU = inv(U) = -S(r, c) / (p_r p_c) above
// the diagonal, 1 / p_r on it.
__device__ __forceinline__ void leaf32_store(const float2 (&a)[RB], int lane, const float2* rcps, float2* IL,
                                             float2* IU) {
    const float2 z = make_float2(0.f, 0.f), one = make_float2(1.f, 0.f);
    const float2 rr = rcps[lane];
#pragma unroll
    for (int c = 0; c < RB; ++c) {
        IL[lane * kRecLd + c] = c < lane ? a[c] : (c == lane ? one : z);
        IU[lane * kRecLd + c] = c > lane ? cnegf(cmulf(cmulf(a[c], rr), rcps[c])) : (c == lane ? rr : z);
    }
}

// Diagonal block k0 (kb rows and columns, padded to NB with the identity)
// by the 2 x 2 recursion above; writes Linv and Uinv (NB x NB column-major,
// zero outside kb) and reads the block of W only. The block's update by the
// previous step is done before (diag_update_kernel). A zero or non-finite
// pivot sets the error word and continues with a zero reciprocal.
__global__ void __launch_bounds__(256) diag_lu_rec_kernel(const float2* __restrict__ W, int64_t ldw, int64_t k0,
                                                          int kb, float2* __restrict__ Linv,
                                                          float2* __restrict__ Uinv, unsigned* __restrict__ err) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2* A = reinterpret_cast<float2*>(dyn_smem);  // NB x (NB + 1), row-major
    float2* blk = A + NB * (NB + 1);
    float2* IL1 = blk;
    float2* IU1 = blk + 1 * RB * kRecLd;
    float2* IL2 = blk + 2 * RB * kRecLd;
    float2* IU2 = blk + 3 * RB * kRecLd;
    float2* U12 = blk + 4 * RB * kRecLd;  // later -inv(U11) U12 inv(U22)
    float2* L21 = blk + 5 * RB * kRecLd;  // later -inv(L22) L21 inv(L11)
    float2* T1 = blk + 6 * RB * kRecLd;   // L21 inv(L11)
    float2* T2 = blk + 7 * RB * kRecLd;   // inv(U11) U12
    float2* rc1 = blk + 8 * RB * kRecLd;
    float2* rc2 = rc1 + RB;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    constexpr int LD = NB + 1;
    for (int e = tid; e < NB * NB; e += 256) {
        const int r = e % NB, c = e / NB;  // rows fastest: coalesced columns of W
        A[r * LD + c] = (r < kb && c < kb) ? W[(k0 + r) + (k0 + c) * ldw]
                                           : make_float2(r == c ? 1.f : 0.f, 0.f);
    }
    __syncthreads();
    if (w == 0) {
        float2 a[RB];
#pragma unroll
        for (int c = 0; c < RB; ++c) a[c] = A[lane * LD + c];
        leaf32(a, lane, rc1, err);
        leaf32_store(a, lane, rc1, IL1, IU1);
    }
    __syncthreads();
    if (w < 4) mm32<128, 0>(IL1, kRecLd, A + RB, LD, U12, kRecLd, tid);             // U12 = inv(L11) A12
    else mm32<128, 0>(A + RB * LD, LD, IU1, kRecLd, L21, kRecLd, tid - 128);         // L21 = A21 inv(U11)
    __syncthreads();
    mm32<256, 2>(L21, kRecLd, U12, kRecLd, A + RB * LD + RB, LD, tid);               // A22 -= L21 U12
    __syncthreads();
    if (w == 0) {
        float2 a[RB];
#pragma unroll
        for (int c = 0; c < RB; ++c) a[c] = A[(RB + lane) * LD + RB + c];
        leaf32(a, lane, rc2, err);
        leaf32_store(a, lane, rc2, IL2, IU2);
    } else if (w >= 4) {
        mm32<128, 0>(L21, kRecLd, IL1, kRecLd, T1, kRecLd, tid - 128);                // T1 = L21 inv(L11)
        mm32<128, 0>(IU1, kRecLd, U12, kRecLd, T2, kRecLd, tid - 128);                // T2 = inv(U11) U12
    }
    __syncthreads();
    if (w < 4) mm32<128, 1>(IL2, kRecLd, T1, kRecLd, L21, kRecLd, tid);              // -inv(L22) T1
    else mm32<128, 1>(T2, kRecLd, IU2, kRecLd, U12, kRecLd, tid - 128);              // -T2 inv(U22)
    __syncthreads();
    const float2 z = make_float2(0.f, 0.f);
    for (int e = tid; e < NB * NB; e += 256) {
        const int r = e % NB, c = e / NB;
        const bool in = r < kb && c < kb;
        const int rl = r % RB, cl = c % RB;
        float2 lv, uv;
        if (r < RB && c < RB) { lv = IL1[rl * kRecLd + cl]; uv = IU1[rl * kRecLd + cl]; }
        else if (r >= RB && c >= RB) { lv = IL2[rl * kRecLd + cl]; uv = IU2[rl * kRecLd + cl]; }
        else if (r >= RB) { lv = L21[rl * kRecLd + cl]; uv = z; }
        else { lv = z; uv = U12[rl * kRecLd + cl]; }
        Linv[r + c * NB] = in ? lv : z;
        Uinv[r + c * NB] = in ? uv : z;
    }
}

// The update of a diagonal block by the earlier block steps kp1 (and kp2,
// -1 = none), A11 -= L21(kp)[k0:k0+kb, :] U12(kp)[:, k0:k0+kb], in place in
// W, on 16 CTAs of 16 x 16 entries (one per thread, the k order and FP32
// FMAs of the update inside diag_lu_kernel, so the result is the same bit
// for bit). Run ahead of diag_lu_kernel it takes the product off that
// kernel's single SM: 64 x 64 x 64 complex FMAs are at least 4.2 us of FP32
// issue on one SM, here spread over 16.
template <class T>
__global__ void __launch_bounds__(256) diag_update_kernel(T* __restrict__ W, int64_t ldw, int64_t k0, int kb,
                                                          int64_t kp1, int64_t kp2) {
    __shared__ T Ls[NB][17];      // [k][row]
    __shared__ T Us[16][NB + 1];  // [col][k]
    const int tid = threadIdx.x;
    const int r = tid & 15, c = tid >> 4;
    const int row = 16 * blockIdx.x + r, col = 16 * blockIdx.y + c;
    const bool in = row < kb && col < kb;
    T a = in ? W[(k0 + row) + (k0 + col) * ldw] : cmk<T>(0.f, 0.f);
    for (int q = 0; q < 2; ++q) {
        const int64_t kp = q == 0 ? kp1 : kp2;
        if (kp < 0) continue;
        __syncthreads();  // the previous update's tiles are no longer read
        for (int e = tid; e < NB * 16; e += 256) {
            const int i = e & 15, kk = e >> 4;  // rows fastest: coalesced columns of L21
            const int gr = 16 * blockIdx.x + i;
            Ls[kk][i] = gr < kb ? W[(k0 + gr) + (kp + kk) * ldw] : cmk<T>(0.f, 0.f);
            const int kk2 = e % NB, j = e / NB;  // k fastest: coalesced columns of U12
            const int gc = 16 * blockIdx.y + j;
            Us[j][kk2] = gc < kb ? W[(kp + kk2) + (k0 + gc) * ldw] : cmk<T>(0.f, 0.f);
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < NB; ++kk) a = cfmsf(a, Ls[kk][r], Us[c][kk]);
    }
    if (in) W[(k0 + row) + (k0 + col) * ldw] = a;
}

// With kp1 >= 0 (and kp2 >= 0) the block first takes those earlier block
// steps' updates, A11 -= L21(kp)[k0:k0+kb, :] U12(kp)[:, k0:k0+kb] (FP32
// FMA), from the factor blocks staged in dynamic shared memory (kSmemDiagUpd;
// that size also keeps the kernel off SMs that hold a trailing-GEMM CTA).
// ELIM 0: diag_steps (one block barrier per step, fully unrolled per row
// half); 1: diag_panel (one named barrier per panel; the coefficient
// columns then live in the dynamic shared memory, after the update tiles
// are no longer read); 2: diag_steps_compact (as 0, one code path).
template <class T, int ELIM>
__global__ void __launch_bounds__(kDiagThreads) diag_lu_kernel(const T* __restrict__ W, int64_t ldw,
                                                               int64_t k0, int kb, T* __restrict__ Linv,
                                                               T* __restrict__ Uinv,
                                                               unsigned* __restrict__ err, int64_t kp1,
                                                               int64_t kp2) {
    constexpr int CW = kDiagCols;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ T cbuf[2][NB];  // c_j, double-buffered across the step barrier
    __shared__ T rcps[NB];     // 1 / p_j
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T a[CW][2];
#pragma unroll
    for (int v = 0; v < CW; ++v)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h, c = CW * w + v;
            a[v][h] = (r < kb && c < kb) ? W[(k0 + r) + (k0 + c) * ldw] : cmk<T>(r == c ? 1.f : 0.f, 0.f);
        }
    for (int q = 0; q < 2; ++q) {
        const int64_t kp = q == 0 ? kp1 : kp2;
        if (kp < 0) continue;
        T(*Ls)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(dyn_smem);           // [k][row]
        T(*Us)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(dyn_smem) + NB;      // [col][k]
        __syncthreads();  // the previous update's tiles are no longer read
        for (int e = threadIdx.x; e < NB * NB; e += kDiagThreads) {
            const int i = e % NB, q = e / NB;  // i fastest: coalesced columns of W
            Ls[q][i] = i < kb ? W[(k0 + i) + (kp + q) * ldw] : cmk<T>(0.f, 0.f);
            Us[q][i] = q < kb ? W[(kp + i) + (k0 + q) * ldw] : cmk<T>(0.f, 0.f);
        }
        __syncthreads();
        for (int kk = 0; kk < NB; ++kk) {
            const T l0 = Ls[kk][lane], l1 = Ls[kk][lane + 32];
#pragma unroll
            for (int v = 0; v < CW; ++v) {
                const T u = Us[CW * w + v][kk];
                a[v][0] = cfmsf(a[v][0], l0, u);
                a[v][1] = cfmsf(a[v][1], l1, u);
            }
        }
    }
    if (ELIM == 2) {
#pragma unroll 1
        for (int bp = 0; bp < kDiagWarps; ++bp)
            diag_steps_compact<T>(a, bp, bp >= kDiagWarps / 2 ? 1 : 0, w, lane, cbuf, rcps, err);
    } else if (ELIM == 1) {
        T(*cb)[NB] = reinterpret_cast<T(*)[NB]>(dyn_smem);
        __syncthreads();  // the update tiles are no longer read
#pragma unroll 1
        for (int p = 0; p < kDiagWarps / 2; ++p) diag_panel<T, 0>(a, p, w, lane, cb, rcps, err);
#pragma unroll 1
        for (int p = kDiagWarps / 2; p < kDiagWarps; ++p) diag_panel<T, 1>(a, p, w, lane, cb, rcps, err);
    } else {
#pragma unroll 1
        for (int bp = 0; bp < kDiagWarps / 2; ++bp) diag_steps<T, 0>(a, bp, w, lane, cbuf, rcps, err);
#pragma unroll 1
        for (int bp = kDiagWarps / 2; bp < kDiagWarps; ++bp) diag_steps<T, 1>(a, bp, w, lane, cbuf, rcps, err);
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < CW; ++v) {
        const int c = CW * w + v;
        const T rc = rcps[c];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h;
            const bool in = r < kb && c < kb;
            const T one = cmk<T>(1.f, 0.f), z = cmk<T>(0.f, 0.f);
            const T lv = r > c ? a[v][h] : (r == c ? one : z);
            const T uv = r < c ? cnegf(cmulf(cmulf(a[v][h], rcps[r]), rc)) : (r == c ? rc : z);
            Linv[r + c * NB] = in ? lv : z;
            Uinv[r + c * NB] = in ? uv : z;
        }
    }
}


template <class T>
using DiagKernel = void (*)(const T*, int64_t, int64_t, int, T*, T*, unsigned*, int64_t, int64_t);

// The elimination variant the switches select (diag_lu_kernel's ELIM).
template <class T>
static DiagKernel<T> diag_kernel_for(const MixedState* st) {
    if (st->diag_panels) return diag_lu_kernel<T, 1>;
    return st->diag_compact ? diag_lu_kernel<T, 2> : diag_lu_kernel<T, 0>;
}

template <class T>
static int diag_set_smem(int bytes) {
    for (DiagKernel<T> k : {diag_lu_kernel<T, 0>, diag_lu_kernel<T, 1>, diag_lu_kernel<T, 2>})
        SIEB_TRY_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    return SIEB200_OK;
}

// Arguments of one block step's panels launch.
//   kp[0], kp[1]: earlier block steps (column offsets, -1 = none) whose
//     updates the L rows take first; kpu: the step whose update the U
//     columns take first (the trailing GEMM runs every second step, so these
//     columns can lag one step behind);
//   Apack (at its K offset), a_ld (row stride in floats), a_r0 (first row
//     packed: pack row 2 (r - a_r0)); Bpack, b_ld, b_c0 likewise for columns;
//   a_lo, b_lo: offset of the lo part from the hi part in the split layout
//     [hi | lo] (0: the three-product layout [hi | hi | lo] / [hi | lo | hi]).
struct PanelArgs {
    int64_t k0 = 0, s0 = 0, np = 0;
    int kb = 0, nL = 0, pack = 0;
    int64_t kp[2] = {-1, -1};
    int64_t kpu = -1;
    float* Apack = nullptr;
    int64_t a_ld = 0, a_r0 = 0;
    float* Bpack = nullptr;
    int64_t b_ld = 0, b_c0 = 0;
    int64_t a_lo = 0, b_lo = 0;
    int lo_rn = 0;  // lo parts rounded to the nearest TF32
    // CTA range of one launch: L21 row blocks and U12 column blocks
    // [b_first, b_first + nl_run) of 32 each (nl_run 0: all nL from 0)
    int b_first = 0, nl_run = 0;
};

// L21 = A21 * inv(U11) for rows [s0, np) of the panel columns [k0, k0+kb);
// writes L21 back into W and the split realified rows into Apack.
// The rows first take the updates of the earlier steps in kp,
// A21 -= L21(kp) U12(kp)[:, k0:k0+kb] (FP32 FMA; the factors are those
// steps' panels in W), so no separate GEMM launch stands between the steps.
// One CTA per 32 rows. Thread (ty, tx) computes rows 2ty, 2ty+1 and columns
// 2tx, 2tx+1, 62-2tx, 63-2tx with k outermost; inv(U11) is upper
// triangular, so each column pair's k loop stops at its last column.
template <class T>
__device__ __forceinline__ void panel_L_body(T* __restrict__ W, int64_t ldw, const PanelArgs& pa,
                                             const T* __restrict__ Uinv, int bx) {
    const int64_t k0 = pa.k0, r0 = pa.s0, np = pa.np;
    const int kb = pa.kb;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    T(*Us)[NB + 4] = reinterpret_cast<T(*)[NB + 4]>(dyn_smem);                       // [k][c]
    T(*Ar)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(dyn_smem + NB * (NB + 4) * sizeof(T));   // [row][k]
    T(*Lr)[NB + 1] = Ar + 32;                                                             // [row][k]
    const int tid = threadIdx.x;
    const int64_t rb = r0 + (int64_t)bx * 32;
    // All of this thread's loads go out before the first shared-memory store
    // (one memory latency per CTA instead of one per loop trip): its A21
    // entries and, in complex64, its entries of inv(U11), which stay in
    // registers until the update phase no longer needs Us.
    // (complex128, the own FP64 LU: the plain loop, which needs no spill)
    constexpr bool kPre = std::is_same<T, float2>::value;
    T ui[kPre ? kPanelInv : 1];
    if constexpr (kPre) {
        T ra[kPanelSlab];
#pragma unroll
        for (int i = 0; i < kPanelSlab; ++i) {
            const int e = tid + kPanelThreads * i;
            const int r = e % 32, c = e / 32;
            const int64_t gr = rb + r;
            ra[i] = (gr < np && c < kb) ? W[gr + (k0 + c) * ldw] : cmk<T>(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < kPanelInv; ++i) ui[i] = Uinv[tid + kPanelThreads * i];
#pragma unroll
        for (int i = 0; i < kPanelSlab; ++i) {
            const int e = tid + kPanelThreads * i;
            Ar[e % 32][e / 32] = ra[i];
        }
    } else {
        for (int e = tid; e < 32 * NB; e += blockDim.x) {
            const int r = e % 32, c = e / 32;
            const int64_t gr = rb + r;
            Ar[r][c] = (gr < np && c < kb) ? W[gr + (k0 + c) * ldw] : cmk<T>(0.f, 0.f);
        }
    }
    const int ty = tid & 15, tx = tid >> 4;
    for (int q = 0; q < 2; ++q) {
        const int64_t kp = pa.kp[q];
        if (kp < 0) continue;
        for (int e = tid; e < NB * NB; e += blockDim.x) {
            const int kk = e % NB, c = e / NB;
            Us[kk][c] = c < kb ? W[(kp + kk) + (k0 + c) * ldw] : cmk<T>(0.f, 0.f);
        }
        for (int e = tid; e < 32 * NB; e += blockDim.x) {
            const int r = e % 32, kk = e / 32;
            const int64_t gr = rb + r;
            Lr[r][kk] = gr < np ? W[gr + (kp + kk) * ldw] : cmk<T>(0.f, 0.f);
        }
        __syncthreads();
        T upd[2][4];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) upd[i][j] = Ar[2 * ty + i][4 * tx + j];
        for (int kk = 0; kk < NB; ++kk) {
            const T l0 = Lr[2 * ty][kk], l1 = Lr[2 * ty + 1][kk];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const T u = Us[kk][4 * tx + j];
                upd[0][j] = cfmsf(upd[0][j], l0, u);
                upd[1][j] = cfmsf(upd[1][j], l1, u);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) Ar[2 * ty + i][4 * tx + j] = upd[i][j];
    }
    if constexpr (kPre) {
#pragma unroll
        for (int i = 0; i < kPanelInv; ++i) {
            const int e = tid + kPanelThreads * i;
            Us[e % NB][e / NB] = ui[i];  // Uinv[k + c*NB]
        }
    } else {
        for (int e = tid; e < NB * NB; e += blockDim.x) Us[e % NB][e / NB] = Uinv[e];
    }
    __syncthreads();
    // Columns of thread tx: the pair 2tx, 2tx+1 and the pair 62-2tx, 63-2tx,
    // so that every warp runs about the same number of k steps of the
    // triangle (2tx+2 with all four columns, then up to 64-2tx with the high
    // pair) instead of the last warps running all 64 while the first wait at
    // the barrier. Each column still sums its k in ascending order.
    T acc[2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = cmk<T>(0.f, 0.f);
    int col[4];
    col[0] = 2 * tx; col[1] = 2 * tx + 1; col[2] = 62 - 2 * tx; col[3] = 63 - 2 * tx;
    const int kend_lo = min(kb, 2 * tx + 2), kend_hi = min(kb, 64 - 2 * tx);
    for (int k = 0; k < kend_lo; ++k) {
        const T a0 = Ar[2 * ty][k], a1 = Ar[2 * ty + 1][k];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const T u = Us[k][col[j]];
            acc[0][j] = cmk<T>(acc[0][j].x + a0.x * u.x - a0.y * u.y, acc[0][j].y + a0.x * u.y + a0.y * u.x);
            acc[1][j] = cmk<T>(acc[1][j].x + a1.x * u.x - a1.y * u.y, acc[1][j].y + a1.x * u.y + a1.y * u.x);
        }
    }
    for (int k = kend_lo; k < kend_hi; ++k) {
        const T a0 = Ar[2 * ty][k], a1 = Ar[2 * ty + 1][k];
#pragma unroll
        for (int j = 2; j < 4; ++j) {
            const T u = Us[k][col[j]];
            acc[0][j] = cmk<T>(acc[0][j].x + a0.x * u.x - a0.y * u.y, acc[0][j].y + a0.x * u.y + a0.y * u.x);
            acc[1][j] = cmk<T>(acc[1][j].x + a1.x * u.x - a1.y * u.y, acc[1][j].y + a1.x * u.y + a1.y * u.x);
        }
    }
    __syncthreads();
    // ... back through shared memory ...
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) Ar[2 * ty + i][col[j]] = acc[i][j];
    __syncthreads();
    // ... to W (rows fastest: coalesced columns) ...
    for (int e = tid; e < 32 * kb; e += blockDim.x) {
        const int rr = e % 32, c = e / 32;
        const int64_t gr = rb + rr;
        if (gr < np) W[gr + (k0 + c) * ldw] = Ar[rr][c];
    }
    if constexpr (!std::is_same<T, float2>::value) return;
    if (!pa.pack) return;
    // ... and to the split realified rows (K fastest: coalesced rows).
    // row 2i: [Re, -Im] per column, row 2i+1: [Im, Re]; layout [hi | hi | lo].
    for (int e = tid; e < 32 * 2 * NB; e += blockDim.x) {
        const int rr = e / (2 * NB), kk = e % (2 * NB);
        const int64_t gr = rb + rr;
        if (gr >= np || gr < pa.a_r0) continue;
        const int c = kk >> 1, h = kk & 1;
        const T v = Ar[rr][c];
        const float v0 = h == 0 ? v.x : -v.y;   // real row
        const float v1 = h == 0 ? v.y : v.x;    // imaginary row
        const float h0 = tf32_hi(v0), h1 = tf32_hi(v1);
        float* row0 = pa.Apack + (2 * (gr - pa.a_r0)) * pa.a_ld;
        float* row1 = row0 + pa.a_ld;
        const float l0 = tf32_lo(v0, h0, pa.lo_rn), l1 = tf32_lo(v1, h1, pa.lo_rn);
        if (pa.a_lo) {
            row0[kk] = h0; row0[pa.a_lo + kk] = l0;
            row1[kk] = h1; row1[pa.a_lo + kk] = l1;
        } else {
            row0[kk] = h0; row0[2 * NB + kk] = h0; row0[4 * NB + kk] = l0;
            row1[kk] = h1; row1[2 * NB + kk] = h1; row1[4 * NB + kk] = l1;
        }
    }
}

// U12 = inv(L11) * A12 for columns [s0, np) of the panel rows [k0, k0+kb);
// writes U12 back into W and the split columns into Bpack. With kpu >= 0 the
// columns first take that step's update, A12 -= L21(kpu)[k0:k0+kb, :]
// U12(kpu)[:, these columns] (FP32 FMA, both factors from W). One CTA per 32
// columns. Thread (ty, tx) computes rows 2ty, 2ty+1, 62-2ty, 63-2ty and
// columns 2tx, 2tx+1 with k outermost; inv(L11) is lower triangular, so each
// row pair's k loop stops at its last row.
template <class T>
__device__ __forceinline__ void panel_U_body(T* __restrict__ W, int64_t ldw, const PanelArgs& pa,
                                             const T* __restrict__ Linv, int bx) {
    const int64_t k0 = pa.k0, c0 = pa.s0, np = pa.np;
    const int kb = pa.kb;
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    T(*Ls)[NB + 4] = reinterpret_cast<T(*)[NB + 4]>(dyn_smem);                       // [k][r]
    T(*Ac)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(dyn_smem + NB * (NB + 4) * sizeof(T));   // [col][k]
    T(*Uc)[NB + 1] = Ac + 32;                                                           // [col][k]
    const int tid = threadIdx.x;
    const int64_t cb = c0 + (int64_t)bx * 32;
    // As in panel_L_body: every load of the thread before the first store.
    constexpr bool kPre = std::is_same<T, float2>::value;
    T li[kPre ? kPanelInv : 1];
    if constexpr (kPre) {
        T ra[kPanelSlab];
#pragma unroll
        for (int i = 0; i < kPanelSlab; ++i) {
            const int e = tid + kPanelThreads * i;
            const int r = e % NB, c = e / NB;
            const int64_t gc = cb + c;
            ra[i] = (gc < np && r < kb) ? W[(k0 + r) + gc * ldw] : cmk<T>(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < kPanelInv; ++i) li[i] = Linv[tid + kPanelThreads * i];
#pragma unroll
        for (int i = 0; i < kPanelSlab; ++i) {
            const int e = tid + kPanelThreads * i;
            Ac[e / NB][e % NB] = ra[i];
        }
    } else {
        for (int e = tid; e < 32 * NB; e += blockDim.x) {
            const int r = e % NB, c = e / NB;
            const int64_t gc = cb + c;
            Ac[c][r] = (gc < np && r < kb) ? W[(k0 + r) + gc * ldw] : cmk<T>(0.f, 0.f);
        }
    }
    const int tx = tid & 15, ty = tid >> 4;
    if (pa.kpu >= 0) {
        const int64_t kp = pa.kpu;
        // L21(kp) rows of this block as Ls[r][kk], U12(kp) columns as Uc[c][kk]
        for (int e = tid; e < NB * NB; e += blockDim.x) {
            const int r = e % NB, kk = e / NB;
            Ls[r][kk] = r < kb ? W[(k0 + r) + (kp + kk) * ldw] : cmk<T>(0.f, 0.f);
        }
        for (int e = tid; e < 32 * NB; e += blockDim.x) {
            const int kk = e % NB, c = e / NB;
            const int64_t gc = cb + c;
            Uc[c][kk] = gc < np ? W[(kp + kk) + gc * ldw] : cmk<T>(0.f, 0.f);
        }
        __syncthreads();
        T upd[4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) upd[i][j] = Ac[2 * tx + j][4 * ty + i];
        for (int kk = 0; kk < NB; ++kk) {
            const T u0 = Uc[2 * tx][kk], u1 = Uc[2 * tx + 1][kk];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const T l = Ls[4 * ty + i][kk];
                upd[i][0] = cfmsf(upd[i][0], l, u0);
                upd[i][1] = cfmsf(upd[i][1], l, u1);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 2; ++j) Ac[2 * tx + j][4 * ty + i] = upd[i][j];
    }
    if constexpr (kPre) {
#pragma unroll
        for (int i = 0; i < kPanelInv; ++i) {
            const int e = tid + kPanelThreads * i;
            Ls[e / NB][e % NB] = li[i];  // Linv[r + k*NB]
        }
    } else {
        for (int e = tid; e < NB * NB; e += blockDim.x) Ls[e / NB][e % NB] = Linv[e];
    }
    __syncthreads();
    // Rows of thread ty: the pairs 2ty, 2ty+1 and 62-2ty, 63-2ty (balanced
    // triangle, as the columns in panel_L_body), each summed in ascending k.
    T acc[4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j] = cmk<T>(0.f, 0.f);
    int row[4];
    row[0] = 2 * ty; row[1] = 2 * ty + 1; row[2] = 62 - 2 * ty; row[3] = 63 - 2 * ty;
    const int kend_lo = min(kb, 2 * ty + 2), kend_hi = min(kb, 64 - 2 * ty);
    for (int k = 0; k < kend_lo; ++k) {
        const T b0 = Ac[2 * tx][k], b1 = Ac[2 * tx + 1][k];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const T l = Ls[k][row[i]];
            acc[i][0] = cmk<T>(acc[i][0].x + l.x * b0.x - l.y * b0.y, acc[i][0].y + l.x * b0.y + l.y * b0.x);
            acc[i][1] = cmk<T>(acc[i][1].x + l.x * b1.x - l.y * b1.y, acc[i][1].y + l.x * b1.y + l.y * b1.x);
        }
    }
    for (int k = kend_lo; k < kend_hi; ++k) {
        const T b0 = Ac[2 * tx][k], b1 = Ac[2 * tx + 1][k];
#pragma unroll
        for (int i = 2; i < 4; ++i) {
            const T l = Ls[k][row[i]];
            acc[i][0] = cmk<T>(acc[i][0].x + l.x * b0.x - l.y * b0.y, acc[i][0].y + l.x * b0.y + l.y * b0.x);
            acc[i][1] = cmk<T>(acc[i][1].x + l.x * b1.x - l.y * b1.y, acc[i][1].y + l.x * b1.y + l.y * b1.x);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) Ac[2 * tx + j][row[i]] = acc[i][j];
    __syncthreads();
    for (int e = tid; e < 32 * NB; e += blockDim.x) {
        const int r = e % NB, c = e / NB;
        const int64_t gc = cb + c;
        if (gc >= np) continue;
        const T v = Ac[c][r];
        if (r < kb) W[(k0 + r) + gc * ldw] = v;
        if (std::is_same<T, float2>::value && pa.pack && gc >= pa.b_c0) {
            float* col = pa.Bpack + (gc - pa.b_c0) * pa.b_ld;
            const float h0 = tf32_hi(v.x), h1 = tf32_hi(v.y);
            const float l0 = tf32_lo(v.x, h0, pa.lo_rn), l1 = tf32_lo(v.y, h1, pa.lo_rn);
            col[2 * r] = h0; col[2 * r + 1] = h1;
            if (pa.b_lo) {
                col[pa.b_lo + 2 * r] = l0; col[pa.b_lo + 2 * r + 1] = l1;
            } else {
                col[2 * NB + 2 * r] = l0; col[2 * NB + 2 * r + 1] = l1;
                col[4 * NB + 2 * r] = h0; col[4 * NB + 2 * r + 1] = h1;
            }
        }
    }
}

// Rows [r0, np) of block column k0 (kb columns) take the update of step kp,
// A21 -= L21(kp)[rows, :] U12(kp)[:, k0:k0+kb], written back to W: the FP32
// FMAs of panel_L_body's update in the same order (same results), ahead of
// a panels launch that then only forms L21 = A21 inv(U11). One CTA per 32
// rows, thread (ty, tx) rows 2ty, 2ty+1 and columns 4tx .. 4tx+3 as there;
// the K range is staged in two halves so that the shared memory (25.8 KB)
// leaves a CTA room beside a trailing-GEMM CTA on its SM.
constexpr int kColUpdK = NB / 2;
__global__ void __launch_bounds__(256) col_update_kernel(float2* __restrict__ W, int64_t ldw, int64_t k0, int kb,
                                                         int64_t r0, int64_t np, int64_t kp) {
    __shared__ float2 Us[kColUpdK][NB + 4];  // [k][c]
    __shared__ float2 Lr[32][kColUpdK + 1];  // [row][k]
    const int tid = threadIdx.x;
    const int ty = tid & 15, tx = tid >> 4;
    const int64_t rb = r0 + (int64_t)blockIdx.x * 32;
    float2 upd[2][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t gr = rb + 2 * ty + i;
            const int c = 4 * tx + j;
            upd[i][j] = (gr < np && c < kb) ? W[gr + (k0 + c) * ldw] : make_float2(0.f, 0.f);
        }
    for (int h = 0; h < NB; h += kColUpdK) {
        __syncthreads();  // the previous half is no longer read
        for (int e = tid; e < kColUpdK * NB; e += blockDim.x) {
            const int kk = e % kColUpdK, c = e / kColUpdK;  // k fastest: coalesced columns of U12
            Us[kk][c] = c < kb ? W[(kp + h + kk) + (k0 + c) * ldw] : make_float2(0.f, 0.f);
        }
        for (int e = tid; e < 32 * kColUpdK; e += blockDim.x) {
            const int r = e % 32, kk = e / 32;  // rows fastest: coalesced columns of L21
            const int64_t gr = rb + r;
            Lr[r][kk] = gr < np ? W[gr + (kp + h + kk) * ldw] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        for (int kk = 0; kk < kColUpdK; ++kk) {
            const float2 l0 = Lr[2 * ty][kk], l1 = Lr[2 * ty + 1][kk];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 u = Us[kk][4 * tx + j];
                upd[0][j] = cfmsf(upd[0][j], l0, u);
                upd[1][j] = cfmsf(upd[1][j], l1, u);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t gr = rb + 2 * ty + i;
            const int c = 4 * tx + j;
            if (gr < np && c < kb) W[gr + (k0 + c) * ldw] = upd[i][j];
        }
}

// Both panels of a block step in one launch: the first nl_run CTAs form
// L21 (rows below the diagonal block, after the updates of the steps in kp),
// the rest U12 (columns right of it, after the update of step kpu), both
// over the 32-row (32-column) blocks from b_first. A block's result does
// not depend on the launch it runs in, so the panels can be split between
// launches (the next block's rows and columns first) bit for bit.
template <class T>
__global__ void __launch_bounds__(256, 3) panels_kernel(T* __restrict__ W, int64_t ldw, const T* __restrict__ Uinv,
                                                        const T* __restrict__ Linv, const PanelArgs pa) {
    const int nl = pa.nl_run > 0 ? pa.nl_run : pa.nL;
    if ((int)blockIdx.x < nl) panel_L_body(W, ldw, pa, Uinv, pa.b_first + (int)blockIdx.x);
    else panel_U_body(W, ldw, pa, Linv, pa.b_first + (int)blockIdx.x - nl);
}

// SIMT trailing update C -= L21 U12 in complex64 (checking path).
__global__ void __launch_bounds__(256) trailing_simt_kernel(float2* __restrict__ W, int64_t ldw,
                                                            int64_t k0, int kb, int64_t s0, int64_t np) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2(*Ls)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn_smem);        // [row][k]
    float2(*Us)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn_smem) + 64;   // [col][k]
    const int64_t rb = s0 + (int64_t)blockIdx.x * 64, cb = s0 + (int64_t)blockIdx.y * 64;
    const int tid = threadIdx.x;
    for (int e = tid; e < 64 * kb; e += blockDim.x) {
        const int r = e % 64, k = e / 64;
        Ls[r][k] = rb + r < np ? W[(rb + r) + (k0 + k) * ldw] : make_float2(0.f, 0.f);
        const int c = e % 64, kk = e / 64;
        Us[c][kk] = cb + c < np ? W[(k0 + kk) + (cb + c) * ldw] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int e = tid; e < 64 * 64; e += blockDim.x) {
        const int r = e % 64, c = e / 64;
        if (rb + r >= np || cb + c >= np) continue;
        float2 acc = make_float2(0.f, 0.f);
        for (int k = 0; k < kb; ++k) {
            acc.x += Ls[r][k].x * Us[c][k].x - Ls[r][k].y * Us[c][k].y;
            acc.y += Ls[r][k].x * Us[c][k].y + Ls[r][k].y * Us[c][k].x;
        }
        float2& w = W[(rb + r) + (cb + c) * ldw];
        w = make_float2(w.x - acc.x, w.y - acc.y);
    }
}

// ------------------------------------------------------------ triangular solves
// Published solution entries: every 8-byte word of the publication buffer
// starts as all ones (a NaN payload arithmetic does not produce) and is
// written once; each word is single-copy atomic, so an entry whose two
// words both differ from it is complete.
__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ bool unpublished(double v) { return __double_as_longlong(v) == -1ll; }

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Blocked forward (lower = 1) or backward solve on the factors, in place in
// x (np entries), FP64 arithmetic on the complex64 factors.
//
// One CTA per 128-row block (two NB sub-blocks), taken in solve order by
// ticket. Warp 8 streams the CTA's factor tiles (128 rows x 32 columns,
// 32 KB) by TMA into a 4-stage shared-memory ring, in the order in which
// their x entries are published, independently of that publication; warps
// 0-7 wait (one poller per warp) until the sub-block a tile multiplies has
// been published, then accumulate. The two diagonal sub-blocks are solved
// inside the CTA: the first with its explicit inverse, published at once,
// then the coupling block and the second inverse.
//
// A solved sub-block is published by writing its entries into xpub (all
// ones beforehand, set by the host), which consumers poll entry by entry;
// progress[0] also counts published sub-blocks; progress[1] is the ticket
// counter; both cleared by the host. A CTA waits only for CTAs with
// smaller tickets, which are already running. Every wait is bounded by
// timeout_ns from the CTA's start; on timeout the error word is set, the CTA
// still consumes every tile its producer issues (so no copy is in flight at
// exit) and returns without publishing.
constexpr int TR_ROWS = 2 * NB;       // rows per CTA
constexpr int TR_COLS = 32;           // columns per streamed tile
constexpr int TR_STAGES = 4;
constexpr int TR_TILE = TR_ROWS * TR_COLS;           // float2 per tile
constexpr int TR_TILE_BYTES = TR_TILE * 8;           // 32 KB
constexpr int TR_DLD = NB + 4;        // staged inverses [col][row]: conflict-free half-warps
constexpr int TR_CONSUMERS = 256;
constexpr int TR_THREADS = TR_CONSUMERS + 32;
constexpr int kSmemTrsv = 1024 + TR_STAGES * TR_TILE_BYTES + 2 * NB * TR_DLD * 8 +
                          (2 * TR_ROWS + 3 * NB) * (int)sizeof(cplx) + 2 * TR_STAGES * 8;
// Stages of the tile ring for CTAs of `rows` rows (32 KB tiles of 128 rows,
// 16 KB tiles of 64) and the shared memory of that variant.
__host__ __device__ constexpr int tr_stages(int rows) { return rows == 2 * NB ? TR_STAGES : 8; }
__host__ __device__ constexpr int trsv_smem(int rows) {
    return 1024 + tr_stages(rows) * rows * TR_COLS * 8 + (rows / NB) * NB * TR_DLD * 8 +
           ((TR_CONSUMERS / rows - 1) * rows + rows + 3 * NB) * (int)sizeof(cplx) + 2 * tr_stages(rows) * 8;
}
static_assert(trsv_smem(2 * NB) == kSmemTrsv, "128-row layout");

__device__ __forceinline__ void consumer_bar() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// Bounded mbarrier wait; false once the deadline has passed.
__device__ __forceinline__ bool tr_wait(uint32_t bar, uint32_t parity, uint64_t deadline) {
    int it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if ((++it & 255) == 0 && global_ns() > deadline) return false;
    }
    return true;
}

template <int ROWS>
__global__ void __launch_bounds__(TR_THREADS, 1)
trsv_tma_kernel(const __grid_constant__ CUtensorMap tmW, int64_t np, int nsb, int lower,
                const float2* __restrict__ Dinv, cplx* __restrict__ x, cplx* __restrict__ xpub,
                unsigned* __restrict__ progress, unsigned* __restrict__ err, unsigned long long timeout_ns) {
    constexpr int SUBS = ROWS / NB;                 // diagonal sub-blocks per CTA (1 or 2)
    constexpr int HG = TR_CONSUMERS / ROWS;         // consumer threads per row
    constexpr int CPT = TR_COLS / HG;               // tile columns per consumer thread
    constexpr int STG = tr_stages(ROWS);
    constexpr int TILE = ROWS * TR_COLS;            // float2 per tile
    constexpr int TILE_BYTES = TILE * 8;
    extern __shared__ __align__(16) unsigned char dyn_smem[];  // aligned to 1024 below
    const uint32_t raw = smem_u32(dyn_smem);
    unsigned char* base = dyn_smem + (((raw + 1023u) & ~1023u) - raw);
    const uint32_t ring = smem_u32(base);
    const float2* ringp = reinterpret_cast<const float2*>(base);
    float2* Ds = reinterpret_cast<float2*>(base + STG * TILE_BYTES);  // SUBS x [NB cols][TR_DLD]
    cplx* red = reinterpret_cast<cplx*>(Ds + SUBS * NB * TR_DLD);              // (HG - 1) x ROWS
    cplx* ys = red + (HG - 1) * ROWS;                                           // ROWS
    cplx* xs = ys + ROWS;                                                       // NB
    cplx* xstage = xs + NB;                                                        // 2 x NB
    const uint32_t full0 = smem_u32(xstage + 2 * NB), empty0 = full0 + 8 * STG;
    __shared__ int s_t, s_go;
    __shared__ volatile int s_abort;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        s_t = (int)atomicAdd(&progress[1], 1u);
        s_abort = 0;
        for (int st = 0; st < STG; ++st) {
            mbar_init(full0 + 8 * st, 1);
            mbar_init(empty0 + 8 * st, TR_CONSUMERS / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const uint64_t deadline = global_ns() + timeout_ns;
    const int ncta = (int)((np + ROWS - 1) / ROWS);
    const int t = s_t;
    if (t >= ncta) return;  // block-uniform
    const int rb = lower ? t : ncta - 1 - t;
    const int64_t R0 = (int64_t)rb * ROWS;
    const int sbA = SUBS * rb, sbB = SUBS * rb + 1;
    const bool has_bot = SUBS == 2 && sbB < nsb;
    // Streamed tiles: the off-diagonal ones in publication order, then the
    // two tiles holding the coupling block between the sub-blocks.
    const int ntile_all = (int)((np + TR_COLS - 1) / TR_COLS);
    int n_off;
    if (lower) {
        n_off = (int)(R0 / TR_COLS);
    } else {
        const int kmin = (int)((R0 + ROWS) / TR_COLS);
        n_off = ntile_all > kmin ? ntile_all - kmin : 0;
    }
    const int n_tiles = n_off + (has_bot ? 2 : 0);
    const int k_intra = (int)((lower ? R0 : R0 + NB) / TR_COLS);
    auto tile_k = [&](int i) -> int {
        if (i < n_off) return lower ? i : ntile_all - 1 - i;
        return k_intra + (i - n_off);
    };

    if (warp == TR_CONSUMERS / 32) {  // producer
        if (lane == 0) {
            for (int i = 0; i < n_tiles; ++i) {
                const int st = i % STG;
                const uint32_t ph = (uint32_t)(i / STG) & 1u;
                if (!tr_wait(empty0 + 8 * st, ph ^ 1u, deadline)) {
                    atomicCAS(err, 0u, 2u);
                    s_abort = 1;
                    break;
                }
                mbar_expect_tx(full0 + 8 * st, TILE_BYTES);
                tma_load_2d(ring + st * TILE_BYTES, &tmW, full0 + 8 * st, (int)R0, tile_k(i) * TR_COLS);
            }
        }
        return;
    }

    // Consumers. Inverses of the two diagonal sub-blocks into shared memory.
    for (int e = tid; e < NB * NB; e += TR_CONSUMERS) {
        const int r = e & (NB - 1), c = e >> 6;
        Ds[c * TR_DLD + r] = Dinv[(size_t)sbA * NB * NB + e];
        if (SUBS == 2)
            Ds[(NB + c) * TR_DLD + r] = has_bot ? Dinv[(size_t)sbB * NB * NB + e] : make_float2(0.f, 0.f);
    }
    // Thread (r, h): row r of the block, columns h*CPT .. h*CPT+CPT-1 of a tile.
    const int r = tid & (ROWS - 1), h = tid / ROWS;
    const int64_t grow = R0 + r;
    cplx b = cx(0, 0);  // written only by this CTA: final from the start
    if (h == 0 && grow < np) b = cx(__ldcg(&x[grow].re), __ldcg(&x[grow].im));
    double acc_re = 0.0, acc_im = 0.0;
    // Off-diagonal tiles in groups of one NB sub-block (two tiles, or one at
    // a ragged end): warp 0 waits until the sub-block is published and
    // stages its NB x entries in shared memory (double-buffered by group
    // parity), so both tiles cost one L2 round trip; one consumer barrier
    // per group hands them to all warps.
    for (int i = 0, g = 0; i < n_off; ++g) {
        const int sb = (tile_k(i) * TR_COLS) / NB;
        const int cnt = (i + 1 < n_off && (tile_k(i + 1) * TR_COLS) / NB == sb) ? 2 : 1;
        cplx* xg = xstage + (g & 1) * NB;
        if (warp == 0) {
            // Each lane polls its two entries of the sub-block (lane, lane +
            // 32) in the publication buffer, both in every round: the value is
            // the flag, one L2 round trip per round for all 64 entries.
            static_assert(NB == 64, "two entries per lane");
            const int64_t c0 = (int64_t)sb * NB + lane, c1 = c0 + 32;
            bool need0 = c0 < np, need1 = c1 < np;
            cplx v0 = cx(0, 0), v1 = cx(0, 0);
            bool okp = !s_abort;
            int it = 0;
            while (okp && (need0 || need1)) {
                double r0 = 0, i0 = 0, r1 = 0, i1 = 0;
                if (need0) { r0 = ld_relaxed_f64(&xpub[c0].re); i0 = ld_relaxed_f64(&xpub[c0].im); }
                if (need1) { r1 = ld_relaxed_f64(&xpub[c1].re); i1 = ld_relaxed_f64(&xpub[c1].im); }
                if (need0 && !unpublished(r0) && !unpublished(i0)) { v0 = cx(r0, i0); need0 = false; }
                if (need1 && !unpublished(r1) && !unpublished(i1)) { v1 = cx(r1, i1); need1 = false; }
                if (!need0 && !need1) break;
                if (++it > 16) __nanosleep(64);
                if ((it & 63) == 0 &&
                    (s_abort || global_ns() > deadline || *reinterpret_cast<volatile unsigned*>(err))) {
                    atomicCAS(err, 0u, 2u);
                    s_abort = 1;
                    okp = false;
                }
            }
            xg[lane] = v0;
            xg[lane + 32] = v1;
            __syncwarp();
        }
        consumer_bar();
        for (int j = 0; j < cnt; ++j, ++i) {
            const int st = i % STG;
            const uint32_t ph = (uint32_t)(i / STG) & 1u;
            // Every issued tile is waited for and released, also after an
            // abort, so that no copy is in flight when the CTA exits.
            bool ok = !s_abort;
            if (!tr_wait(full0 + 8 * st, ph, deadline)) {
                if (lane == 0) atomicCAS(err, 0u, 2u);
                s_abort = 1;
                ok = false;
            }
            if (ok) {
                const float2* tile = ringp + st * TILE;
                const cplx* xt = xg + (tile_k(i) * TR_COLS - sb * NB) + h * CPT;
#pragma unroll
                for (int u = 0; u < CPT; ++u) {
                    const float2 w = tile[(h * CPT + u) * ROWS + r];
                    const cplx xv = xt[u];
                    acc_re += (double)w.x * xv.re - (double)w.y * xv.im;
                    acc_im += (double)w.x * xv.im + (double)w.y * xv.re;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * st);
        }
    }
    if (h >= 1) red[(h - 1) * ROWS + r] = cx(acc_re, acc_im);
    consumer_bar();
    if (h == 0) {
#pragma unroll
        for (int g2 = 0; g2 < HG - 1; ++g2) {
            acc_re += red[g2 * ROWS + r].re;
            acc_im += red[g2 * ROWS + r].im;
        }
        ys[r] = cx(b.re - acc_re, b.im - acc_im);
    }
    if (tid == 0) s_go = !s_abort;
    consumer_bar();
    if (!s_go) return;  // block-uniform

    // Diagonal phase. Thread (dr, part): row dr of a sub-block, columns part + 4u.
    const int dr = tid >> 2, part = tid & 3;
    auto solve_sub = [&](int which) {
        const float2* D = Ds + which * NB * TR_DLD;
        const cplx* y = ys + which * NB;
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int u = 0; u < NB / 4; ++u) {
            const int c = part + 4 * u;
            const float2 d = D[c * TR_DLD + dr];
            const cplx yv = y[c];
            re += (double)d.x * yv.re - (double)d.y * yv.im;
            im += (double)d.x * yv.im + (double)d.y * yv.re;
        }
        re += __shfl_xor_sync(0xffffffffu, re, 1);
        im += __shfl_xor_sync(0xffffffffu, im, 1);
        re += __shfl_xor_sync(0xffffffffu, re, 2);
        im += __shfl_xor_sync(0xffffffffu, im, 2);
        const int64_t gr = R0 + which * NB + dr;
        if (part == 0) {
            xs[dr] = cx(re, im);
            if (gr < np) {
                __stcg(&x[gr].re, re);
                __stcg(&x[gr].im, im);
                __stcg(&xpub[gr].re, re);
                __stcg(&xpub[gr].im, im);
            }
        }
        // The barrier orders every store of the sub-block before the release.
        consumer_bar();
        const int sb = which ? sbB : sbA;
        if (tid == 0) st_release_gpu(&progress[0], lower ? (unsigned)sb + 1u : (unsigned)(nsb - sb));
    };
    if (!has_bot) {
        solve_sub(0);
        return;
    }
    const int first = lower ? 0 : 1, second = 1 - first;
    solve_sub(first);
    // Coupling block: rows of `second` x columns of `first`, in the last two tiles.
    bool ok = true;
    for (int j = 0; j < 2; ++j) {
        const int i = n_off + j;
        ok = tr_wait(full0 + 8 * (i % STG), (uint32_t)(i / STG) & 1u, deadline) && ok;
    }
    if (!ok && tid == 0) atomicCAS(err, 0u, 2u);
    const int roff = second * NB;
    double re = 0.0, im = 0.0;
    if (ok) {
#pragma unroll
        for (int u = 0; u < NB / 4; ++u) {
            const int c = part + 4 * u;
            const float2* tile = ringp + ((n_off + (c >> 5)) % STG) * TILE;
            const float2 w = tile[(c & 31) * ROWS + roff + dr];
            const cplx xv = xs[c];
            re += (double)w.x * xv.re - (double)w.y * xv.im;
            im += (double)w.x * xv.im + (double)w.y * xv.re;
        }
    }
    re += __shfl_xor_sync(0xffffffffu, re, 1);
    im += __shfl_xor_sync(0xffffffffu, im, 1);
    re += __shfl_xor_sync(0xffffffffu, re, 2);
    im += __shfl_xor_sync(0xffffffffu, im, 2);
    if (part == 0) ys[roff + dr] = cx(ys[roff + dr].re - re, ys[roff + dr].im - im);
    if (tid == 0) s_go = ok;
    consumer_bar();
    if (!s_go) return;  // block-uniform
    solve_sub(second);
}

// Coupling products for trsv_fold_kernel: for sub-block k and its
// neighbours at distance d in solve order (lower: k - d, upper: k + d),
// Pd[k] = Dinv_k F(k, k -/+ d), F the factor (W or its conjugate transpose;
// rows and columns beyond np read as zero), Dinv_k the sub-block's inverse
// (NB x NB column-major). grid (nsb, D): blockIdx.y + 1 is d (zero where
// the neighbour does not exist); P = P1 (nsb blocks), P2, .., each NB x NB
// column-major complex64, accumulated in FP64.
constexpr int kSmemCouple = 2 * NB * (NB + 1) * (int)sizeof(float2);
__global__ void __launch_bounds__(256) trsv_couple_kernel(const float2* __restrict__ M, int64_t ldm, int64_t np,
                                                          int nsb, int lower, const float2* __restrict__ Dinv,
                                                          float2* __restrict__ P) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    float2(*Ds)[NB + 1] = reinterpret_cast<float2(*)[NB + 1]>(dyn_smem);  // [row][q]
    float2(*Fs)[NB + 1] = Ds + NB;                                           // [q][col]
    const int k = blockIdx.x, dist = blockIdx.y + 1;
    const int nb = lower ? k - dist : k + dist;  // neighbour sub-block
    float2* out = P + ((size_t)blockIdx.y * nsb + k) * NB * NB;
    const int tid = threadIdx.x;
    if (nb < 0 || nb >= nsb) {
        for (int e = tid; e < NB * NB; e += 256) out[e] = make_float2(0.f, 0.f);
        return;
    }
    for (int e = tid; e < NB * NB; e += 256) {
        const int r = e % NB, c = e / NB;  // rows fastest: coalesced columns
        Ds[r][c] = Dinv[(size_t)k * NB * NB + e];
        const int64_t gr = (int64_t)k * NB + r, gc = (int64_t)nb * NB + c;
        Fs[r][c] = (gr < np && gc < np) ? M[gr + gc * ldm] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int r = tid % NB, c0 = tid / NB;  // columns c0 + 4i
    double re[NB / 4], im[NB / 4];
#pragma unroll
    for (int i = 0; i < NB / 4; ++i) re[i] = im[i] = 0.0;
    for (int q = 0; q < NB; ++q) {
        const float2 d = Ds[r][q];
#pragma unroll
        for (int i = 0; i < NB / 4; ++i) {
            const float2 f = Fs[q][c0 + 4 * i];
            re[i] += (double)d.x * f.x - (double)d.y * f.y;
            im[i] += (double)d.x * f.y + (double)d.y * f.x;
        }
    }
#pragma unroll
    for (int i = 0; i < NB / 4; ++i) out[r + (c0 + 4 * i) * NB] = make_float2((float)re[i], (float)im[i]);
}

// trsv_tma_kernel for 128-row CTAs with the coupling to the newest
// sub-block folded into precomputed products (trsv_couple_kernel). A CTA's
// sub-blocks in solve order are s1, s2; p is the one published just before
// s1 (its neighbour). Then
//   x_s1 = Dinv_s1 y_s1 - P1[s1] x_p,
//   x_s2 = (Dinv_s2 y_s2 - P2[s2] x_p) - P1[s2] x_s1,
// y the CTA's right-hand side less the contributions of every sub-block
// published before p, which are streamed and accumulated as before, and
// Dinv y formed while p is still awaited. Once x_p is in, s1 is one 64 x 64
// product away from publication and s2 one more, with no coupling tiles
// (the P slices are read into registers at the start): 203 against 213 us
// per solve at N = 6016. Folding the previous CTA's first sub-block as well
// (P3, one poll for both) measured slower, 246-254 us: the longer FP64
// product then sits on the chain. The same bounded waits, abort and
// publication protocol as trsv_tma_kernel.
constexpr int kSmemTrsvFold = kSmemTrsv + NB * (int)sizeof(cplx);
// Registers are granted to 288 threads in units of four warps (12 warps'
// worth), which caps a thread at 168.
__global__ void __launch_bounds__(TR_THREADS, 1)
trsv_fold_kernel(const __grid_constant__ CUtensorMap tmW, int64_t np, int nsb, int lower,
                 const float2* __restrict__ Dinv, const float2* __restrict__ P, cplx* __restrict__ x,
                 cplx* __restrict__ xpub, unsigned* __restrict__ progress, unsigned* __restrict__ err,
                 unsigned long long timeout_ns) {
    constexpr int ROWS = TR_ROWS, STG = TR_STAGES, TILE = TR_TILE, TILE_BYTES = TR_TILE_BYTES;
    constexpr int HG = TR_CONSUMERS / ROWS;  // consumer threads per row (2)
    constexpr int CPT = TR_COLS / HG;        // tile columns per consumer thread
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const uint32_t raw = smem_u32(dyn_smem);
    unsigned char* base = dyn_smem + (((raw + 1023u) & ~1023u) - raw);
    const uint32_t ring = smem_u32(base);
    const float2* ringp = reinterpret_cast<const float2*>(base);
    float2* Ds = reinterpret_cast<float2*>(base + STG * TILE_BYTES);  // 2 x [NB cols][TR_DLD]
    cplx* red = reinterpret_cast<cplx*>(Ds + 2 * NB * TR_DLD);        // ROWS: partial sums, then Dinv y
    cplx* ys = red + (HG - 1) * ROWS;                                   // ROWS
    cplx* xs = ys + ROWS;                                               // NB: x_s1
    cplx* xstage = xs + NB;                                             // 2 x NB
    const uint32_t full0 = smem_u32(xstage + 2 * NB), empty0 = full0 + 8 * STG;
    cplx* ts = reinterpret_cast<cplx*>(xstage + 2 * NB) + STG;          // NB: s2 before its last term
    __shared__ int s_t, s_go;
    __shared__ volatile int s_abort;
    static_assert(HG == 2, "two consumer threads per row");

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        s_t = (int)atomicAdd(&progress[1], 1u);
        s_abort = 0;
        for (int st = 0; st < STG; ++st) {
            mbar_init(full0 + 8 * st, 1);
            mbar_init(empty0 + 8 * st, TR_CONSUMERS / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const uint64_t deadline = global_ns() + timeout_ns;
    const int ncta = (int)((np + ROWS - 1) / ROWS);
    const int t = s_t;
    if (t >= ncta) return;  // block-uniform
    const int rb = lower ? t : ncta - 1 - t;
    const int64_t R0 = (int64_t)rb * ROWS;
    const int sbA = 2 * rb, sbB = 2 * rb + 1;
    const bool has_bot = sbB < nsb;
    const int s1 = (lower || !has_bot) ? sbA : sbB;   // solve order within the CTA
    const int s2 = lower ? sbB : sbA;
    const int w1 = s1 - sbA, w2 = s2 - sbA;           // 0 (rows 0..63) or 1 (rows 64..127)
    const int pnb = lower ? s1 - 1 : s1 + 1;          // the neighbour published just before s1
    const bool has_p = pnb >= 0 && pnb < nsb;
    // Streamed tiles: the off-diagonal ones of every sub-block before pnb,
    // in publication order.
    const int ntile_all = (int)((np + TR_COLS - 1) / TR_COLS);
    int n_off;
    if (lower) {
        n_off = R0 >= NB ? (int)((R0 - NB) / TR_COLS) : 0;
    } else {
        const int64_t c_first = R0 + ROWS + NB;  // columns from here on come before pnb
        n_off = c_first < np ? ntile_all - (int)(c_first / TR_COLS) : 0;
    }
    auto tile_k = [&](int i) -> int { return lower ? i : ntile_all - 1 - i; };

    if (warp == TR_CONSUMERS / 32) {  // producer
        if (lane == 0) {
            for (int i = 0; i < n_off; ++i) {
                const int st = i % STG;
                const uint32_t ph = (uint32_t)(i / STG) & 1u;
                if (!tr_wait(empty0 + 8 * st, ph ^ 1u, deadline)) {
                    atomicCAS(err, 0u, 2u);
                    s_abort = 1;
                    break;
                }
                mbar_expect_tx(full0 + 8 * st, TILE_BYTES);
                tma_load_2d(ring + st * TILE_BYTES, &tmW, full0 + 8 * st, (int)R0, tile_k(i) * TR_COLS);
            }
        }
        return;
    }
    // Consumers. Inverses of the two diagonal sub-blocks into shared memory.
    for (int e = tid; e < NB * NB; e += TR_CONSUMERS) {
        const int r = e & (NB - 1), c = e >> 6;
        Ds[c * TR_DLD + r] = Dinv[(size_t)sbA * NB * NB + e];
        Ds[(NB + c) * TR_DLD + r] = has_bot ? Dinv[(size_t)sbB * NB * NB + e] : make_float2(0.f, 0.f);
    }
    // The coupling slices, read at the start. Phase 1 (x_p): threads 0..127
    // form P1[s1] x_p for the s1 rows, threads 128..255 P2[s2] x_p for the
    // s2 rows, thread (row q >> 1, half q & 1) over columns (q & 1) + 2u.
    // Phase 2: P1[s2] x_s1, thread (row tid >> 2, part tid & 3) over
    // columns (tid & 3) + 4u.
    const int q1 = tid & 127, r1 = q1 >> 1, c1 = q1 & 1;
    const bool ph1_s2 = tid >= 128;
    const int kk1 = ph1_s2 ? s2 : s1;
    const int d1 = ph1_s2 ? 2 : 1;  // distance of p from kk1
    const float2* srca = P + ((size_t)(d1 - 1) * nsb + kk1) * NB * NB;  // P1[s1] or P2[s2]
    const bool use_a = ph1_s2 ? (has_bot && has_p) : has_p;
    float2 pa[NB / 2], pb[NB / 4];
    {
#pragma unroll
        for (int u = 0; u < NB / 2; ++u) pa[u] = use_a ? __ldg(&srca[r1 + (c1 + 2 * u) * NB]) : make_float2(0.f, 0.f);
        const float2* src2 = P + (size_t)s2 * NB * NB;
#pragma unroll
        for (int u = 0; u < NB / 4; ++u)
            pb[u] = has_bot ? __ldg(&src2[(tid >> 2) + ((tid & 3) + 4 * u) * NB]) : make_float2(0.f, 0.f);
    }
    // Thread (r, h): row r of the block, columns h*CPT .. h*CPT+CPT-1 of a tile.
    const int r = tid & (ROWS - 1), h = tid / ROWS;
    const int64_t grow = R0 + r;
    cplx b = cx(0, 0);  // written only by this CTA: final from the start
    if (h == 0 && grow < np) b = cx(__ldcg(&x[grow].re), __ldcg(&x[grow].im));
    double acc_re = 0.0, acc_im = 0.0;
    // Polls the NB entries of sub-block sb, and of sub-block sb2 as well
    // when sb2 >= 0 (warp 0, two entries of each per lane, all in every
    // round) into dst / dst2; false on abort or timeout.
    auto poll_sub = [&](int sb, cplx* dst, int sb2, cplx* dst2) -> bool {
        int64_t e[4];
        bool need[4];
        cplx v[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int sbq = q < 2 ? sb : sb2;
            e[q] = (int64_t)sbq * NB + lane + 32 * (q & 1);
            need[q] = sbq >= 0 && e[q] < np;
            v[q] = cx(0, 0);
        }
        bool okp = !s_abort;
        int it = 0;
        while (okp && (need[0] || need[1] || need[2] || need[3])) {
            double a[4], b2[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                a[q] = 0; b2[q] = 0;
                if (need[q]) { a[q] = ld_relaxed_f64(&xpub[e[q]].re); b2[q] = ld_relaxed_f64(&xpub[e[q]].im); }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (need[q] && !unpublished(a[q]) && !unpublished(b2[q])) { v[q] = cx(a[q], b2[q]); need[q] = false; }
            if (!(need[0] || need[1] || need[2] || need[3])) break;
            if (++it > 16) __nanosleep(64);
            if ((it & 63) == 0 && (s_abort || global_ns() > deadline || *reinterpret_cast<volatile unsigned*>(err))) {
                atomicCAS(err, 0u, 2u);
                s_abort = 1;
                okp = false;
            }
        }
        dst[lane] = v[0];
        dst[lane + 32] = v[1];
        if (sb2 >= 0) {
            dst2[lane] = v[2];
            dst2[lane + 32] = v[3];
        }
        __syncwarp();
        return okp;
    };
    // Off-diagonal tiles of the sub-blocks before pnb, a group of one NB
    // sub-block (two tiles, or one at a ragged end) per poll.
    for (int i = 0, g = 0; i < n_off; ++g) {
        const int sb = (tile_k(i) * TR_COLS) / NB;
        const int cnt = (i + 1 < n_off && (tile_k(i + 1) * TR_COLS) / NB == sb) ? 2 : 1;
        cplx* xg = xstage + (g & 1) * NB;
        if (warp == 0) poll_sub(sb, xg, -1, nullptr);
        consumer_bar();
        for (int j = 0; j < cnt; ++j, ++i) {
            const int st = i % STG;
            const uint32_t ph = (uint32_t)(i / STG) & 1u;
            bool ok = !s_abort;
            if (!tr_wait(full0 + 8 * st, ph, deadline)) {
                if (lane == 0) atomicCAS(err, 0u, 2u);
                s_abort = 1;
                ok = false;
            }
            if (ok) {
                const float2* tile = ringp + st * TILE;
                const cplx* xt = xg + (tile_k(i) * TR_COLS - sb * NB) + h * CPT;
#pragma unroll
                for (int u = 0; u < CPT; ++u) {
                    const float2 w = tile[(h * CPT + u) * ROWS + r];
                    const cplx xv = xt[u];
                    acc_re += (double)w.x * xv.re - (double)w.y * xv.im;
                    acc_im += (double)w.x * xv.im + (double)w.y * xv.re;
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(empty0 + 8 * st);
        }
    }
    if (h >= 1) red[(h - 1) * ROWS + r] = cx(acc_re, acc_im);
    consumer_bar();
    if (h == 0) ys[r] = cx(b.re - (acc_re + red[r].re), b.im - (acc_im + red[r].im));
    consumer_bar();
    // z = Dinv y for both sub-blocks (into red), thread (row dr, part) of
    // sub-block `which` over columns part + 4u.
    const int dr = tid >> 2, part = tid & 3;
    auto dinv_apply = [&](int which) {
        const float2* D = Ds + which * NB * TR_DLD;
        const cplx* y = ys + which * NB;
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int u = 0; u < NB / 4; ++u) {
            const int c = part + 4 * u;
            const float2 d = D[c * TR_DLD + dr];
            const cplx yv = y[c];
            re += (double)d.x * yv.re - (double)d.y * yv.im;
            im += (double)d.x * yv.im + (double)d.y * yv.re;
        }
        re += __shfl_xor_sync(0xffffffffu, re, 1);
        im += __shfl_xor_sync(0xffffffffu, im, 1);
        re += __shfl_xor_sync(0xffffffffu, re, 2);
        im += __shfl_xor_sync(0xffffffffu, im, 2);
        if (part == 0) red[which * NB + dr] = cx(re, im);
    };
    dinv_apply(0);
    if (has_bot) dinv_apply(1);
    // The neighbour's NB entries.
    cplx* xp = xstage;  // both group buffers are free once the loop is done
    if (warp == 0 && has_p) poll_sub(pnb, xp, -1, nullptr);
    if (tid == 0) s_go = !s_abort;
    consumer_bar();
    if (!s_go) return;  // block-uniform
    {
        double re = 0.0, im = 0.0;
        if (use_a) {
#pragma unroll
            for (int u = 0; u < NB / 2; ++u) {
                const cplx xv = xp[c1 + 2 * u];
                re += (double)pa[u].x * xv.re - (double)pa[u].y * xv.im;
                im += (double)pa[u].x * xv.im + (double)pa[u].y * xv.re;
            }
        }
        re += __shfl_xor_sync(0xffffffffu, re, 1);
        im += __shfl_xor_sync(0xffffffffu, im, 1);
        if (c1 == 0) {
            if (!ph1_s2) {
                const cplx z = red[w1 * NB + r1];
                const cplx v = cx(z.re - re, z.im - im);
                xs[r1] = v;
                const int64_t gr = R0 + w1 * NB + r1;
                if (gr < np) {
                    __stcg(&x[gr].re, v.re);
                    __stcg(&x[gr].im, v.im);
                    __stcg(&xpub[gr].re, v.re);
                    __stcg(&xpub[gr].im, v.im);
                }
            } else if (has_bot) {
                const cplx z = red[w2 * NB + r1];
                ts[r1] = cx(z.re - re, z.im - im);
            }
        }
    }
    consumer_bar();  // orders the stores of s1 before the release
    if (tid == 0) st_release_gpu(&progress[0], lower ? (unsigned)s1 + 1u : (unsigned)(nsb - s1));
    if (!has_bot) return;
    {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int u = 0; u < NB / 4; ++u) {
            const cplx xv = xs[part + 4 * u];
            re += (double)pb[u].x * xv.re - (double)pb[u].y * xv.im;
            im += (double)pb[u].x * xv.im + (double)pb[u].y * xv.re;
        }
        re += __shfl_xor_sync(0xffffffffu, re, 1);
        im += __shfl_xor_sync(0xffffffffu, im, 1);
        re += __shfl_xor_sync(0xffffffffu, re, 2);
        im += __shfl_xor_sync(0xffffffffu, im, 2);
        if (part == 0) {
            const cplx v = cx(ts[dr].re - re, ts[dr].im - im);
            const int64_t gr = R0 + w2 * NB + dr;
            if (gr < np) {
                __stcg(&x[gr].re, v.re);
                __stcg(&x[gr].im, v.im);
                __stcg(&xpub[gr].re, v.re);
                __stcg(&xpub[gr].im, v.im);
            }
        }
    }
    consumer_bar();
    if (tid == 0) st_release_gpu(&progress[0], lower ? (unsigned)s2 + 1u : (unsigned)(nsb - s2));
}

// ------------------------------------------------------------ small vector ops
__global__ void dot_partial_kernel(int64_t n, int k, const cplx* __restrict__ V, int64_t ldv,
                                   const cplx* __restrict__ w, cplx* __restrict__ out) {
    // out[blockIdx.y + k * blockIdx.x] = sum over this block's slice of conj(V_j) w
    const int j = blockIdx.y;
    __shared__ double sr[8], si[8];
    double re = 0, im = 0;
    const cplx* v = V + (int64_t)j * ldv;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const cplx a = v[i], b = w[i];
        re += a.re * b.re + a.im * b.im;
        im += a.re * b.im - a.im * b.re;
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if ((threadIdx.x & 31) == 0) { sr[threadIdx.x >> 5] = re; si[threadIdx.x >> 5] = im; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tre = 0, tim = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { tre += sr[q]; tim += si[q]; }
        out[(int64_t)blockIdx.x * k + j] = cx(tre, tim);
    }
}

__global__ void dot_finish_kernel(int k, int parts, const cplx* __restrict__ partial, cplx* __restrict__ h) {
    const int j = threadIdx.x;
    if (j >= k) return;
    cplx s = cx(0, 0);
    for (int p = 0; p < parts; ++p) s += partial[(int64_t)p * k + j];
    h[j] = s;
}

// w -= V[:, 0:k] h
__global__ void axpy_multi_kernel(int64_t n, int k, const cplx* __restrict__ V, int64_t ldv,
                                  const cplx* __restrict__ h, cplx* __restrict__ w) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cplx s = w[i];
    for (int j = 0; j < k; ++j) s = s - V[i + (int64_t)j * ldv] * h[j];
    w[i] = s;
}

__global__ void scale_copy_kernel(int64_t n, const cplx* __restrict__ x, double s, cplx* __restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = x[i] * s;
}

__global__ void combo_kernel(int64_t n, int k, const cplx* __restrict__ V, int64_t ldv,
                             const cplx* __restrict__ y, cplx* __restrict__ out) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cplx s = cx(0, 0);
    for (int j = 0; j < k; ++j) s += V[i + (int64_t)j * ldv] * y[j];
    out[i] = s;
}

__global__ void add_kernel(int64_t n, const cplx* __restrict__ a, cplx* __restrict__ x) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += a[i];
}

// Adjoint support: W^H solves are done on the conjugate transpose factors.
__global__ void conj_transpose_c64_kernel(const float2* __restrict__ W, int64_t ldw, int64_t np,
                                          float2* __restrict__ WT) {
    __shared__ float2 tile[32][33];
    const int64_t bx = (int64_t)blockIdx.x * 32, by = (int64_t)blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t r = bx + threadIdx.x, c = by + j;
        if (r < np && c < np) tile[j][threadIdx.x] = W[r + c * ldw];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int64_t r = by + threadIdx.x, c = bx + j;
        if (r < np && c < np) {
            const float2 v = tile[threadIdx.x][j];
            WT[r + c * ldw] = make_float2(v.x, -v.y);
        }
    }
}

// Complex128 (ld lda) to complex64 (ld n) copy of an n x n matrix.
__global__ void to_c64_kernel(const cplx* __restrict__ A, int64_t lda, int64_t n, float2* __restrict__ W) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (r >= n) return;
    const cplx v = A[r + c * lda];
    W[r + c * n] = make_float2((float)v.re, (float)v.im);
}

// dinv[i] = 1 / A[i][i] (Jacobi preconditioner of GMRES_C64).
__global__ void inv_diag_kernel(const cplx* __restrict__ A, int64_t lda, int64_t n, cplx* __restrict__ dinv) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const cplx d = A[i + i * lda];
    const double m = d.re * d.re + d.im * d.im;
    dinv[i] = m > 0.0 ? cx(d.re / m, -d.im / m) : cx(1.0, 0.0);
}

// z = dinv .* v (or conj(dinv) .* v for the adjoint).
__global__ void diag_scale_kernel(int64_t n, const cplx* __restrict__ dinv, const cplx* __restrict__ v, int conj_d,
                                  cplx* __restrict__ z) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const cplx d = conj_d ? cx(dinv[i].re, -dinv[i].im) : dinv[i];
    z[i] = d * v[i];
}

// Conjugate transpose of each NB x NB block (column-major) of `in`, one CTA per block.
__global__ void conj_transpose_blocks_kernel(const float2* __restrict__ in, float2* __restrict__ out) {
    const float2* src = in + (size_t)blockIdx.x * NB * NB;
    float2* dst = out + (size_t)blockIdx.x * NB * NB;
    for (int e = threadIdx.x; e < NB * NB; e += blockDim.x) {
        const int r = e % NB, c = e / NB;
        const float2 v = src[c + r * NB];
        dst[e] = make_float2(v.x, -v.y);
    }
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

// Own FP64 LU: diagonal block k of a triangular solve, Y_k = Inv_k Y_k in
// place for 16 columns per CTA (complex128; rows beyond the block's width
// are left alone, the inverse is padded with the identity). Thread (r, p)
// holds row r of Inv_k over columns 16p .. 16p+15 in registers (all its
// loads issued at once), forms that quarter of each column's product, and
// the four quarters are summed through shared memory.
__global__ void __launch_bounds__(256) fp64_diag_apply_kernel(cplx* __restrict__ Y, int64_t ldy, int64_t k0, int kb,
                                                              int nrhs, const double2* __restrict__ Inv) {
    __shared__ double2 ys[16][NB];
    __shared__ double2 red[4][NB];
    const int tid = threadIdx.x;
    const int c0 = blockIdx.x * 16;
    const int r = tid & (NB - 1), p = tid >> 6;
    double2 inv[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) inv[u] = __ldg(&Inv[r + (16 * p + u) * NB]);  // column-major
    for (int e = tid; e < 16 * NB; e += blockDim.x) {
        const int rr = e % NB, c = e / NB;
        const cplx v = (c0 + c < nrhs && rr < kb) ? Y[(k0 + rr) + (int64_t)(c0 + c) * ldy] : cx(0, 0);
        ys[c][rr] = make_double2(v.re, v.im);
    }
    __syncthreads();
    const int ncol = min(16, nrhs - c0);
    for (int c = 0; c < ncol; ++c) {
        double2 acc = make_double2(0.0, 0.0);
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            const double2 y = ys[c][16 * p + u];
            acc.x = fma(inv[u].x, y.x, fma(-inv[u].y, y.y, acc.x));
            acc.y = fma(inv[u].x, y.y, fma(inv[u].y, y.x, acc.y));
        }
        red[p][r] = acc;
        __syncthreads();
        if (p == 0 && r < kb) {
            const double2 s1 = red[1][r], s2 = red[2][r], s3 = red[3][r];
            Y[(k0 + r) + (int64_t)(c0 + c) * ldy] = cx(acc.x + s1.x + s2.x + s3.x, acc.y + s1.y + s2.y + s3.y);
        }
        __syncthreads();
    }
}

// X(:, c) += D(:, c)
__global__ void add_cols_kernel(int64_t n, const cplx* __restrict__ D, int64_t ldd, cplx* __restrict__ X,
                                int64_t ldx) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r < n) X[r + c * ldx] += D[r + c * ldd];
}

// Y(:, c) = X(:, c) (rectangular copy between leading dimensions)
__global__ void copy_cols_kernel(int64_t n, const cplx* __restrict__ X, int64_t ldx, cplx* __restrict__ Y,
                                 int64_t ldy) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r < n) Y[r + c * ldy] = X[r + c * ldx];
}

}  // namespace

// ------------------------------------------------------------ host side

static MixedState* state_of(DenseSolver* s) { return static_cast<MixedState*>(s->gemm_state); }

void mixed_release(DenseSolver* s) {
    MixedState* st = state_of(s);
    if (st) {
        drop_graphs(st);
        block_solve_release(st);
        if (st->gemm) gemm_tc_destroy(st->gemm);
        if (st->ev_cols) cudaEventDestroy(st->ev_cols);
        if (st->ev_diag) cudaEventDestroy(st->ev_diag);
        if (st->ev_pan) cudaEventDestroy(st->ev_pan);
        if (st->ev_lcol) cudaEventDestroy(st->ev_lcol);
        if (st->ev_gemm) cudaEventDestroy(st->ev_gemm);
        if (st->ev_head) cudaEventDestroy(st->ev_head);
        if (st->side) cudaStreamDestroy(st->side);
        if (st->side2) cudaStreamDestroy(st->side2);
        delete st;
    }
    s->gemm_state = nullptr;
    s->lu.release(); s->perm.release(); s->panel.release(); s->gemm_a.release(); s->gemm_b.release();
    s->krylov.release(); s->vec.release(); s->flags.release(); s->gemv_scratch.release(); s->couple.release();
}

static int check_err(DenseSolver* s, const char* what) {
    MixedState* st = state_of(s);
    unsigned e = 0;
    SIEB_TRY_CUDA(cudaMemcpyAsync(&e, st->err, sizeof(unsigned), cudaMemcpyDeviceToHost, s->ctx->stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(s->ctx->stream));
    if (e == 1u) {
        set_error(std::string(what) + ": zero or non-finite pivot in the unpivoted LU of the randomized matrix");
        return SIEB200_SINGULAR;
    }
    if (e == 2u) {
        set_error(std::string(what) + ": a triangular-solve block waited past its bound");
        return SIEB200_TIMEOUT;
    }
    if (e != 0u) {
        set_error(std::string(what) + ": device error word " + std::to_string(e));
        return SIEB200_CUDA_ERROR;
    }
    return SIEB200_OK;
}

static int mixed_enqueue(DenseSolver* s, MixedState* st, size_t bFlags, int K3);
// Overlapped block steps (see mixed_enqueue): trailing updates at least this
// many columns wide (0: none), and the SMs they leave to the panels.
constexpr int kOverlapMinDefault = 0;
// Pair schedule for block steps whose paired GEMM is at least this wide (0:
// none; SIEB200_PAIR_UPDATE=1 makes every step a pair step). Measured with
// every step paired: N = 6000 factor + solve 9.75 against 8.99 ms (the chain
// of the steps without a GEMM is exposed), N = 17280 factorization 106 against
// 117 ms and the N = 58,800 adjoint gradient 5.21 against 5.96 s (the GEMM
// sets the pace there): so only updates at least this wide are paired. The
// paired updates also leave slightly less accurate factors: with 8192 the
// config-3 system (N = 17280, 64 right-hand sides) needed one refinement
// iteration more (6 instead of 5), which cost more than the faster
// factorization gained; 20000 keeps such systems on single steps.
constexpr int kPairMinDefault = 20000;
// Stop an FGMRES cycle at an Arnoldi residual estimate of this fraction of
// the tolerance (the true residual is checked after the cycle; 0.5 cost the
// 17280-unknown GSTC batch 16 ms more per solve, 129 against 113 ms).
constexpr double kGmresEstFactorDefault = 0.9;
constexpr int kOverlapSmsDefault = 20;
// Split panels (SIEB200_PANEL_HEAD_MAX): 0 = off.
constexpr int kPanelHeadMaxDefault = 0;

static int fp64_factorize(DenseSolver* s);

int mixed_factorize(DenseSolver* s) {
    if (s->method == SIEB200_SOLVER_LU_FP64) return fp64_factorize(s);
    SIEB_CHECK(s->method == SIEB200_SOLVER_MIXED_IR, SIEB200_INVALID_ARG, "unsupported solver method");
    sieb200_ctx* ctx = s->ctx;
    cudaStream_t stream = ctx->stream;
    MixedState* st = state_of(s);
    if (!st) {
        st = new MixedState();
        s->gemm_state = st;
    }
    const int64_t n = s->n;
    const int64_t np = ((n + 3) / 4) * 4;
    const int64_t ldw = ((np + 31) / 32) * 32;
    const int64_t nbl = (np + NB - 1) / NB;
    st->n = n; st->np = np; st->ldw = ldw; st->nbl = nbl;
    st->adj_ready = false;
    st->couple_ready[0] = st->couple_ready[1] = false;
    block_solve_invalidate(st);
    const char* env = getenv("SIEB200_TRAILING_SIMT");
    st->use_tc = (env && env[0] == '1') ? 0 : 1;
    const char* pair_env = getenv("SIEB200_PAIR_UPDATE");
    st->pair = (pair_env && pair_env[0] == '1') ? 1 : 0;
    const char* pmin_env = getenv("SIEB200_PAIR_MIN");
    st->pair_min = pmin_env ? std::max(0, atoi(pmin_env)) : kPairMinDefault;
    const char* hilo_env = getenv("SIEB200_GEMM_HILO");
    st->hilo = (hilo_env && hilo_env[0] == '0') ? 0 : 1;
    const char* ovl_env = getenv("SIEB200_OVERLAP_MIN");
    st->ovl_min = ovl_env ? std::max(0, atoi(ovl_env)) : kOverlapMinDefault;
    const char* ovs_env = getenv("SIEB200_OVERLAP_SMS");
    st->ovl_sms = ovs_env ? std::max(2, std::min(s->ctx->sm_count / 2, atoi(ovs_env))) : kOverlapSmsDefault;
    const char* lcol_env = getenv("SIEB200_GEMM_LCOL");
    st->lcol = (lcol_env && lcol_env[0] >= '0' && lcol_env[0] <= '3' && lcol_env[1] == 0) ? lcol_env[0] - '0' : 1;
    const char* lorn_env = getenv("SIEB200_TF32_LO_RN");
    st->lo_rn = (lorn_env && lorn_env[0] == '1') ? 1 : 0;
    st->diag_split = diag_split_env();
    st->diag_panels = diag_panels_env();
    st->diag_compact = diag_compact_env();
    const char* rec_env = getenv("SIEB200_DIAG_REC");
    st->diag_rec = (rec_env && rec_env[0] == '1') ? 1 : 0;
    const char* head_env = getenv("SIEB200_PANEL_HEAD_MAX");
    st->head_max = head_env ? std::max(0, atoi(head_env)) : kPanelHeadMaxDefault;
    const char* hsm_env = getenv("SIEB200_PANEL_HEAD_SMEM");
    st->head_smem = hsm_env ? std::max(kSmemPanel, std::min(kSmemPanelHeadMax, atoi(hsm_env))) : kSmemPanel;

    // Workspace layout in s->lu: W | Linv | Uinv | diag | err+flags ; packs separate.
    const size_t bW = sizeof(float2) * ldw * np;
    const size_t bInv = sizeof(float2) * NB * NB * nbl;
    const size_t bDiag = sizeof(double) * 8 * np;
    const size_t bFlags = sizeof(unsigned) * (4 * nbl + 16);
    auto up = [](size_t b) { return ((b + 255) / 256) * 256; };
    SIEB_RETURN_IF(s->lu.reserve(up(bW) + 2 * up(bInv) + up(bDiag) + up(bFlags)));
    char* base = s->lu.as<char>();
    st->W = reinterpret_cast<float2*>(base);
    st->Linv = reinterpret_cast<float2*>(base + up(bW));
    st->Uinv = reinterpret_cast<float2*>(base + up(bW) + up(bInv));
    st->diag = reinterpret_cast<double*>(base + up(bW) + 2 * up(bInv));
    st->err = reinterpret_cast<unsigned*>(base + up(bW) + 2 * up(bInv) + up(bDiag));
    st->tri_flags = st->err + 16;
    const int K3 = 6 * NB;
    const size_t bApack = ((sizeof(float) * 2 * np * K3 + 255) / 256) * 256;
    SIEB_RETURN_IF(s->gemm_a.reserve(2 * bApack));
    // two step buffers (single-step schedule) or the pair schedule's K = 2 x 384
    SIEB_RETURN_IF(s->gemm_b.reserve(sizeof(float) * np * 2 * K3));
    st->Apack[0] = s->gemm_a.as<float>();
    st->Apack[1] = reinterpret_cast<float*>(s->gemm_a.as<char>() + bApack);
    st->Bpack = s->gemm_b.as<float>();
    if (st->use_tc && !st->gemm) SIEB_RETURN_IF(gemm_tc_create(&st->gemm));
    if (!st->side) {
        int least = 0, greatest = 0;
        SIEB_TRY_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        SIEB_TRY_CUDA(cudaStreamCreateWithPriority(&st->side, cudaStreamNonBlocking, greatest));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_cols, cudaEventDisableTiming));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_diag, cudaEventDisableTiming));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_pan, cudaEventDisableTiming));
    }
    if (!st->side2) {
        int least = 0, greatest = 0;
        SIEB_TRY_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        SIEB_TRY_CUDA(cudaStreamCreateWithPriority(&st->side2, cudaStreamNonBlocking, greatest));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_lcol, cudaEventDisableTiming));
    }
    if (!st->ev_gemm) {
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_gemm, cudaEventDisableTiming));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_head, cudaEventDisableTiming));
    }

    static bool attrs_set = false;
    if (!attrs_set) {
        SIEB_TRY_CUDA(cudaFuncSetAttribute(trailing_simt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemDiag));
        // (a head launch may ask for more, up to kSmemPanelHeadMax)
        SIEB_TRY_CUDA(cudaFuncSetAttribute(panels_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kSmemPanelHeadMax));
        SIEB_RETURN_IF(diag_set_smem<float2>(kSmemDiagUpd));
        SIEB_TRY_CUDA(cudaFuncSetAttribute(diag_lu_rec_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kSmemDiagRec));
        attrs_set = true;
    }

    // Replay, capture or run eagerly (see MixedState::graphs).
    MixedState::GraphKey key;
    key.A = s->A; key.lda = s->lda; key.n = n; key.W = st->W; key.pack = st->Apack[0];
    const int gemm_sms = s->sm_cap > 0 ? std::min(s->sm_cap, ctx->sm_count - 1) : ctx->sm_count - 1;
    key.use_tc = st->use_tc + 2 * st->pair + 4 * st->hilo + 8 * st->lcol + 16 * st->lo_rn + 32 * st->diag_split +
                 64 * st->diag_panels + 128 * st->diag_rec + 256 * st->diag_compact;
    key.sms = gemm_sms;
    key.ovl = ((int64_t)st->pair_min << 32) | (int64_t)(st->ovl_min * 1000 + st->ovl_sms);
    key.head = ((int64_t)st->head_max << 20) | (int64_t)st->head_smem;
    const char* no_graphs = getenv("SIEB200_NO_GRAPHS");
    const bool graphs = !ctx->prof.enabled && !(no_graphs && no_graphs[0] == '1');
    if (graphs) {
        for (auto& g : st->graphs) {
            if (g.exec && g.key == key) {
                g.used = ++st->tick;
                SIEB_TRY_CUDA(cudaGraphLaunch(g.exec, stream));
                note_launches(g.launches);
                return check_err(s, "mixed LU factorization");
            }
        }
    }
    const bool capture = graphs && (key == st->seen[0] || key == st->seen[1]);
    if (!(key == st->seen[0])) {
        st->seen[1] = st->seen[0];
        st->seen[0] = key;
    }
    if (capture) {
        MixedState::Graph& g = st->graphs[st->graphs[0].used <= st->graphs[1].used ? 0 : 1];
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = MixedState::Graph();
        const long long launches0 = launch_count();
        SIEB_TRY_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int rc = mixed_enqueue(s, st, bFlags, K3);
        cudaGraph_t cg = nullptr;
        cudaError_t ce = cudaStreamEndCapture(stream, &cg);
        if (rc == SIEB200_OK && ce == cudaSuccess) ce = cudaGraphInstantiate(&g.exec, cg, 0);
        if (cg) cudaGraphDestroy(cg);
        if (rc != SIEB200_OK || ce != cudaSuccess) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g = MixedState::Graph();
            if (rc != SIEB200_OK) return rc;
            cudaGetLastError();
            set_error(std::string("capturing the factorization as a CUDA graph failed: ") + cudaGetErrorString(ce));
            return SIEB200_CUDA_ERROR;
        }
        g.key = key;
        g.launches = launch_count() - launches0;
        g.used = ++st->tick;
        SIEB_TRY_CUDA(cudaGraphLaunch(g.exec, stream));
    } else {
        SIEB_RETURN_IF(mixed_enqueue(s, st, bFlags, K3));
    }
    return check_err(s, "mixed LU factorization");
}

// Enqueues one mixed factorization on the context stream and the lookahead
// stream (joined back at the end): eager or under stream capture.
static int mixed_enqueue(DenseSolver* s, MixedState* st, size_t bFlags, int K3) {
    sieb200_ctx* ctx = s->ctx;
    cudaStream_t stream = ctx->stream;
    const int64_t n = st->n, np = st->np, ldw = st->ldw, nbl = st->nbl;
    cudaEvent_t ev_fact;
    ctx->prof.begin(stream, 6, (8.0 / 3.0) * 4.0 * (double)np * np * np, 0.0, &ev_fact);
    SIEB_TRY_CUDA(cudaMemsetAsync(st->err, 0, bFlags, stream));
    rbt_init_kernel<<<blocks_for(8 * np, 256), 256, 0, stream>>>(st->diag, np, 0x5EB200ull);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    const int64_t q = np / 4;
    rbt_matrix_kernel<float2><<<dim3(blocks_for(q, 128), (unsigned)q), 128, 0, stream>>>(
        reinterpret_cast<const cplx*>(s->A), s->lda, n, np, st->diag, st->diag + 4 * np, st->W, ldw);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());

    // Diagonal block bk after the updates of the block steps at column
    // offsets kp1, kp2 (-1 = none).
    auto diag_blk = [&](int64_t bk, int64_t kp1, int64_t kp2, cudaStream_t sm) -> int {
        const int64_t k0 = bk * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        const int nupd = (kp1 >= 0) + (kp2 >= 0);
        cudaEvent_t ev;
        ctx->prof.begin(sm, 3, (8.0 / 3.0 + 8.0 / 3.0) * NB * NB * NB + nupd * 8.0 * NB * NB * NB,
                        8.0 * NB * NB * (3.0 + 2.0 * nupd), &ev);
        if (nupd > 0 && (st->diag_split || st->diag_rec)) {
            diag_update_kernel<float2><<<dim3(NB / 16, NB / 16), 256, 0, sm>>>(st->W, ldw, k0, kb, kp1, kp2);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
            kp1 = kp2 = -1;
        }
        if (st->diag_rec) {
            diag_lu_rec_kernel<<<1, 256, kSmemDiagRec, sm>>>(st->W, ldw, k0, kb, st->Linv + (size_t)bk * NB * NB,
                                                             st->Uinv + (size_t)bk * NB * NB, st->err);
            SIEB_NOTE_LAUNCH();
            ctx->prof.end(sm, ev);
            SIEB_TRY_CUDA(cudaGetLastError());
            return SIEB200_OK;
        }
        diag_kernel_for<float2>(st)<<<1, kDiagThreads, kSmemDiagUpd, sm>>>(
            st->W, ldw, k0, kb, st->Linv + (size_t)bk * NB * NB, st->Uinv + (size_t)bk * NB * NB, st->err, kp1, kp2);
        SIEB_NOTE_LAUNCH();
        ctx->prof.end(sm, ev);
        SIEB_TRY_CUDA(cudaGetLastError());
        return SIEB200_OK;
    };
    // Both panels of block bk on the context stream: L21 after the updates
    // of the steps kp1, kp2 into the A pack, U12 after the update of step
    // kpu into the B pack. Pair schedule: the trailing GEMM of an odd step q
    // applies steps q - 1 and q together (K = 2 x 384), so step j's packs go
    // to K half j & 1 of one buffer, rows from s0(q) and columns from
    // s0(q) + NB (q = j | 1); single-step schedule: one K = 384 pack per
    // step, rows from s0(j), all columns (the GEMM offsets them).
    // Split layout (hilo): a step's pack is [hi | lo], 2 x 2NB = 256 wide,
    // and the GEMM forms the three products from it; in the pair schedule
    // the two steps' hi parts come first, then their lo parts.
    // Block step bk runs the pair schedule when SIEB200_PAIR_UPDATE=1, or
    // when the GEMM of its pair (at the odd step bk | 1) is at least
    // st->pair_min columns wide: the early, wide updates of a large system,
    // where the GEMM rather than the chain sets the pace; both steps of a
    // pair decide alike, and once a pair is too narrow every later one is.
    auto pair_at = [&](int64_t bk) -> bool {
        if (!st->use_tc) return false;
        if (st->pair) return true;
        if (st->pair_min <= 0) return false;
        const int64_t q = bk | 1;
        const int64_t mq = np - std::min(np, (q + 1) * NB);  // rows below block q
        return mq - NB >= st->pair_min;
    };
    const bool hilo = st->hilo != 0;
    const int64_t KS = hilo ? 4 * NB : K3;  // pack width of one step
    const int64_t KP = 2 * KS;              // pack width of a pair
    const int layout = hilo ? 1 : 0;
    // part 0: all of the panels; 1: the head, the rows and columns of the
    // next block (the next diagonal block's update needs only these); 2: the
    // rest (none when the head is all).
    auto panels = [&](int64_t bk, int64_t kp1, int64_t kp2, int64_t kpu, cudaStream_t ps, int part) -> int {
        const int64_t k0 = bk * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        const int64_t s0 = k0 + kb;
        if (s0 >= np) return SIEB200_OK;
        const int64_t m = np - s0;
        PanelArgs pa;
        pa.k0 = k0; pa.kb = kb; pa.s0 = s0; pa.np = np;
        pa.nL = (int)blocks_for(m, 32);
        const int nhead = std::min(pa.nL, NB / 32);
        if (part == 1) {
            pa.b_first = 0; pa.nl_run = nhead;
        } else if (part == 2) {
            if (pa.nL <= nhead) return SIEB200_OK;
            pa.b_first = nhead; pa.nl_run = pa.nL - nhead;
        }
        const int run = pa.nl_run > 0 ? pa.nl_run : pa.nL;
        const double share = (double)run / (double)pa.nL;
        pa.pack = st->use_tc;
        pa.kp[0] = kp1; pa.kp[1] = kp2; pa.kpu = kpu;
        pa.lo_rn = st->lo_rn;
        if (pair_at(bk)) {
            const int half = (int)(bk & 1);
            const int64_t q_s0 = half ? s0 : s0 + NB;  // s0 of the step whose GEMM uses this pack
            const int64_t off = half * (hilo ? 2 * NB : K3);
            pa.Apack = st->Apack[0] + off; pa.a_ld = KP; pa.a_r0 = q_s0;
            pa.Bpack = st->Bpack + off; pa.b_ld = KP; pa.b_c0 = q_s0 + NB;
            pa.a_lo = pa.b_lo = hilo ? 4 * NB : 0;
        } else {
            // both packs double-buffered by step parity: an overlapped GEMM
            // still reads step bk - 1's while these are written
            pa.Apack = st->Apack[bk & 1]; pa.a_ld = KS; pa.a_r0 = s0;
            pa.Bpack = st->Bpack + (bk & 1) * np * KS; pa.b_ld = KS; pa.b_c0 = s0;
            pa.a_lo = pa.b_lo = hilo ? 2 * NB : 0;
        }
        const int nupd = (kp1 >= 0) + (kp2 >= 0) + (kpu >= 0);
        cudaEvent_t ev;
        ctx->prof.begin(ps, 4, share * 8.0 * NB * NB * (double)m * (2 + nupd),
                        share * 8.0 * NB * (double)m * (4 + nupd), &ev);
        panels_kernel<float2><<<(unsigned)(2 * run), 256, part == 1 ? st->head_smem : kSmemPanel, ps>>>(
            st->W, ldw, st->Uinv + (size_t)bk * NB * NB, st->Linv + (size_t)bk * NB * NB, pa);
        SIEB_NOTE_LAUNCH();
        ctx->prof.end(ps, ev);
        SIEB_TRY_CUDA(cudaGetLastError());
        return SIEB200_OK;
    };
    // shift: the first block row (128 real rows) starts that many columns in
    auto gemm = [&](int64_t s0, int64_t c0, int64_t ncols, const float* A, const float* B, int K,
                    int max_ctas, int64_t shift) -> int {
        const int64_t m = np - s0;
        float* C = reinterpret_cast<float*>(st->W + s0 + c0 * ldw);
        cudaEvent_t ev;
        // tensor work: three products of K/3 (one sweep) or K/2 (split) columns
        const double keff = hilo ? 1.5 * K : (double)K;
        const double elems = (2.0 * m) * ncols - (double)std::min<int64_t>(128, 2 * m) * shift;
        ctx->prof.begin(stream, 0, 2.0 * elems * keff, 4.0 * (2.0 * elems + (2.0 * m + ncols) * K), &ev);
        SIEB_RETURN_IF(gemm_tc_sub(st->gemm, stream, C, 2 * ldw, A, B, 2 * m, ncols, K, max_ctas, layout, shift));
        ctx->prof.end(stream, ev);
        return SIEB200_OK;
    };
    const int gemm_ctas = s->sm_cap > 0 ? std::min(s->sm_cap, ctx->sm_count - 1) : ctx->sm_count - 1;

    // Right-looking block LU with a lookahead of one block. Step bk: the
    // panels of block bk are formed on the context stream; the next
    // diagonal block takes its update(s) from them and is factored on the
    // side stream while the tensor-core trailing update runs here; then the
    // next panels, which apply the pending updates to the next block's
    // column (and, in the pair schedule after an even step, to its row).
    // In a single step the trailing update skips only the next diagonal
    // block (the side stream factors it meanwhile): its first block row
    // starts one block column further right and its other rows cover the
    // next block column too, so the next L21 panel is only a triangular
    // product (SIEB200_GEMM_LCOL=1, default). On the 6016-unknown system
    // this takes the factorization from 6.93 to 5.99 ms (with the diagonal
    // block's update in its own kernel). That column's last update then
    // comes from TF32 products accumulated on the tensor cores instead of
    // FP32 FMAs, and the 17280-unknown GSTC batch needs a sixth refinement
    // iteration (about 20 of 235 ms). The alternatives keep the FP32 update
    // (same factors as the panels, bit for bit): =0 the panels apply it,
    // =2 col_update_kernel on a third stream beside the GEMM (its CTAs
    // crowd the diagonal kernel's SM: 6.7-6.9 ms), =3 col_update_kernel
    // ahead of the GEMM (6.72 ms); the GEMM then skips the whole next block
    // column. In the pair schedule the update skips the next block column
    // and runs after odd steps only, for both steps of the pair at once
    // (half the C traffic per flop). The persistent GEMM leaves one SM to
    // the diagonal kernel (whose shared memory keeps it off the GEMM's SMs).
    // The single-step schedule is the default (SIEB200_PAIR_UPDATE=1 selects
    // the pair schedule): on the 6016-unknown system the pair schedule's
    // GEMM runs at 360 TFLOP/s against 297, but the steps without a GEMM put
    // the panels and the diagonal block back to back and the extra updates
    // lengthen that chain, so the factorization takes longer overall.
    //
    // Overlapped steps (single-step schedule, trailing update at least
    // st->ovl_min columns wide): the trailing GEMM skips the next block row
    // as well and runs on all but st->ovl_sms SMs, the next panels take this
    // step's update of that row themselves (kpu, as after an even pair step)
    // and run on the side stream right after the next diagonal block, on the
    // SMs the GEMM leaves free; so the panels leave the critical path while
    // the GEMM is the longer of the two. The next GEMM waits for them (event).
    SIEB_RETURN_IF(diag_blk(0, -1, -1, stream));
    SIEB_RETURN_IF(panels(0, -1, -1, -1, stream, 0));
    bool pan_side = false;  // the last panels ran on the side stream
    // Split panels (single steps with the GEMM covering the next block
    // column, no overlapped steps): when the next panels are at most
    // st->head_max wide, their head runs on the side stream right after the
    // next diagonal block and the GEMM, followed there by the diagonal block
    // after it, while the rest of the panels run here; the chain of a step
    // whose diagonal block outlasts the GEMM is then head + diagonal block
    // instead of all of the panels + diagonal block.
    const int64_t head_max = (st->ovl_min > 0 || st->lcol != 1) ? 0 : st->head_max;
    bool head_prev = false;  // this step's panels ran split (head on the side stream, ev_head)
    // The side stream joins only after it has been forked from this one: a
    // system of one block has no lookahead, and under stream capture a wait
    // on an event of the never-forked side stream is refused.
    bool side_forked = false;
    for (int64_t bk = 0; bk < nbl; ++bk) {
        const int64_t k0 = bk * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        const int64_t s0 = k0 + kb;
        if (s0 >= np) break;
        const int64_t m = np - s0;
        if (st->use_tc) {
            const int64_t n1 = std::min<int64_t>(NB, m);  // the next block's columns
            const bool pair = pair_at(bk);
            const bool odd = pair && (bk & 1);
            const int64_t kprev = odd ? k0 - NB : -1;      // the first step of the pair
            if (!head_prev) {  // (else the head went before on the side stream)
                SIEB_TRY_CUDA(cudaEventRecord(st->ev_cols, stream));
                SIEB_TRY_CUDA(cudaStreamWaitEvent(st->side, st->ev_cols, 0));
                side_forked = true;
            }
            SIEB_RETURN_IF(diag_blk(bk + 1, k0, kprev, st->side));
            const bool ovl = !pair && st->ovl_min > 0 && m - n1 >= st->ovl_min && m > 2 * n1;
            if (pan_side) SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, st->ev_pan, 0));  // GEMM operands
            if (head_prev) SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, st->ev_head, 0));  // the head's packs
            head_prev = false;
            if (ovl) {
                const int octas = std::max(1, std::min(gemm_ctas, ctx->sm_count - st->ovl_sms));
                SIEB_RETURN_IF(gemm(s0 + n1, s0 + n1, m - n1, st->Apack[bk & 1] + 2 * n1 * KS,
                                    st->Bpack + (bk & 1) * np * KS + n1 * KS, (int)KS, octas, 0));
                SIEB_RETURN_IF(panels(bk + 1, k0, -1, k0, st->side, 0));
                SIEB_TRY_CUDA(cudaEventRecord(st->ev_pan, st->side));
                pan_side = true;
                continue;
            }
            const bool pan_was_side = pan_side;
            pan_side = false;
            SIEB_TRY_CUDA(cudaEventRecord(st->ev_diag, st->side));
            // lcol 1: the GEMM covers the next block column below its
            // diagonal block; lcol 2: col_update_kernel does, on the
            // third stream beside the GEMM (which skips that column);
            // lcol 3: col_update_kernel on this stream before the GEMM
            const bool lcol = !pair && st->lcol == 1;
            const bool lside = !pair && st->lcol == 2;
            const bool lmain = !pair && st->lcol == 3;
            if (lmain && m > n1) {  // lcol 3: the same kernel here, ahead of the GEMM, on the whole GPU
                col_update_kernel<<<(unsigned)blocks_for(m - n1, 32), 256, 0, stream>>>(st->W, ldw, s0, (int)n1,
                                                                                       s0 + n1, np, k0);
                SIEB_NOTE_LAUNCH();
                SIEB_TRY_CUDA(cudaGetLastError());
            }
            if (lside && m > n1) {
                // after panels (stream order of the context stream, or the
                // side stream after an overlapped step)
                SIEB_TRY_CUDA(cudaStreamWaitEvent(st->side2, st->ev_cols, 0));
                if (pan_was_side) SIEB_TRY_CUDA(cudaStreamWaitEvent(st->side2, st->ev_pan, 0));
                col_update_kernel<<<(unsigned)blocks_for(m - n1, 32), 256, 0, st->side2>>>(st->W, ldw, s0, (int)n1,
                                                                                           s0 + n1, np, k0);
                SIEB_NOTE_LAUNCH();
                SIEB_TRY_CUDA(cudaGetLastError());
                SIEB_TRY_CUDA(cudaEventRecord(st->ev_lcol, st->side2));
            }
            if (!pair) {
                if (m > n1 && lcol)
                    SIEB_RETURN_IF(gemm(s0, s0, m, st->Apack[bk & 1], st->Bpack + (bk & 1) * np * KS, (int)KS,
                                        gemm_ctas, n1));
                else if (m > n1)
                    SIEB_RETURN_IF(gemm(s0, s0 + n1, m - n1, st->Apack[bk & 1],
                                        st->Bpack + (bk & 1) * np * KS + n1 * KS, (int)KS, gemm_ctas, 0));
            } else if (odd && m > n1) {
                SIEB_RETURN_IF(gemm(s0, s0 + n1, m - n1, st->Apack[0], st->Bpack, (int)KP, gemm_ctas, 0));
            }
            const int64_t m1 = m - n1;  // width of the next panels
            if (lcol && head_max > 0 && m1 > 0 && m1 <= head_max) {
                // split: the head after this GEMM and the next diagonal block
                // (side stream order), the rest here after both
                SIEB_TRY_CUDA(cudaEventRecord(st->ev_gemm, stream));
                SIEB_TRY_CUDA(cudaStreamWaitEvent(st->side, st->ev_gemm, 0));
                SIEB_RETURN_IF(panels(bk + 1, -1, -1, -1, st->side, 1));
                SIEB_TRY_CUDA(cudaEventRecord(st->ev_head, st->side));
                SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, st->ev_diag, 0));
                SIEB_RETURN_IF(panels(bk + 1, -1, -1, -1, stream, 2));
                head_prev = true;
                continue;
            }
            SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, st->ev_diag, 0));
            if (lside && m > n1) SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, st->ev_lcol, 0));
            // The next L21 rows take this step's update themselves unless
            // the GEMM or col_update_kernel applied it (lcol, lside); after
            // an even step of the pair schedule the next block row has not
            // had it either.
            SIEB_RETURN_IF(panels(bk + 1, (lcol || lside || lmain) ? -1 : k0, kprev, pair && !odd ? k0 : -1, stream,
                                  0));
        } else {
            trailing_simt_kernel<<<dim3(blocks_for(m, 64), blocks_for(m, 64)), 256, kSmemDiag, stream>>>(
                st->W, ldw, k0, kb, s0, np);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
            SIEB_RETURN_IF(diag_blk(bk + 1, -1, -1, stream));
            SIEB_RETURN_IF(panels(bk + 1, -1, -1, -1, stream, 0));
        }
    }
    // Join the side stream (its last panels or diagonal block).
    if (side_forked) {
        SIEB_TRY_CUDA(cudaEventRecord(st->ev_pan, st->side));
        SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, st->ev_pan, 0));
    }
    ctx->prof.end(stream, ev_fact);
    return SIEB200_OK;
}

// GMRES on a complex64 copy of Z: no factorization, the copy serves the
// Krylov products, the FP64 matrix the restart residuals, and the inverse
// diagonal of Z is the (right) preconditioner.
int gmres_c64_prepare(DenseSolver* s) {
    MixedState* st = state_of(s);
    if (!st) {
        st = new MixedState();
        s->gemm_state = st;
    }
    const int64_t n = s->n;
    st->n = n; st->np = n; st->ldw = n; st->nbl = 0;
    st->adj_ready = false;
    const size_t bW = ((sizeof(float2) * n * n + 255) / 256) * 256;
    const size_t bD = ((sizeof(cplx) * n + 255) / 256) * 256;
    SIEB_RETURN_IF(s->lu.reserve(bW + bD + 256));
    st->W = s->lu.as<float2>();
    st->dinv = reinterpret_cast<cplx*>(s->lu.as<char>() + bW);
    st->err = reinterpret_cast<unsigned*>(s->lu.as<char>() + bW + bD);
    cudaStream_t stream = s->ctx->stream;
    SIEB_TRY_CUDA(cudaMemsetAsync(st->err, 0, 256, stream));
    to_c64_kernel<<<dim3(blocks_for(n, 256), (unsigned)n), 256, 0, stream>>>(reinterpret_cast<const cplx*>(s->A),
                                                                             s->lda, n, st->W);
    SIEB_NOTE_LAUNCH();
    inv_diag_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(reinterpret_cast<const cplx*>(s->A), s->lda, n,
                                                            st->dinv);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

// Apply M^{-1} = V U^{-1} L^{-1} U^T (or its conjugate transpose) to r
// (length n) into z (length n).
static int apply_precond(DenseSolver* s, const cplx* r, cplx* z, cplx* work, bool adjoint) {
    MixedState* st = state_of(s);
    cudaStream_t stream = s->ctx->stream;
    const int64_t n = st->n, np = st->np, q = np / 4;
    const double* du = st->diag;
    const double* dv = st->diag + 4 * np;
    // Adjoint: (V W^{-1} U^T)^H = U W^{-H} V^T, with W^H = U^H L^H.
    const double* d_first = adjoint ? dv : du;
    const double* d_last = adjoint ? du : dv;
    rbt_vec_T_kernel<<<blocks_for(q, 256), 256, 0, stream>>>(r, n, np, d_first, work);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    unsigned* fl = st->tri_flags;
    const int nbl = (int)st->nbl;
    // Rows per triangular-solve CTA: 128 (two 64-row sub-blocks and their
    // coupling tiles) or 64 (SIEB200_TRSV_ROWS=64: one sub-block, twice the
    // CTAs, each hop one sub-block).
    const char* rows_env = getenv("SIEB200_TRSV_ROWS");
    const int rows = (rows_env && atoi(rows_env) == 64) ? NB : TR_ROWS;
    if (st->tm_rows != rows) {
        st->tm_base = nullptr;
        st->adj_ready = false;
        st->couple_ready[0] = st->couple_ready[1] = false;
        st->tm_rows = rows;
    }
    // 128-row CTAs fold the coupling to the newest sub-blocks into
    // precomputed products (trsv_fold_kernel; SIEB200_TRSV_FOLD=0 streams
    // those tiles as well, trsv_tma_kernel).
    const char* fold_env = getenv("SIEB200_TRSV_FOLD");
    const bool fold = rows == TR_ROWS && !(fold_env && fold_env[0] == '0');
    if (st->tm_base != st->W || st->tm_np != np) {
        // W as 8-byte elements: rows inner, 128 x 32 boxes; rows/columns
        // beyond np read as zero.
        SIEB_RETURN_IF(encode_tensor_map_2d(&st->tmW, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, st->W, (uint64_t)np,
                                            (uint64_t)np, (uint64_t)st->ldw * sizeof(float2), (uint32_t)rows,
                                            TR_COLS, CU_TENSOR_MAP_SWIZZLE_NONE));
        st->tm_base = st->W;
        st->tm_np = np;
    }
    if (adjoint && !st->adj_ready) {
        // W^H y = c is U^H (lower) then L^H (unit upper): the same two block
        // solves on the conjugate transpose of W, with the conjugate
        // transposes of the diagonal-block inverses.
        const size_t bW = ((sizeof(float2) * st->ldw * np + 255) / 256) * 256;
        const size_t bInv = sizeof(float2) * NB * NB * nbl;
        SIEB_RETURN_IF(s->panel.reserve(bW + 2 * bInv));
        st->WH = s->panel.as<float2>();
        st->LinvH = reinterpret_cast<float2*>(s->panel.as<char>() + bW);
        st->UinvH = st->LinvH + (size_t)NB * NB * nbl;
        conj_transpose_c64_kernel<<<dim3(blocks_for(np, 32), blocks_for(np, 32)), dim3(32, 8), 0, stream>>>(
            st->W, st->ldw, np, st->WH);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        conj_transpose_blocks_kernel<<<nbl, 256, 0, stream>>>(st->Linv, st->LinvH);
        SIEB_NOTE_LAUNCH();
        conj_transpose_blocks_kernel<<<nbl, 256, 0, stream>>>(st->Uinv, st->UinvH);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        SIEB_RETURN_IF(encode_tensor_map_2d(&st->tmWH, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, st->WH, (uint64_t)np,
                                            (uint64_t)np, (uint64_t)st->ldw * sizeof(float2), (uint32_t)rows,
                                            TR_COLS, CU_TENSOR_MAP_SWIZZLE_NONE));
        st->adj_ready = true;
    }
    static bool attr_set = false;
    if (!attr_set) {
        SIEB_TRY_CUDA(cudaFuncSetAttribute(trsv_tma_kernel<TR_ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           trsv_smem(TR_ROWS)));
        SIEB_TRY_CUDA(cudaFuncSetAttribute(trsv_tma_kernel<NB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           trsv_smem(NB)));
        SIEB_TRY_CUDA(cudaFuncSetAttribute(trsv_fold_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kSmemTrsvFold));
        SIEB_TRY_CUDA(cudaFuncSetAttribute(trsv_couple_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kSmemCouple));
        attr_set = true;
    }
    const unsigned ncta = (unsigned)((np + rows - 1) / rows);
    const unsigned long long timeout_ns = 2000000000ull;
    // algorithmic bytes: the triangle of c64 factors plus the diagonal inverses
    const double tri_bytes = 8.0 * (double)np * (double)np / 2.0 + 8.0 * NB * NB * nbl;
    SIEB_RETURN_IF(s->flags.reserve(sizeof(cplx) * (size_t)np));
    cplx* xpub = s->flags.as<cplx>();
    // Coupling products: [adjoint][lower] x (P1, P2) x nbl blocks, formed
    // once per factorization and direction.
    const size_t per_dir = (size_t)2 * nbl * NB * NB;
    auto couple_of = [&](int lower) { return s->couple.as<float2>() + ((adjoint ? 2 : 0) + lower) * per_dir; };
    if (fold && !st->couple_ready[adjoint ? 1 : 0]) {
        SIEB_RETURN_IF(s->couple.reserve(sizeof(float2) * per_dir * 4));
        for (int lower = 1; lower >= 0; --lower) {
            const float2* dinv = adjoint ? (lower ? st->UinvH : st->LinvH) : (lower ? st->Linv : st->Uinv);
            trsv_couple_kernel<<<dim3((unsigned)nbl, 2), 256, kSmemCouple, stream>>>(
                adjoint ? st->WH : st->W, st->ldw, np, nbl, lower, dinv, couple_of(lower));
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
        }
        st->couple_ready[adjoint ? 1 : 0] = true;
    }
    for (int lower = 1; lower >= 0; --lower) {
        const float2* dinv = adjoint ? (lower ? st->UinvH : st->LinvH) : (lower ? st->Linv : st->Uinv);
        SIEB_TRY_CUDA(cudaMemsetAsync(fl, 0, sizeof(unsigned) * 2, stream));
        SIEB_TRY_CUDA(cudaMemsetAsync(xpub, 0xFF, sizeof(cplx) * (size_t)np, stream));
        cudaEvent_t ev;
        s->ctx->prof.begin(stream, 1, 0.0, tri_bytes, &ev);
        if (fold)
            trsv_fold_kernel<<<ncta, TR_THREADS, kSmemTrsvFold, stream>>>(
                adjoint ? st->tmWH : st->tmW, np, nbl, lower, dinv, couple_of(lower), work, xpub, fl, st->err,
                timeout_ns);
        else if (rows == NB)
            trsv_tma_kernel<NB><<<ncta, TR_THREADS, trsv_smem(NB), stream>>>(
                adjoint ? st->tmWH : st->tmW, np, nbl, lower, dinv, work, xpub, fl, st->err, timeout_ns);
        else
            trsv_tma_kernel<TR_ROWS><<<ncta, TR_THREADS, trsv_smem(TR_ROWS), stream>>>(
                adjoint ? st->tmWH : st->tmW, np, nbl, lower, dinv, work, xpub, fl, st->err, timeout_ns);
        SIEB_NOTE_LAUNCH();
        s->ctx->prof.end(stream, ev);
        SIEB_TRY_CUDA(cudaGetLastError());
    }
    rbt_vec_N_kernel<<<blocks_for(q, 256), 256, 0, stream>>>(work, n, np, d_last, z);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}


// Restarted flexible GMRES on A x = b or A^H x = b (FP64, A the intact complex128 matrix)
// with right preconditioner M^{-1}, started from x = 0. The preconditioned
// directions z_j = M^{-1} v_j are kept, so the update x += Z y costs no
// further preconditioner application.
double gmres_est_factor() {
    const char* e = getenv("SIEB200_GMRES_EST_FACTOR");
    const double f = e ? atof(e) : kGmresEstFactorDefault;
    return (f > 0.0 && f <= 1.0) ? f : kGmresEstFactorDefault;
}

static int gmres_ir(DenseSolver* s, cplx* b, int64_t ldb_unused, double tol, int maxit, bool adjoint,
                    int* iters) {
    (void)ldb_unused;
    MixedState* st = state_of(s);
    sieb200_ctx* ctx = s->ctx;
    cudaStream_t stream = ctx->stream;
    const int64_t n = st->n, np = st->np;
    // Restart length: the whole iteration budget up to 100 directions (V and
    // Z together hold 2 n m complex128); restarts slow FGMRES down sharply on
    // ill-conditioned systems.
    const int m = std::max(1, std::min(maxit, 100));
    const int parts = 64;
    // vectors: x, r, w, work(np), V (n x (m+1)), Z (n x m), partial, h
    // h: two CGS passes of up to m + 1 coefficients each and ||w||^2
    const size_t vbytes =
        sizeof(cplx) * (4 * np + (int64_t)(m + 1) * n + (int64_t)m * n + parts * (m + 1) + (2 * m + 4));
    SIEB_RETURN_IF(s->krylov.reserve(vbytes));
    cplx* x = s->krylov.as<cplx>();
    cplx* r = x + np;
    cplx* w = r + np;
    cplx* work = w + np;
    cplx* V = work + np;
    cplx* Zb = V + (int64_t)(m + 1) * n;
    cplx* partial = Zb + (int64_t)m * n;
    cplx* h = partial + parts * (m + 1);
    const double* A = s->A;
    const int64_t lda = s->lda;

    // ||b|| is the first residual norm (x0 = 0), read with it below.
    double bnorm = 0.0;
    const double est_factor = gmres_est_factor();

    SIEB_TRY_CUDA(cudaMemsetAsync(x, 0, sizeof(cplx) * n, stream));
    int total = 0;
    std::vector<cplx> H((size_t)(m + 1) * m), g(m + 1), cs(m), sn(m), hh(2 * m + 4);
    for (int outer = 0; outer < 1000; ++outer) {
        // r = A x - b (for x = 0 simply -b)
        if (outer == 0) {
            scale_copy_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, b, -1.0, r);
            SIEB_NOTE_LAUNCH();
        } else {
            SIEB_TRY_CUDA(cudaMemcpyAsync(r, b, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, stream));
            if (adjoint)
                SIEB_RETURN_IF(gemv_h_device(ctx, n, A, lda, x, -1.0, r));
            else
                SIEB_RETURN_IF(gemv_device(ctx, n, A, lda, 0, x, -1.0, r, s->gemv_scratch));
        }
        dot_partial_kernel<<<dim3(parts, 1), 256, 0, stream>>>(n, 1, r, n, r, partial);
        SIEB_NOTE_LAUNCH();
        dot_finish_kernel<<<1, 32, 0, stream>>>(1, parts, partial, h);
        SIEB_NOTE_LAUNCH();
        cplx rr;
        SIEB_TRY_CUDA(cudaMemcpyAsync(&rr, h, sizeof(cplx), cudaMemcpyDeviceToHost, stream));
        SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
        const double beta = std::sqrt(std::max(rr.re, 0.0));
        if (outer == 0) {
            bnorm = beta;
            SIEB_CHECK(bnorm > 0 && std::isfinite(bnorm), SIEB200_INVALID_ARG,
                       "right-hand side norm must be finite and nonzero");
        }
        if (!std::isfinite(beta)) {
            set_error("GMRES refinement produced a non-finite residual");
            return SIEB200_NONFINITE;
        }
        if (beta <= tol * bnorm) break;
        if (total >= maxit) {
            if (iters) *iters = total;
            set_error("GMRES refinement did not reach the tolerance within max_iterations");
            return SIEB200_NOT_CONVERGED;
        }
        // r holds A x - b: v1 = -r / beta
        scale_copy_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, r, -1.0 / beta, V);
        SIEB_NOTE_LAUNCH();
        std::fill(g.begin(), g.end(), cx(0, 0));
        g[0] = cx(beta, 0);
        int j = 0;
        double est = beta;
        for (; j < m && total < maxit; ++j, ++total) {
            cplx* vj = V + (int64_t)j * n;
            cplx* zj = Zb + (int64_t)j * n;
            if (s->method == SIEB200_SOLVER_GMRES_C64) {
                // Jacobi preconditioner; Krylov products with the complex64 copy
                diag_scale_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, st->dinv, vj, adjoint ? 1 : 0, zj);
                SIEB_NOTE_LAUNCH();
                if (adjoint)
                    SIEB_RETURN_IF(gemv_h_device(ctx, n, A, lda, zj, 0.0, w));
                else
                    SIEB_RETURN_IF(gemv_device(ctx, n, st->W, n, 1, zj, 0.0, w, s->gemv_scratch));
            } else {
                SIEB_RETURN_IF(apply_precond(s, vj, zj, work, adjoint));
                if (adjoint)
                    SIEB_RETURN_IF(gemv_h_device(ctx, n, A, lda, zj, 0.0, w));
                else
                    SIEB_RETURN_IF(gemv_device(ctx, n, A, lda, 0, zj, 0.0, w, s->gemv_scratch));
            }
            // Classical Gram-Schmidt with one reorthogonalization (CGS2): the
            // two passes' coefficients (h, h + j + 1) and ||w||^2 (h + 2j + 2)
            // stay on the device and come back in one copy.
            const int fin_threads = std::min(1024, ((j + 1 + 31) / 32) * 32);
            for (int pass = 0; pass < 2; ++pass) {
                cplx* hp = h + pass * (j + 1);
                dot_partial_kernel<<<dim3(parts, j + 1), 256, 0, stream>>>(n, j + 1, V, n, w, partial);
                SIEB_NOTE_LAUNCH();
                dot_finish_kernel<<<1, fin_threads, 0, stream>>>(j + 1, parts, partial, hp);
                SIEB_NOTE_LAUNCH();
                axpy_multi_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, j + 1, V, n, hp, w);
                SIEB_NOTE_LAUNCH();
                SIEB_TRY_CUDA(cudaGetLastError());
            }
            dot_partial_kernel<<<dim3(parts, 1), 256, 0, stream>>>(n, 1, w, n, w, partial);
            SIEB_NOTE_LAUNCH();
            dot_finish_kernel<<<1, 32, 0, stream>>>(1, parts, partial, h + 2 * (j + 1));
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaMemcpyAsync(hh.data(), h, sizeof(cplx) * (2 * (j + 1) + 1), cudaMemcpyDeviceToHost,
                                          stream));
            SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
            for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = hh[i] + hh[j + 1 + i];
            const cplx ww = hh[2 * (j + 1)];
            const double hn = std::sqrt(std::max(ww.re, 0.0));
            cplx hj1 = cx(hn, 0);
            if (j + 1 <= m) {
                scale_copy_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, w, hn > 0 ? 1.0 / hn : 0.0,
                                                                           V + (int64_t)(j + 1) * n);
                SIEB_NOTE_LAUNCH();
            }
            // Givens on column j
            for (int i = 0; i < j; ++i) {
                const cplx a = H[(size_t)i * m + j], bb = H[(size_t)(i + 1) * m + j];
                // [c s; -conj(s) c] with real c
                const cplx t1 = cx(cs[i].re * a.re + (sn[i] * bb).re, cs[i].re * a.im + (sn[i] * bb).im);
                const cplx conj_s = cx(sn[i].re, -sn[i].im);
                const cplx t2 = cx(-(conj_s * a).re + cs[i].re * bb.re, -(conj_s * a).im + cs[i].re * bb.im);
                H[(size_t)i * m + j] = t1;
                H[(size_t)(i + 1) * m + j] = t2;
            }
            const cplx a = H[(size_t)j * m + j];
            const double an = std::hypot(a.re, a.im), bn = hn;
            const double den = std::hypot(an, bn);
            if (den == 0.0) { cs[j] = cx(1, 0); sn[j] = cx(0, 0); }
            else if (an == 0.0) { cs[j] = cx(0, 0); sn[j] = cx(1, 0); }
            else {
                cs[j] = cx(an / den, 0);
                // s = (a/|a|) * conj(b) / den with b = hn real
                sn[j] = cx(a.re / an * bn / den, a.im / an * bn / den);
            }
            H[(size_t)j * m + j] = cx(cs[j].re * a.re + sn[j].re * hn, cs[j].re * a.im + sn[j].im * hn);
            (void)hj1;
            const cplx gj = g[j];
            const cplx conj_s = cx(sn[j].re, -sn[j].im);
            g[j] = cx(cs[j].re * gj.re, cs[j].re * gj.im);
            g[j + 1] = cx(-(conj_s * gj).re, -(conj_s * gj).im);
            est = std::hypot(g[j + 1].re, g[j + 1].im);
            if (est <= est_factor * tol * bnorm || hn == 0.0) { ++j; ++total; break; }
        }
        // y = H^{-1} g (upper triangular j x j)
        std::vector<cplx> y(j);
        for (int i = j - 1; i >= 0; --i) {
            cplx sacc = g[i];
            for (int k = i + 1; k < j; ++k) sacc = sacc - H[(size_t)i * m + k] * y[k];
            const cplx d = H[(size_t)i * m + i];
            const double dd = d.re * d.re + d.im * d.im;
            y[i] = cx((sacc.re * d.re + sacc.im * d.im) / dd, (sacc.im * d.re - sacc.re * d.im) / dd);
        }
        SIEB_TRY_CUDA(cudaMemcpyAsync(h, y.data(), sizeof(cplx) * j, cudaMemcpyHostToDevice, stream));
        combo_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, j, Zb, n, h, w);
        SIEB_NOTE_LAUNCH();
        add_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(n, w, x);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        SIEB_RETURN_IF(check_err(s, "GMRES refinement"));
    }
    SIEB_TRY_CUDA(cudaMemcpyAsync(b, x, sizeof(cplx) * n, cudaMemcpyDeviceToDevice, stream));
    if (iters) *iters = total;
    return check_err(s, "GMRES refinement");
}

static int fp64_solve(DenseSolver* s, int64_t nrhs, double* B, int64_t ldb, double tol, int maxit, int* iters);

int mixed_solve(DenseSolver* s, int64_t nrhs, double* B, int64_t ldb, bool adjoint, double tol,
                int maxit, int* iters) {
    if (s->method == SIEB200_SOLVER_LU_FP64) {
        SIEB_CHECK(!adjoint, SIEB200_INVALID_ARG,
                   "conjugate-transpose solves use the mixed or the cuSOLVER method, not the own FP64 LU");
        return fp64_solve(s, nrhs, B, ldb, tol, maxit, iters);
    }
    SIEB_CHECK(s->method == SIEB200_SOLVER_MIXED_IR || s->method == SIEB200_SOLVER_GMRES_C64, SIEB200_INVALID_ARG,
               "unsupported solver method");
    if (!(tol > 0)) tol = 1e-10;
    if (maxit <= 0) maxit = 50;
    MixedState* st = state_of(s);
    const char* per_column = getenv("SIEB200_PER_COLUMN_SOLVE");
    if (nrhs >= 2 && !adjoint && s->method == SIEB200_SOLVER_MIXED_IR && st && st->use_tc &&
        !(per_column && per_column[0] == '1')) {
        // All columns together (tensor-core block triangular solves, batched
        // FGMRES); -1: the packed factors do not fit, solve column by column.
        cudaEvent_t ev;
        s->ctx->prof.begin(s->ctx->stream, 7, 0.0, 0.0, &ev);
        const int rc = block_solve(s, st, nrhs, B, ldb, tol, maxit, iters);
        s->ctx->prof.end(s->ctx->stream, ev);
        if (rc != -1) return rc;
    }
    int total = 0;
    for (int64_t c = 0; c < nrhs; ++c) {
        int it = 0;
        cudaEvent_t ev;
        s->ctx->prof.begin(s->ctx->stream, 7, 0.0, 0.0, &ev);
        const int st = gmres_ir(s, reinterpret_cast<cplx*>(B) + c * ldb, ldb, tol, maxit, adjoint, &it);
        s->ctx->prof.end(s->ctx->stream, ev);
        total = std::max(total, it);
        if (st != SIEB200_OK) {
            if (iters) *iters = total;
            return st;
        }
    }
    if (iters) *iters = total;
    return SIEB200_OK;
}

// ------------------------------------------------------------ own FP64 LU
// SIEB200_SOLVER_LU_FP64: the drop-in for the reference's cusolverDnZgetrf /
// Zgetrs path (include/sie_mom/cuda/dense_lu_solver.cuh:42-166) built from
// this library's own kernels, all in complex128: the butterfly transform
// W = U^T A V (A is left intact), blocked LU of W without pivoting (the
// transform makes pivoting unnecessary with high probability; a zero or
// non-finite pivot is reported as SIEB200_SINGULAR), the diagonal blocks and
// both triangular inverses by diag_lu_kernel<double2>, the panels by
// panels_kernel<double2>, the trailing update C -= L21 U12 by the FP64
// complex GEMM (zgemm_device), with the same one-block lookahead on a side
// stream as the mixed factorization. A solve applies V U^{-1} L^{-1} U^T
// (blocked triangular solves: diagonal inverses plus FP64 GEMM updates) and
// refines against the intact A in FP64 until the relative residual of every
// column is <= tol (one correction at most, in practice).
static int fp64_factorize(DenseSolver* s) {
    sieb200_ctx* ctx = s->ctx;
    cudaStream_t stream = ctx->stream;
    MixedState* st = state_of(s);
    if (!st) {
        st = new MixedState();
        s->gemm_state = st;
    }
    const int64_t n = s->n;
    const int64_t np = ((n + 3) / 4) * 4;
    const int64_t ldw = ((np + 31) / 32) * 32;
    const int64_t nbl = (np + NB - 1) / NB;
    st->n = n; st->np = np; st->ldw = ldw; st->nbl = nbl;
    st->adj_ready = false;
    block_solve_invalidate(st);
    auto up = [](size_t b) { return ((b + 255) / 256) * 256; };
    const size_t bW = sizeof(double2) * ldw * np;
    const size_t bInv = sizeof(double2) * NB * NB * nbl;
    const size_t bDiag = sizeof(double) * 8 * np;
    const size_t bFlags = sizeof(unsigned) * 16;
    SIEB_RETURN_IF(s->lu.reserve(up(bW) + 2 * up(bInv) + up(bDiag) + up(bFlags)));
    char* base = s->lu.as<char>();
    st->W64 = reinterpret_cast<double2*>(base);
    st->Linv64 = reinterpret_cast<double2*>(base + up(bW));
    st->Uinv64 = reinterpret_cast<double2*>(base + up(bW) + up(bInv));
    st->diag = reinterpret_cast<double*>(base + up(bW) + 2 * up(bInv));
    st->err = reinterpret_cast<unsigned*>(base + up(bW) + 2 * up(bInv) + up(bDiag));
    st->diag_split = diag_split_env();
    st->diag_panels = diag_panels_env();
    st->diag_compact = diag_compact_env();
    st->diag_rec = 0;  // complex64 only
    if (!st->side) {
        int least = 0, greatest = 0;
        SIEB_TRY_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        SIEB_TRY_CUDA(cudaStreamCreateWithPriority(&st->side, cudaStreamNonBlocking, greatest));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_cols, cudaEventDisableTiming));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_diag, cudaEventDisableTiming));
        SIEB_TRY_CUDA(cudaEventCreateWithFlags(&st->ev_pan, cudaEventDisableTiming));
    }
    static bool attrs64 = false;
    if (!attrs64) {
        SIEB_TRY_CUDA(cudaFuncSetAttribute(panels_kernel<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           kSmemPanel64));
        SIEB_RETURN_IF(diag_set_smem<double2>(kSmemDiagUpd64));
        attrs64 = true;
    }
    cudaEvent_t ev_fact;
    ctx->prof.begin(stream, 6, (8.0 / 3.0) * (double)np * np * np, 0.0, &ev_fact);
    SIEB_TRY_CUDA(cudaMemsetAsync(st->err, 0, bFlags, stream));
    rbt_init_kernel<<<blocks_for(8 * np, 256), 256, 0, stream>>>(st->diag, np, 0x5EB200ull);
    SIEB_NOTE_LAUNCH();
    const int64_t q = np / 4;
    rbt_matrix_kernel<double2><<<dim3(blocks_for(q, 128), (unsigned)q), 128, 0, stream>>>(
        reinterpret_cast<const cplx*>(s->A), s->lda, n, np, st->diag, st->diag + 4 * np, st->W64, ldw);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    auto diag_blk = [&](int64_t bk, int64_t kp, cudaStream_t sm) -> int {
        const int64_t k0 = bk * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        cudaEvent_t ev;
        ctx->prof.begin(sm, 3, (16.0 / 3.0) * NB * NB * NB + (kp >= 0 ? 8.0 * NB * NB * NB : 0.0), 0.0, &ev);
        if (kp >= 0 && st->diag_split) {
            diag_update_kernel<double2><<<dim3(NB / 16, NB / 16), 256, 0, sm>>>(st->W64, ldw, k0, kb, kp, -1);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
            kp = -1;
        }
        diag_kernel_for<double2>(st)<<<1, kDiagThreads, kSmemDiagUpd64, sm>>>(
            st->W64, ldw, k0, kb, st->Linv64 + (size_t)bk * NB * NB, st->Uinv64 + (size_t)bk * NB * NB, st->err, kp,
            -1);
        SIEB_NOTE_LAUNCH();
        ctx->prof.end(sm, ev);
        SIEB_TRY_CUDA(cudaGetLastError());
        return SIEB200_OK;
    };
    auto panels = [&](int64_t bk, int64_t kp) -> int {
        const int64_t k0 = bk * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        const int64_t s0 = k0 + kb;
        if (s0 >= np) return SIEB200_OK;
        const int64_t m = np - s0;
        const int nL = (int)blocks_for(m, 32);
        cudaEvent_t ev;
        ctx->prof.begin(stream, 4, 8.0 * NB * NB * (double)m * (kp >= 0 ? 2.0 : 1.0), 0.0, &ev);
        PanelArgs pa;
        pa.k0 = k0; pa.kb = kb; pa.s0 = s0; pa.np = np; pa.nL = nL; pa.pack = 0;
        pa.kp[0] = kp;
        panels_kernel<double2><<<(unsigned)(2 * nL), 256, kSmemPanel64, stream>>>(
            st->W64, ldw, st->Uinv64 + (size_t)bk * NB * NB, st->Linv64 + (size_t)bk * NB * NB, pa);
        SIEB_NOTE_LAUNCH();
        ctx->prof.end(stream, ev);
        SIEB_TRY_CUDA(cudaGetLastError());
        return SIEB200_OK;
    };
    SIEB_RETURN_IF(diag_blk(0, -1, stream));
    SIEB_RETURN_IF(panels(0, -1));
    cplx* W = reinterpret_cast<cplx*>(st->W64);
    for (int64_t bk = 0; bk < nbl; ++bk) {
        const int64_t k0 = bk * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        const int64_t s0 = k0 + kb;
        if (s0 >= np) break;
        const int64_t m = np - s0;
        const int64_t n1 = std::min<int64_t>(NB, m);
        SIEB_TRY_CUDA(cudaEventRecord(st->ev_cols, stream));
        SIEB_TRY_CUDA(cudaStreamWaitEvent(st->side, st->ev_cols, 0));
        SIEB_RETURN_IF(diag_blk(bk + 1, k0, st->side));
        SIEB_TRY_CUDA(cudaEventRecord(st->ev_diag, st->side));
        if (m > n1) {
            cudaEvent_t ev;
            ctx->prof.begin(stream, 0, 8.0 * (double)m * (double)(m - n1) * kb,
                            16.0 * (2.0 * (double)m * (m - n1) + (double)(m + m - n1) * kb), &ev);
            SIEB_RETURN_IF(zgemm_device(stream, m, m - n1, kb, W + s0 + k0 * ldw, ldw, W + k0 + (s0 + n1) * ldw, ldw,
                                        W + s0 + (s0 + n1) * ldw, ldw, cx(-1, 0), cx(1, 0)));
            ctx->prof.end(stream, ev);
        }
        SIEB_TRY_CUDA(cudaStreamWaitEvent(stream, st->ev_diag, 0));
        SIEB_RETURN_IF(panels(bk + 1, k0));
    }
    ctx->prof.end(stream, ev_fact);
    unsigned e = 0;
    SIEB_TRY_CUDA(cudaMemcpyAsync(&e, st->err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
    if (e != 0u) {
        set_error("own FP64 LU: zero or non-finite pivot in a diagonal block (the matrix is singular or the "
                  "butterfly transform met an unlucky pivot)");
        return SIEB200_SINGULAR;
    }
    return SIEB200_OK;
}

// Y (np x nrhs, ldy) <- W^{-1} Y with the complex128 factors.
static int fp64_triangular(DenseSolver* s, MixedState* st, cplx* Y, int64_t ldy, int nrhs) {
    cudaStream_t stream = s->ctx->stream;
    const int64_t np = st->np, nbl = st->nbl, ldw = st->ldw;
    const cplx* W = reinterpret_cast<const cplx*>(st->W64);
    const unsigned g = blocks_for(nrhs, 16);
    for (int64_t k = 0; k < nbl; ++k) {
        const int64_t k0 = k * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        fp64_diag_apply_kernel<<<g, 256, 0, stream>>>(Y, ldy, k0, kb, nrhs, st->Linv64 + (size_t)k * NB * NB);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        const int64_t s0 = k0 + kb;
        if (s0 < np)
            SIEB_RETURN_IF(zgemm_device(stream, np - s0, nrhs, kb, W + s0 + k0 * ldw, ldw, Y + k0, ldy, Y + s0, ldy,
                                        cx(-1, 0), cx(1, 0)));
    }
    for (int64_t k = nbl - 1; k >= 0; --k) {
        const int64_t k0 = k * NB;
        const int kb = (int)std::min<int64_t>(NB, np - k0);
        fp64_diag_apply_kernel<<<g, 256, 0, stream>>>(Y, ldy, k0, kb, nrhs, st->Uinv64 + (size_t)k * NB * NB);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        if (k0 > 0)
            SIEB_RETURN_IF(zgemm_device(stream, k0, nrhs, kb, W + k0 * ldw, ldw, Y + k0, ldy, Y, ldy, cx(-1, 0),
                                        cx(1, 0)));
    }
    return SIEB200_OK;
}

static int fp64_solve(DenseSolver* s, int64_t nrhs64, double* Bd, int64_t ldb, double tol, int maxit, int* iters) {
    MixedState* st = state_of(s);
    SIEB_CHECK(st && st->W64, SIEB200_INVALID_ARG, "own FP64 LU: factorize() has not run");
    sieb200_ctx* ctx = s->ctx;
    cudaStream_t stream = ctx->stream;
    const int nrhs = (int)nrhs64;
    const int64_t n = st->n, np = st->np, q = np / 4;
    const int64_t ldy = ((np + 31) / 32) * 32;
    if (!(tol > 0)) tol = 1e-10;
    if (maxit <= 0) maxit = 5;
    // Y (ldy x nrhs) | X | R | B0 (n x nrhs each)
    const size_t blk = (size_t)n * nrhs;
    SIEB_RETURN_IF(s->krylov.reserve(sizeof(cplx) * ((size_t)ldy * nrhs + 3 * blk)));
    cplx* Y = s->krylov.as<cplx>();
    cplx* X = Y + (size_t)ldy * nrhs;
    cplx* R = X + blk;
    cplx* B0 = R + blk;
    cplx* B = reinterpret_cast<cplx*>(Bd);
    const dim3 gv(blocks_for(n, 256), (unsigned)nrhs);
    copy_cols_kernel<<<gv, 256, 0, stream>>>(n, B, ldb, B0, n);
    SIEB_NOTE_LAUNCH();
    copy_cols_kernel<<<gv, 256, 0, stream>>>(n, B, ldb, R, n);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaMemsetAsync(X, 0, sizeof(cplx) * blk, stream));
    std::vector<cplx> hb(blk);
    SIEB_TRY_CUDA(cudaMemcpyAsync(hb.data(), B0, sizeof(cplx) * blk, cudaMemcpyDeviceToHost, stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
    std::vector<double> bnorm(nrhs);
    for (int c = 0; c < nrhs; ++c) {
        long double acc = 0;
        for (int64_t i = 0; i < n; ++i) {
            const cplx v = hb[(size_t)c * n + i];
            acc += (long double)v.re * v.re + (long double)v.im * v.im;
        }
        bnorm[c] = std::sqrt((double)acc);
        SIEB_CHECK(bnorm[c] > 0 && std::isfinite(bnorm[c]), SIEB200_INVALID_ARG,
                   "right-hand side norm must be finite and nonzero");
    }
    int it = 0;
    std::vector<cplx> hr(blk);
    for (;;) {
        // correction D = V W^{-1} U^T R, X += D
        for (int c = 0; c < nrhs; ++c) {
            rbt_vec_T_kernel<<<blocks_for(q, 256), 256, 0, stream>>>(R + (size_t)c * n, n, np, st->diag,
                                                                     Y + (size_t)c * ldy);
            SIEB_NOTE_LAUNCH();
        }
        cudaEvent_t ev;
        ctx->prof.begin(stream, 1, 0.0, 16.0 * (double)np * np, &ev);
        SIEB_RETURN_IF(fp64_triangular(s, st, Y, ldy, nrhs));
        ctx->prof.end(stream, ev);
        for (int c = 0; c < nrhs; ++c) {
            rbt_vec_N_kernel<<<blocks_for(q, 256), 256, 0, stream>>>(Y + (size_t)c * ldy, n, np, st->diag + 4 * np,
                                                                     R + (size_t)c * n);
            SIEB_NOTE_LAUNCH();
        }
        add_cols_kernel<<<gv, 256, 0, stream>>>(n, R, n, X, n);
        SIEB_NOTE_LAUNCH();
        ++it;
        // R = B - A X in FP64 against the intact matrix
        copy_cols_kernel<<<gv, 256, 0, stream>>>(n, B0, n, R, n);
        SIEB_NOTE_LAUNCH();
        ctx->prof.begin(stream, 2, 8.0 * (double)n * n * nrhs, 16.0 * (double)n * n, &ev);
        SIEB_RETURN_IF(zgemm_device(stream, n, nrhs, n, reinterpret_cast<const cplx*>(s->A), s->lda, X, n, R, n,
                                    cx(-1, 0), cx(1, 0)));
        ctx->prof.end(stream, ev);
        SIEB_TRY_CUDA(cudaMemcpyAsync(hr.data(), R, sizeof(cplx) * blk, cudaMemcpyDeviceToHost, stream));
        SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
        bool done = true;
        for (int c = 0; c < nrhs && done; ++c) {
            long double acc = 0;
            for (int64_t i = 0; i < n; ++i) {
                const cplx v = hr[(size_t)c * n + i];
                acc += (long double)v.re * v.re + (long double)v.im * v.im;
            }
            const double rn = std::sqrt((double)acc);
            if (!std::isfinite(rn)) {
                set_error("own FP64 LU produced a non-finite residual");
                return SIEB200_NONFINITE;
            }
            done = rn <= tol * bnorm[c];
        }
        if (done) break;
        if (it >= maxit) {
            copy_cols_kernel<<<gv, 256, 0, stream>>>(n, X, n, B, ldb);
            SIEB_NOTE_LAUNCH();
            if (iters) *iters = it;
            set_error("own FP64 LU refinement did not reach the tolerance within max_iterations");
            return SIEB200_NOT_CONVERGED;
        }
    }
    copy_cols_kernel<<<gv, 256, 0, stream>>>(n, X, n, B, ldb);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    if (iters) *iters = it;
    return SIEB200_OK;
}

}  // namespace sieb200
