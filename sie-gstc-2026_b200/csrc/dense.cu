// Dense complex linear algebra on the context stream: the reference's
// cuSolverDn LU (include/sie_mom/cuda/dense_lu_solver.cuh:17-184), the
// FP64 matvec that replaces its cublasZgemv residual
// (src/sie_mom/solvers/gstc_sie.cu:398-457), and the solver object that
// dispatches to the mixed-precision path (mixed.cu).

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cusolverDn.h>

#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "dense.cuh"
#include "sm100.cuh"

namespace sieb200 {

namespace {

// y = A x (+ beta y). Column-major A, one thread per row, a column chunk per
// grid.y; deterministic two-pass reduction over chunks.
template <class TA>
__global__ void gemv_partial_kernel(int64_t n, const TA* __restrict__ A, int64_t lda,
                                    const cplx* __restrict__ x, int64_t cols_per_chunk,
                                    cplx* __restrict__ partial) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c0 = (int64_t)blockIdx.y * cols_per_chunk;
    const int64_t c1 = min(n, c0 + cols_per_chunk);
    if (i >= n) return;
    double re = 0.0, im = 0.0;
    int64_t c = c0;
    for (; c + 4 <= c1; c += 4) {
        TA a[4];
        cplx xv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a[u] = A[i + (c + u) * lda];
            xv[u] = x[c + u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double ar = (double)a[u].x, ai = (double)a[u].y;
            re += ar * xv[u].re - ai * xv[u].im;
            im += ar * xv[u].im + ai * xv[u].re;
        }
    }
    for (; c < c1; ++c) {
        const TA a = A[i + c * lda];
        const cplx xv = x[c];
        re += (double)a.x * xv.re - (double)a.y * xv.im;
        im += (double)a.x * xv.im + (double)a.y * xv.re;
    }
    partial[(int64_t)blockIdx.y * n + i] = cx(re, im);
}

__global__ void gemv_finish_kernel(int64_t n, int chunks, const cplx* __restrict__ partial,
                                   double beta, cplx* __restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    cplx s = beta != 0.0 ? y[i] * beta : cx(0, 0);
    for (int k = 0; k < chunks; ++k) s += partial[(int64_t)k * n + i];
    y[i] = s;
}

// y = A^H x (+ beta y): one warp per output entry, reading column i of the
// column-major A contiguously; FP64 accumulation, warp-shuffle reduction.
template <class TA>
__global__ void gemv_h_kernel(int64_t n, const TA* __restrict__ A, int64_t lda, const cplx* __restrict__ x,
                              double beta, cplx* __restrict__ y) {
    const int64_t i = (int64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= n) return;  // warp-uniform
    const TA* col = A + i * lda;
    double re = 0.0, im = 0.0;
    for (int64_t k = lane; k < n; k += 32) {
        const TA a = col[k];
        const cplx xv = x[k];
        // conj(a) * x
        re += (double)a.x * xv.re + (double)a.y * xv.im;
        im += (double)a.x * xv.im - (double)a.y * xv.re;
    }
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    if (lane == 0) {
        const cplx old = beta != 0.0 ? y[i] * beta : cx(0, 0);
        y[i] = cx(old.re + re, old.im + im);
    }
}

// y = A x, TMA-staged. Each CTA owns GV_ROWS rows and one column chunk; a
// producer warp streams 16 KB tiles (GV_ROWS rows x the chunk's next CB
// columns, one cp.async.bulk.tensor per tile) and the CB entries of x they
// multiply (one cp.async.bulk) through a GV_STAGES-deep ring in shared
// memory, and each of the GV_ROWS consumer threads accumulates its row from
// the tiles in FP64, in the same column order as gemv_partial_kernel. The tensor map views A as reals: inner extent 2n
// (re, im of n rows), outer extent n columns, row stride lda elements.
// Every wait is bounded: past timeout_ns the CTA stops streaming and writes
// NaN partial sums, so the caller's residual shows the failure.
constexpr int GV_ROWS = 128;
constexpr int GV_STAGES = 6;
constexpr int GV_TILE_BYTES = 16384;
constexpr int GV_THREADS = GV_ROWS + 32;
constexpr int GV_XSLOT = 256;  // bytes of x per stage (16 complex128 at most)
constexpr int GV_SMEM = GV_STAGES * (GV_TILE_BYTES + GV_XSLOT) + 1024;

__device__ __forceinline__ bool gv_wait(uint32_t bar, uint32_t parity, uint64_t deadline) {
    int it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if ((++it & 255) == 0 && global_ns() > deadline) return false;
    }
    return true;
}

template <class TA>
__global__ void __launch_bounds__(GV_THREADS, 2)
gemv_tma_kernel(const __grid_constant__ CUtensorMap tmA, int64_t n, const cplx* __restrict__ x,
                int64_t cols_per_chunk, cplx* __restrict__ partial, unsigned long long timeout_ns) {
    constexpr int CB = GV_TILE_BYTES / (GV_ROWS * (int)sizeof(TA));  // columns per tile
    extern __shared__ __align__(16) unsigned char gv_smem[];
    const uint32_t raw = smem_u32(gv_smem);
    unsigned char* base = gv_smem + (((raw + 1023u) & ~1023u) - raw);
    const uint32_t ring = smem_u32(base);
    const uint32_t xring = ring + GV_STAGES * GV_TILE_BYTES;
    static_assert(CB * (int)sizeof(cplx) <= GV_XSLOT, "x slot");
    __shared__ __align__(8) uint64_t bars[2 * GV_STAGES];
    __shared__ volatile int s_abort;
    const uint32_t full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[GV_STAGES]);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t i0 = (int64_t)blockIdx.x * GV_ROWS;
    const int64_t c0 = (int64_t)blockIdx.y * cols_per_chunk;
    const int64_t c1 = min(n, c0 + cols_per_chunk);
    const int ntile = (int)((c1 - c0 + CB - 1) / CB);
    if (tid == 0) {
        s_abort = 0;
        for (int st = 0; st < GV_STAGES; ++st) {
            mbar_init(full0 + 8 * st, 1);
            mbar_init(empty0 + 8 * st, GV_ROWS / 32);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    const uint64_t deadline = global_ns() + timeout_ns;

    if (warp == GV_ROWS / 32) {  // producer
        if (lane == 0) {
            for (int i = 0; i < ntile; ++i) {
                const int st = i % GV_STAGES;
                const uint32_t ph = (uint32_t)(i / GV_STAGES) & 1u;
                if (!gv_wait(empty0 + 8 * st, ph ^ 1u, deadline)) {
                    s_abort = 1;
                    break;
                }
                const int64_t cb = c0 + (int64_t)i * CB;
                const uint32_t xbytes = (uint32_t)(min((int64_t)CB, c1 - cb) * (int64_t)sizeof(cplx));
                mbar_expect_tx(full0 + 8 * st, GV_TILE_BYTES + xbytes);
                tma_load_2d(ring + st * GV_TILE_BYTES, &tmA, full0 + 8 * st, (int)(2 * i0), (int)cb);
                bulk_load_1d(xring + st * GV_XSLOT, x + cb, xbytes, full0 + 8 * st);
            }
        }
        return;
    }

    double re = 0.0, im = 0.0;
    bool ok = true;
    for (int i = 0; i < ntile; ++i) {
        const int st = i % GV_STAGES;
        const uint32_t ph = (uint32_t)(i / GV_STAGES) & 1u;
        if (s_abort || !gv_wait(full0 + 8 * st, ph, deadline)) {
            ok = false;
            break;
        }
        const TA* tile = reinterpret_cast<const TA*>(base + st * GV_TILE_BYTES);
        const cplx* xs = reinterpret_cast<const cplx*>(base + GV_STAGES * GV_TILE_BYTES + st * GV_XSLOT);
        const int64_t cb = c0 + (int64_t)i * CB;
        const int ncol = (int)min((int64_t)CB, c1 - cb);
#pragma unroll 4
        for (int j = 0; j < ncol; ++j) {
            const TA a = tile[j * GV_ROWS + tid];
            const cplx xv = xs[j];
            const double ar = (double)a.x, ai = (double)a.y;
            re += ar * xv.re - ai * xv.im;
            im += ar * xv.im + ai * xv.re;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(empty0 + 8 * st);
    }
    if (i0 + tid < n) {
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        partial[(int64_t)blockIdx.y * n + i0 + tid] = ok ? cx(re, im) : cx(nan, nan);
    }
}

template <class TA>
int gemv_tma_launch(sieb200_ctx* ctx, const CUtensorMap* tm, int64_t n, const cplx* x, int64_t cpc, int chunks,
                    cplx* partial) {
    static bool attr_set[64] = {};  // per device
    const int dev = ctx->device & 63;
    if (!attr_set[dev]) {
        SIEB_TRY_CUDA(cudaFuncSetAttribute(gemv_tma_kernel<TA>, cudaFuncAttributeMaxDynamicSharedMemorySize, GV_SMEM));
        attr_set[dev] = true;
    }
    const dim3 grid((unsigned)((n + GV_ROWS - 1) / GV_ROWS), (unsigned)chunks);
    gemv_tma_kernel<TA><<<grid, GV_THREADS, GV_SMEM, ctx->stream>>>(*tm, n, x, cpc, partial, 2000000000ull);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

}  // namespace

int gemv_h_device(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, const cplx* x, double beta,
                  cplx* y) {
    const int threads = 256;
    const unsigned blocks = (unsigned)((n + 7) / 8);
    cudaEvent_t ev;
    ctx->prof.begin(ctx->stream, 2, 8.0 * (double)n * (double)n, 16.0 * (double)n * (double)n + 16.0 * 3.0 * n,
                    &ev);
    gemv_h_kernel<double2><<<blocks, threads, 0, ctx->stream>>>(n, static_cast<const double2*>(A), lda, x, beta,
                                                                 y);
    SIEB_NOTE_LAUNCH();
    ctx->prof.end(ctx->stream, ev);
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

int gemv_device(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec, const cplx* x,
                double beta, cplx* y, DeviceBuffer& scratch) {
    const int threads = 256;
    // The TMA-staged kernel needs a 16-byte aligned A whose column stride is a
    // multiple of 16 bytes; other operands (and SIEB200_GEMV_TMA=0) take the
    // per-thread-load kernel.
    const size_t esz = prec == 0 ? 16 : 8;
    const char* tma_env = getenv("SIEB200_GEMV_TMA");
    bool tma_ok = !(tma_env && tma_env[0] == '0') && n >= 2 * GV_ROWS && n <= (int64_t)1 << 30 &&
                  (reinterpret_cast<uintptr_t>(A) & 15) == 0 && ((size_t)lda * esz) % 16 == 0 &&
                  (reinterpret_cast<uintptr_t>(x) & 15) == 0;
    CUtensorMap tm;
    int64_t row_blocks, chunks, cpc;
    if (tma_ok) {
        SIEB_RETURN_IF(encode_tensor_map_2d(&tm, prec == 0 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                                            A, (uint64_t)(2 * n), (uint64_t)n, (uint64_t)lda * esz, 2 * GV_ROWS,
                                            (uint32_t)(GV_TILE_BYTES / (GV_ROWS * esz)), CU_TENSOR_MAP_SWIZZLE_NONE));
        // Two CTAs per SM. The column chunk count maximises the filled share of
        // the CTA waves times the streaming share of a CTA (a CTA pays about
        // two tiles' time to fill its ring), with chunks of whole tiles, at
        // least four tiles each; the smaller count wins within 1 %.
        const int64_t cb = GV_TILE_BYTES / (GV_ROWS * (int64_t)esz);
        const int64_t slots = 2 * (int64_t)std::max(1, ctx->sm_count);
        row_blocks = (n + GV_ROWS - 1) / GV_ROWS;
        const int64_t max_chunks = std::max<int64_t>(1, std::min<int64_t>(32, n / (4 * cb)));
        double best = -1.0;
        chunks = 1;
        for (int64_t c = 1; c <= max_chunks; ++c) {
            const int64_t t = row_blocks * c;
            const double tiles = (double)((n + c - 1) / c) / (double)cb;
            const double fill = (double)t / (double)(((t + slots - 1) / slots) * slots) * tiles / (tiles + 2.0);
            if (fill > best + 0.01) {
                best = fill;
                chunks = c;
            }
        }
        cpc = ((n + chunks - 1) / chunks + cb - 1) / cb * cb;
        chunks = (n + cpc - 1) / cpc;
    } else {
        row_blocks = (n + threads - 1) / threads;
        // Aim for ~4 CTAs per SM.
        chunks = std::max<int64_t>(1, (int64_t)ctx->sm_count * 4 / std::max<int64_t>(1, row_blocks));
        chunks = std::min<int64_t>(chunks, std::max<int64_t>(1, n / 64));
        cpc = (n + chunks - 1) / chunks;
        chunks = (n + cpc - 1) / cpc;
    }
    SIEB_RETURN_IF(scratch.reserve(sizeof(cplx) * n * chunks));
    const dim3 grid((unsigned)row_blocks, (unsigned)chunks);
    cudaEvent_t ev;
    ctx->prof.begin(ctx->stream, 2, 8.0 * (double)n * (double)n,
                    (prec == 0 ? 16.0 : 8.0) * (double)n * (double)n + 16.0 * 3.0 * n, &ev);
    if (tma_ok) {
        SIEB_RETURN_IF(prec == 0 ? gemv_tma_launch<double2>(ctx, &tm, n, x, cpc, (int)chunks, scratch.as<cplx>())
                                 : gemv_tma_launch<float2>(ctx, &tm, n, x, cpc, (int)chunks, scratch.as<cplx>()));
    } else {
        if (prec == 0)
            gemv_partial_kernel<double2><<<grid, threads, 0, ctx->stream>>>(
                n, static_cast<const double2*>(A), lda, x, cpc, scratch.as<cplx>());
        else
            gemv_partial_kernel<float2><<<grid, threads, 0, ctx->stream>>>(
                n, static_cast<const float2*>(A), lda, x, cpc, scratch.as<cplx>());
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
    }
    gemv_finish_kernel<<<(unsigned)((n + threads - 1) / threads), threads, 0, ctx->stream>>>(
        n, (int)chunks, scratch.as<cplx>(), beta, y);
    SIEB_NOTE_LAUNCH();
    ctx->prof.end(ctx->stream, ev);
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

// ------------------------------------------------- matvec without allocation
// Some callers of the residual matvec may not allocate device memory at the
// point of the call: a refinement loop that runs beside other streams of the
// same device (cudaFree waits for the whole device, stalling them), or a
// caller that has already committed the rest of HBM to the matrix and its
// factors (an allocation there can fail in mid-iteration). For them the
// partial sums live in one fixed file-scope device array instead of a
// workspace allocated per call.
//
// Limit: kStaticScratchElems complex128 partial sums (2 MiB), i.e. at most
// that many rows x column chunks; the chunk count shrinks to fit, and n
// above kStaticScratchElems is rejected. Nothing in the array needs to start
// at zero: every partial sum is written before it is read. There is one
// array per device, so calls whose kernels overlap in time (from two host
// threads, or on two contexts of one device) race on it.
constexpr int64_t kStaticScratchElems = 131072;
static __device__ __align__(256) cplx g_static_scratch[kStaticScratchElems];

namespace {
std::mutex g_static_scratch_mu;
// Per device: the array's device address and the id of the CUDA context it
// was resolved in. A device reset (cudaDeviceReset) ends that context and
// unloads the module, so a later call under a new context resolves again.
struct StaticScratchSlot {
    void* ptr = nullptr;
    unsigned long long ctx_id = 0;
};
StaticScratchSlot g_static_scratch_slot[64];

typedef CUresult (*PFN_ctxGetCurrent)(CUcontext*);
typedef CUresult (*PFN_ctxGetId)(CUcontext, unsigned long long*);

// Id of the calling thread's current CUDA context (0 if it cannot be read).
unsigned long long current_context_id() {
    static PFN_ctxGetCurrent get_current = nullptr;
    static PFN_ctxGetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PFN_ctxGetCurrent>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_ctxGetId>(fn);
        looked_up = true;
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current && get_id && get_current(&c) == CUDA_SUCCESS && c && get_id(c, &id) == CUDA_SUCCESS)
        return id;
    return 0;
}
}  // namespace

int static_scratch_setup(int device, cplx** out) {
    SIEB_CHECK(device >= 0 && device < 64, SIEB200_INVALID_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_scratch_mu);
    StaticScratchSlot& slot = g_static_scratch_slot[device];
    // The caller has made `device` current; its CUDA context exists (the
    // library context owns a stream there).
    const unsigned long long id = current_context_id();
    if (!slot.ptr || slot.ctx_id != id) {
        // This device's instance of the array; the first resolution loads the
        // module on the device.
        void* p = nullptr;
        SIEB_TRY_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
        SIEB_CHECK(p != nullptr, SIEB200_CUDA_ERROR, "cudaGetSymbolAddress returned no address");
        // With lazy loading (the default since CUDA 12.2) a kernel's code is
        // put on the device at its first launch, which can allocate device
        // memory; querying the three kernels of this path loads them now, in
        // the set-up call.
        cudaFuncAttributes fa;
        SIEB_TRY_CUDA(cudaFuncGetAttributes(&fa, gemv_partial_kernel<double2>));
        SIEB_TRY_CUDA(cudaFuncGetAttributes(&fa, gemv_partial_kernel<float2>));
        SIEB_TRY_CUDA(cudaFuncGetAttributes(&fa, gemv_finish_kernel));
        slot.ptr = p;
        slot.ctx_id = id;
    }
    *out = static_cast<cplx*>(slot.ptr);
    return SIEB200_OK;
}

int gemv_device_static_scratch(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec,
                               const cplx* x, double beta, cplx* y) {
    SIEB_CHECK(n <= kStaticScratchElems, SIEB200_INVALID_ARG,
               "matvec without allocation: n = " + std::to_string(n) + " exceeds its fixed scratch (n <= " +
                   std::to_string(kStaticScratchElems) + ")");
    cplx* scratch = nullptr;
    SIEB_RETURN_IF(static_scratch_setup(ctx->device, &scratch));
    const int threads = 256;
    const int64_t row_blocks = (n + threads - 1) / threads;
    int64_t chunks = std::max<int64_t>(1, (int64_t)ctx->sm_count * 4 / std::max<int64_t>(1, row_blocks));
    chunks = std::min<int64_t>(chunks, std::max<int64_t>(1, n / 64));
    chunks = std::min<int64_t>(chunks, kStaticScratchElems / n);  // fit the fixed array
    const int64_t cpc = (n + chunks - 1) / chunks;
    chunks = (n + cpc - 1) / cpc;
    const dim3 grid((unsigned)row_blocks, (unsigned)chunks);
    cudaEvent_t ev;
    ctx->prof.begin(ctx->stream, 2, 8.0 * (double)n * (double)n,
                    (prec == 0 ? 16.0 : 8.0) * (double)n * (double)n + 16.0 * 3.0 * n, &ev);
    if (prec == 0)
        gemv_partial_kernel<double2><<<grid, threads, 0, ctx->stream>>>(n, static_cast<const double2*>(A), lda, x,
                                                                          cpc, scratch);
    else
        gemv_partial_kernel<float2><<<grid, threads, 0, ctx->stream>>>(n, static_cast<const float2*>(A), lda, x,
                                                                         cpc, scratch);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    gemv_finish_kernel<<<(unsigned)row_blocks, threads, 0, ctx->stream>>>(n, (int)chunks, scratch, beta, y);
    SIEB_NOTE_LAUNCH();
    ctx->prof.end(ctx->stream, ev);
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

static int cusolver_handle(sieb200_ctx* ctx, cusolverDnHandle_t* h) {
    if (!ctx->cusolver) {
        cusolverDnHandle_t hh = nullptr;
        SIEB_CHECK(cusolverDnCreate(&hh) == CUSOLVER_STATUS_SUCCESS, SIEB200_CUDA_ERROR,
                   "cusolverDnCreate failed");
        SIEB_CHECK(cusolverDnSetStream(hh, ctx->stream) == CUSOLVER_STATUS_SUCCESS,
                   SIEB200_CUDA_ERROR, "cusolverDnSetStream failed");
        ctx->cusolver = hh;
    }
    *h = static_cast<cusolverDnHandle_t>(ctx->cusolver);
    return SIEB200_OK;
}

void destroy_cusolver(sieb200_ctx* ctx) {
    if (ctx->cusolver) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(ctx->cusolver));
    ctx->cusolver = nullptr;
}

int DenseSolver::factorize(double* A_, int64_t lda_) {
    A = A_;
    lda = lda_;
    factored = false;
    if (method == SIEB200_SOLVER_LU_CUSOLVER) {
        cusolverDnHandle_t h;
        SIEB_RETURN_IF(cusolver_handle(ctx, &h));
        int lwork = 0;
        SIEB_CHECK(cusolverDnZgetrf_bufferSize(h, (int)n, (int)n, reinterpret_cast<cuDoubleComplex*>(A),
                                               (int)lda, &lwork) == CUSOLVER_STATUS_SUCCESS,
                   SIEB200_CUDA_ERROR, "cusolverDnZgetrf_bufferSize failed");
        SIEB_RETURN_IF(work.reserve(sizeof(cuDoubleComplex) * (size_t)std::max(lwork, 1)));
        SIEB_RETURN_IF(ipiv.reserve(sizeof(int) * (n + 1)));
        int* d_info = ipiv.as<int>() + n;
        SIEB_CHECK(cusolverDnZgetrf(h, (int)n, (int)n, reinterpret_cast<cuDoubleComplex*>(A), (int)lda,
                                    work.as<cuDoubleComplex>(), ipiv.as<int>(), d_info) ==
                       CUSOLVER_STATUS_SUCCESS,
                   SIEB200_CUDA_ERROR, "cusolverDnZgetrf failed");
        int info = 0;
        SIEB_TRY_CUDA(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
        if (info > 0) {
            set_error("LU factorization failed: matrix is singular (U(" + std::to_string(info) + "," +
                      std::to_string(info) + ") is zero)");
            return SIEB200_SINGULAR;
        }
        SIEB_CHECK(info == 0, SIEB200_INVALID_ARG, "cusolverDnZgetrf reported an invalid argument");
        factored = true;
        return SIEB200_OK;
    }
    if (method == SIEB200_SOLVER_GMRES_C64) {
        const int st = gmres_c64_prepare(this);
        if (st == SIEB200_OK) factored = true;
        return st;
    }
    if (method == SIEB200_SOLVER_LU_FP64 || method == SIEB200_SOLVER_MIXED_IR) {
        const int st = mixed_factorize(this);
        if (st == SIEB200_OK) factored = true;
        return st;
    }
    set_error("unsupported dense solver method");
    return SIEB200_INVALID_ARG;
}

int DenseSolver::solve(int64_t nrhs, double* B, int64_t ldb, bool adjoint, double tol, int maxit,
                       int* iters) {
    SIEB_CHECK(factored, SIEB200_INVALID_ARG, "dense solver: factorize() has not succeeded");
    if (iters) *iters = 0;
    if (method == SIEB200_SOLVER_LU_CUSOLVER) {
        cusolverDnHandle_t h;
        SIEB_RETURN_IF(cusolver_handle(ctx, &h));
        int* d_info = ipiv.as<int>() + n;
        SIEB_CHECK(cusolverDnZgetrs(h, adjoint ? CUBLAS_OP_C : CUBLAS_OP_N, (int)n, (int)nrhs,
                                    reinterpret_cast<cuDoubleComplex*>(A), (int)lda, ipiv.as<int>(),
                                    reinterpret_cast<cuDoubleComplex*>(B), (int)ldb,
                                    d_info) == CUSOLVER_STATUS_SUCCESS,
                   SIEB200_CUDA_ERROR, "cusolverDnZgetrs failed");
        return SIEB200_OK;
    }
    return mixed_solve(this, nrhs, B, ldb, adjoint, tol, maxit, iters);
}


// FP64 FMA throughput probe: 8 independent dependent-FMA chains per thread,
// 4 CTAs of 256 threads per SM; the result is written only if it equals a
// value it never takes, which keeps the chains live.
__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(double* out, int iters) {
    const double m = 1.0000000001, c = 1e-12;
    double a[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = 1.0 + 1e-6 * (threadIdx.x + 32 * j);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) a[j] = fma(a[j], m, c);
    }
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) sum += a[j];
    if (sum == -1.0) out[0] = sum;
}

// The same with the FP64 tensor cores: eight independent accumulators of
// mma.sync m8n8k4 .f64 per warp (256 FMAs per instruction).
__global__ void __launch_bounds__(256) fp64_mma_probe_kernel(double* out, int iters) {
    const double a = 1e-3 * (threadIdx.x & 31), b = 1e-3 * blockIdx.x;
    double d[8][2];
#pragma unroll
    for (int j = 0; j < 8; ++j) d[j][0] = d[j][1] = 0.0;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j)
            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                         : "+d"(d[j][0]), "+d"(d[j][1])
                         : "d"(a), "d"(b));
    }
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) sum += d[j][0] + d[j][1];
    if (sum == -1.0) out[0] = sum;
}

static int fp64_probe(sieb200_ctx* ctx, bool mma, double* tflops) {
    const int iters = 8192;
    const unsigned grid = (unsigned)ctx->sm_count * 4u;
    DeviceBuffer sink;
    SIEB_RETURN_IF(sink.reserve(sizeof(double)));
    cudaEvent_t a, b;
    SIEB_TRY_CUDA(cudaEventCreate(&a));
    SIEB_TRY_CUDA(cudaEventCreate(&b));
    float best = 1e30f;
    for (int rep = 0; rep < 6; ++rep) {
        cudaEventRecord(a, ctx->stream);
        if (mma)
            fp64_mma_probe_kernel<<<grid, 256, 0, ctx->stream>>>(sink.as<double>(), iters / 8);
        else
            fp64_fma_probe_kernel<<<grid, 256, 0, ctx->stream>>>(sink.as<double>(), iters);
        SIEB_NOTE_LAUNCH();
        cudaEventRecord(b, ctx->stream);
        cudaEventSynchronize(b);
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess && rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    SIEB_TRY_CUDA(cudaGetLastError());
    // FMA: 8 chains per thread; MMA: 8 accumulators per warp, 256 FMAs each
    const double flops = mma ? 2.0 * 256.0 * 8.0 * (iters / 8) * (double)grid * 8.0
                             : 2.0 * 8.0 * iters * (double)grid * 256.0;
    *tflops = flops / (best * 1e-3) / 1e12;
    return SIEB200_OK;
}

int fp64_fma_rate(sieb200_ctx* ctx, double* tflops) { return fp64_probe(ctx, false, tflops); }
int fp64_mma_rate(sieb200_ctx* ctx, double* tflops) { return fp64_probe(ctx, true, tflops); }

}  // namespace sieb200
