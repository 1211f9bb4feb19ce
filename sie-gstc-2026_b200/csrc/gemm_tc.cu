// Trailing-update GEMM of the mixed-precision LU on the 5th-generation tensor
// cores (sm_100a):
//   C[2M x N] (fp32, column-major, ldc) -= A[2M x K] * B[N x K]^T,
// A and B K-major fp32 (TF32 hi/lo split laid out along K by the panel
// kernels, so the three products hi*hi + hi*lo + lo*hi are one K sweep).
//
// One CTA per 128 x 128 output tile, 128 threads:
//   warp 0 lane 0  TMA producer: 128B-swizzled 128 x 32 fp32 boxes of A and B
//                  into a 3-stage shared-memory ring (mbarrier expect_tx),
//   warp 1 lane 0  MMA issuer: tcgen05.mma.cta_group::1.kind::tf32, M=128,
//                  N=128, K=8 per instruction, accumulator in TMEM;
//                  tcgen05.commit frees a stage / signals the accumulator,
//   warp 2         allocates and frees 128 TMEM columns,
//   warps 0-3      epilogue: tcgen05.ld 32x32b (each warp its 32 lanes =
//                  rows), C -= acc with coalesced column stores.
// 96 KB of shared memory lets two CTAs share an SM, so one tile's epilogue
// overlaps the other's main loop. Every mbarrier wait is bounded; on timeout
// the kernel records an error word, drains what it issued and returns.

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>

#include "common.cuh"
#include "gemm_tc.cuh"
#include "sm100.cuh"

namespace sieb200 {

namespace {

constexpr int BM = 128, BN = 128, BK = 32;  // BK fp32 = 128 bytes = one swizzle atom
constexpr int STAGES = 3;
constexpr int STAGE_A = BM * BK * 4, STAGE_B = BN * BK * 4;
constexpr int SMEM_BYTES = STAGES * (STAGE_A + STAGE_B) + 1024 /*align*/ + 256 /*barriers*/;
constexpr long long kSpinLimit = 1ll << 26;

// Bounded wait: false on timeout (and sets the error word).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, unsigned* err) {
    long long it = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++it > kSpinLimit) {
            atomicCAS(err, 0u, 3u);
            return false;
        }
        if ((it & 1023) == 0 && *reinterpret_cast<volatile unsigned*>(err) != 0u) return false;
    }
    return true;
}

// K-major, 128-byte swizzle shared-memory matrix descriptor (sm_100 layout:
// start>>4 [0,14), LBO>>4 [16,30), SBO>>4 [32,46), version 1 [46,48),
// layout SWIZZLE_128B = 2 [61,64)); 8-row core groups 1024 bytes apart.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t addr) {
    return (uint64_t)((addr & 0x3FFFF) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D f32 [4,6)=1, A tf32 [7,10)=2, B tf32 [10,13)=2,
// both K-major, N>>3 at [17,23), M>>4 at [24,29).
constexpr uint32_t idesc_tf32(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}
constexpr uint32_t kIdesc = idesc_tf32(BN);
constexpr uint32_t kIdesc2 = idesc_tf32(2 * BN);  // N = 256: B_hi and B_lo in one MMA

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate,
                                          uint32_t idesc = kIdesc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(128, 2)
gemm_tf32_sub_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                     float* __restrict__ C, int64_t ldc, int M2, int N, int K, int shift0, unsigned* err) {
    // The first row tile starts shift0 columns in (see gemm_tc_sub); a tile
    // left wholly past the last column has nothing to do.
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN + (blockIdx.x == 0 ? shift0 : 0);
    if (n0 >= N) return;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned stage area (required by the 128B swizzle atoms).
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);
    const uint32_t sA = base;
    const uint32_t sB = base + STAGES * STAGE_A;
    uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + STAGES * (STAGE_A + STAGE_B));
    const uint32_t full0 = smem_u32(&bars[0]);
    const uint32_t empty0 = smem_u32(&bars[STAGES]);
    const uint32_t accb = smem_u32(&bars[2 * STAGES]);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(&bars[2 * STAGES + 1]);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int kblocks = K / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(accb, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

    bool ok = true;
    if (warp == 0 && lane == 0) {
        // Producer.
        for (int kb = 0; kb < kblocks; ++kb) {
            const int s = kb % STAGES;
            const uint32_t ph = (kb / STAGES) & 1;
            if (!mbar_wait(empty0 + 8 * s, ph ^ 1, err)) { ok = false; break; }
            mbar_expect_tx(full0 + 8 * s, STAGE_A + STAGE_B);
            tma_load_2d(sA + s * STAGE_A, &tmA, full0 + 8 * s, kb * BK, m0);
            tma_load_2d(sB + s * STAGE_B, &tmB, full0 + 8 * s, kb * BK, n0);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.
        for (int kb = 0; kb < kblocks; ++kb) {
            const int s = kb % STAGES;
            const uint32_t ph = (kb / STAGES) & 1;
            if (!mbar_wait(full0 + 8 * s, ph, err)) { ok = false; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint64_t ad = smem_desc_sw128(sA + s * STAGE_A);
            const uint64_t bd = smem_desc_sw128(sB + s * STAGE_B);
#pragma unroll
            for (int k = 0; k < BK / 8; ++k)  // 8 tf32 = 32 bytes per instruction: start address += 2
                umma_tf32(tmem, ad + 2 * k, bd + 2 * k, (kb | k) != 0 ? 1u : 0u);
            umma_commit(empty0 + 8 * s);
        }
        umma_commit(accb);  // fires when every MMA issued above has completed
    }
    __syncwarp();

    // Epilogue: all four warps. Lane 0 waits and broadcasts, so the warp stays
    // converged for the .sync.aligned TMEM loads.
    const int row = m0 + warp * 32 + lane;
    const bool row_ok = row < M2;
    // Software-pipelined: the 32 C values of the next chunk are in flight
    // while the current chunk is combined and stored; the first chunk is
    // fetched before the accumulator is ready.
    float cur[32], nxt[32];
    auto load_chunk = [&](int chunk, float (&dst)[32]) {
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const int col = n0 + chunk * 32 + j;
            dst[j] = (row_ok && col < N) ? __ldcs(C + (int64_t)col * ldc + row) : 0.f;
        }
    };
    load_chunk(0, cur);
    int got = 0;
    if (lane == 0) got = mbar_wait(accb, 0, err) ? 1 : 0;
    got = __shfl_sync(0xffffffffu, got, 0);
    __syncwarp();
    if (got) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
        for (int chunk = 0; chunk < BN / 32; ++chunk) {
            if (chunk + 1 < BN / 32) load_chunk(chunk + 1, nxt);
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + chunk * 32, v);
            if (row_ok) {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int col = n0 + chunk * 32 + j;
                    if (col < N) __stcs(C + (int64_t)col * ldc + row, cur[j] - v[j]);
                }
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) cur[j] = nxt[j];
        }
    } else {
        ok = false;
    }
    (void)ok;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 2) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
    }
}

// Persistent variant: one CTA per SM walks the output tiles t = blockIdx.x,
// blockIdx.x + gridDim.x, ... (row tiles fastest, so the CTAs in flight share
// B tiles and all of A stays in L2). 192 threads:
//   warp 0 lane 0  TMA producer of A and B boxes into a 4-stage ring,
//   warp 1         TMEM owner (256 columns: two 128-column accumulators);
//                  lane 0 issues the MMAs, alternating accumulators by tile,
//   warps 2-5      epilogue: the C tile (128 x 128 fp32, 64 KB) comes in by
//                  TMA while the tile's MMAs run; each warp reads its 32 TMEM
//                  lanes, subtracts in shared memory, releases the
//                  accumulator, and one thread stores the tile by TMA and
//                  starts loading the next one.
// So a tile's C traffic overlaps the next tile's main loop inside one CTA.
// Every mbarrier wait is bounded and reports through the error word.
constexpr int P_STAGES = 4;
constexpr int P_THREADS = 192;
constexpr int C_TILE_BYTES = BM * BN * 4;
constexpr int P_SMEM_BYTES = P_STAGES * (STAGE_A + STAGE_B) + C_TILE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
// Split-operand layout (HILO): two stages of [A_hi | A_lo] and [B_hi | B_lo]
// k-blocks, the same shared memory as four single stages.
constexpr int H_STAGES = 2;
static_assert(H_STAGES * 2 * (STAGE_A + STAGE_B) == P_STAGES * (STAGE_A + STAGE_B), "HILO stage budget");

__device__ __forceinline__ void epilogue_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// HILO = true: A = [A_hi | A_lo] and B = [B_hi | B_lo] along K (K/2 columns
// each) and the tile takes A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T. A stage
// holds one k-block of all four; B_hi and B_lo sit back to back as one
// 256-row operand, so a single N = 256 MMA forms A_hi [B_hi; B_lo]^T into
// 256 accumulator columns and an N = 128 MMA adds A_lo B_hi^T to the first
// 128. Each operand crosses from L2 once per tile (two thirds of the bytes
// of the three-product sweep); the epilogue sums the two halves.
// REDUCE = true: the epilogue does not load C. It writes the negated
// accumulator into the staging tile and adds it to C with a TMA reduction
// (cp.reduce.async.bulk.tensor .add, performed at L2), so no CTA waits for a
// 64 KB C load between tiles; the staging tile is reused once the previous
// reduction has read it. C + (-acc) rounds exactly as C - acc, and each
// element takes one reduction per launch, so results are unchanged and
// deterministic.
template <bool REDUCE, bool HILO, int CH>
__global__ void __launch_bounds__(P_THREADS, 1)
gemm_tf32_sub_persistent_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                                const __grid_constant__ CUtensorMap tmC, int M2, int N, int K, int shift0,
                                int lolo, unsigned* err) {
    constexpr int NS = HILO ? H_STAGES : P_STAGES;     // ring stages
    constexpr int SA = HILO ? 2 * STAGE_A : STAGE_A;   // A bytes per stage
    constexpr int SB = HILO ? 2 * STAGE_B : STAGE_B;   // B bytes per stage
    constexpr int ACC = HILO ? 2 * BN : BN;            // accumulator columns per buffer
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    unsigned char* gbase = smem_raw + (base - raw);
    const uint32_t sA = base;
    const uint32_t sB = base + NS * SA;
    const uint32_t sC = base + NS * (SA + SB);
    float* cs = reinterpret_cast<float*>(gbase + NS * (SA + SB));
    uint64_t* bars = reinterpret_cast<uint64_t*>(gbase + NS * (SA + SB) + C_TILE_BYTES);
    const uint32_t full0 = smem_u32(&bars[0]);
    const uint32_t empty0 = smem_u32(&bars[NS]);
    const uint32_t accf0 = smem_u32(&bars[2 * NS]);      // accumulator b ready (MMA -> epilogue)
    const uint32_t acce0 = smem_u32(&bars[2 * NS + 2]);  // accumulator b drained (epilogue -> MMA)
    const uint32_t cfull0 = smem_u32(&bars[2 * NS + 4]);  // C slot c in shared memory (CH of them)
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(&bars[2 * NS + 4 + CH]);
    static_assert(CH == 1 || CH == 2 || CH == 4, "C slots");
    static_assert((2 * NS + 4 + CH) * 8 + 4 <= 256, "barrier area");

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = (M2 + BM - 1) / BM, nt = (N + BN - 1) / BN;
    const int tiles = mt * nt;
    const int KR = HILO ? K / 2 : K;  // columns of one K sweep (the hi half)
    const int kblocks = KR / BK;
    // A_lo against B_hi only (N = 128), or against the stacked [B_hi; B_lo]
    // as well (lolo: the fourth product lo.lo lands beside hi.lo)
    const uint32_t idesc_lo = lolo ? kIdesc2 : kIdesc;
    // Tile t covers rows (t % mt) BM and columns (t / mt) BN, the first row
    // tile shift0 columns further right; a tile wholly past the last column
    // is skipped alike by all three roles (first: this CTA's first tile,
    // next: its tile after t).
    auto col0 = [&](int t) { return (t / mt) * BN + ((t % mt) == 0 ? shift0 : 0); };
    auto first = [&]() {
        int t = blockIdx.x;
        while (t < tiles && col0(t) >= N) t += gridDim.x;
        return t;
    };
    auto next = [&](int t) {
        t += gridDim.x;
        while (t < tiles && col0(t) >= N) t += gridDim.x;
        return t;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < NS; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(accf0 + 8 * b, 1);
            mbar_init(acce0 + 8 * b, 4);
        }
        for (int c = 0; c < CH; ++c) mbar_init(cfull0 + 8 * c, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(2 * ACC));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);

    if (warp == 0) {
        if (lane == 0) {
            int g = 0;
            bool ok = true;
            for (int t = first(); t < tiles && ok; t = next(t)) {
                const int m0 = (t % mt) * BM, n0 = col0(t);
                for (int kb = 0; kb < kblocks; ++kb, ++g) {
                    const int s = g % NS;
                    const uint32_t ph = (uint32_t)(g / NS) & 1u;
                    if (!mbar_wait(empty0 + 8 * s, ph ^ 1u, err)) { ok = false; break; }
                    mbar_expect_tx(full0 + 8 * s, SA + SB);
                    tma_load_2d(sA + s * SA, &tmA, full0 + 8 * s, kb * BK, m0);
                    tma_load_2d(sB + s * SB, &tmB, full0 + 8 * s, kb * BK, n0);
                    if (HILO) {
                        tma_load_2d(sA + s * SA + STAGE_A, &tmA, full0 + 8 * s, KR + kb * BK, m0);
                        tma_load_2d(sB + s * SB + STAGE_B, &tmB, full0 + 8 * s, KR + kb * BK, n0);
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int g = 0, li = 0;
            bool ok = true;
            for (int t = first(); t < tiles && ok; t = next(t), ++li) {
                const int b = li & 1;
                const uint32_t u = (uint32_t)(li >> 1);
                if (!mbar_wait(acce0 + 8 * b, (u & 1u) ^ 1u, err)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc = tmem + (uint32_t)(b * ACC);
                for (int kb = 0; kb < kblocks; ++kb, ++g) {
                    const int s = g % NS;
                    const uint32_t ph = (uint32_t)(g / NS) & 1u;
                    if (!mbar_wait(full0 + 8 * s, ph, err)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint64_t ad = smem_desc_sw128(sA + s * SA);
                    const uint64_t bd = smem_desc_sw128(sB + s * SB);
                    if (HILO) {
                        const uint64_t adl = smem_desc_sw128(sA + s * SA + STAGE_A);
#pragma unroll
                        for (int k = 0; k < BK / 8; ++k) {
                            umma_tf32(acc, ad + 2 * k, bd + 2 * k, (kb | k) != 0 ? 1u : 0u, kIdesc2);
                            umma_tf32(acc, adl + 2 * k, bd + 2 * k, 1u, idesc_lo);
                        }
                    } else {
#pragma unroll
                        for (int k = 0; k < BK / 8; ++k)
                            umma_tf32(acc, ad + 2 * k, bd + 2 * k, (kb | k) != 0 ? 1u : 0u);
                    }
                    umma_commit(empty0 + 8 * s);
                }
                if (ok) umma_commit(accf0 + 8 * b);  // fires when the tile's MMAs have completed
            }
        }
    } else {
        // C moves through CH slots of BN / CH columns: a slot's store (or
        // reduction) is followed at once by the load of the same columns of
        // the CTA's next tile, so with CH > 1 the next tile's first columns
        // are already in flight while this tile's last ones are processed.
        constexpr int CC = BN / CH;
        constexpr int CHUNK_BYTES = BM * CC * 4;
        const int q = warp & 3;            // TMEM lane quarter of this warp
        const int et = threadIdx.x - 64;   // 0..127
        const int rt = q * 32 + lane;      // row of the tile
        const bool e0 = et == 0;
        int t = first();
        if (!REDUCE && e0 && t < tiles) {
            for (int c = 0; c < CH; ++c) {
                mbar_expect_tx(cfull0 + 8 * c, CHUNK_BYTES);
                tma_load_2d(sC + c * CHUNK_BYTES, &tmC, cfull0 + 8 * c, (t % mt) * BM, col0(t) + c * CC);
            }
        }
        for (int li = 0; t < tiles; t = next(t), ++li) {
            const int b = li & 1;
            const uint32_t u = (uint32_t)(li >> 1);
            const int tn = next(t);
            int got = 0;
            if (lane == 0) got = mbar_wait(accf0 + 8 * b, u & 1u, err) ? 1 : 0;
            got = __shfl_sync(0xffffffffu, got, 0);
            __syncwarp();
            if (got) asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
            for (int c = 0; c < CH; ++c) {
                const bool okc = REDUCE ? true : mbar_wait(cfull0 + 8 * c, (uint32_t)li & 1u, err);
                float* cc = cs + c * (BM * CC);
                if (got && okc) {
#pragma unroll 1
                    for (int sub = 0; sub < CC / 32; ++sub) {
                        float v[32];
                        const uint32_t ta =
                            tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * ACC + c * CC + sub * 32);
                        tmem_ld32(ta, v);
                        if (HILO) {
                            float w[32];
                            tmem_ld32(ta + BN, w);
#pragma unroll
                            for (int j = 0; j < 32; ++j) v[j] += w[j];
                        }
                        if (REDUCE) {
#pragma unroll
                            for (int j = 0; j < 32; ++j) cc[(sub * 32 + j) * BM + rt] = -v[j];
                        } else {
#pragma unroll
                            for (int j = 0; j < 32; ++j) cc[(sub * 32 + j) * BM + rt] -= v[j];
                        }
                    }
                }
                if (c == CH - 1) {  // every TMEM column of accumulator b has been read
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) mbar_arrive(acce0 + 8 * b);
                }
                // Generic-proxy writes of the slot, then the async-proxy store.
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                epilogue_bar();
                if (e0) {
                    const int x = (t % mt) * BM, y = col0(t) + c * CC;
                    if (REDUCE) {
                        // A tile whose accumulator wait failed adds nothing.
                        if (got) tma_reduce_add_2d(&tmC, sC + c * CHUNK_BYTES, x, y);
                    } else {
                        tma_store_2d(&tmC, sC + c * CHUNK_BYTES, x, y);
                    }
                    bulk_commit();
                    if (REDUCE)
                        // the slot written next was last reduced CH - 1 groups
                        // ago: only that read has to be complete
                        bulk_wait_read<CH - 1>();
                    else
                        bulk_wait_read_all();  // the slot is reloaded at once
                    if (!REDUCE && tn < tiles) {
                        mbar_expect_tx(cfull0 + 8 * c, CHUNK_BYTES);
                        tma_load_2d(sC + c * CHUNK_BYTES, &tmC, cfull0 + 8 * c, (tn % mt) * BM,
                                    col0(tn) + c * CC);
                    }
                }
                // REDUCE: the next slot is written only after its previous
                // reduction has read it (the wait above). Otherwise the next
                // tile's writes wait for the slot's new load (cfull), issued
                // after the read.
                if (REDUCE) epilogue_bar();
            }
        }
        if (e0) bulk_wait_all();
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * ACC));
    }
}

// SIMT reference on the same packed operands (checking path).
// hilo: A = [A_hi | A_lo], B = [B_hi | B_lo] along K; the sum is
// a_hi (b_hi + b_lo) + a_lo b_hi per k of the first half.
__global__ void gemm_simt_sub_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                     float* __restrict__ C, int64_t ldc, int M2, int N, int K, int hilo,
                                     int shift0) {
    __shared__ float As[64][33], Bs[64][33], Al[64][33], Bl[64][33];
    // rows [0, BM) start shift0 columns in, like the tensor-core kernels
    const int r0 = blockIdx.x * 64, c0 = blockIdx.y * 64 + (r0 < BM ? shift0 : 0);
    if (c0 >= N) return;
    const int tr = threadIdx.x & 63, tc = threadIdx.x >> 6;  // 256 threads: 64 rows x 4 col groups
    const int KR = hilo ? K / 2 : K;
    float acc[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) acc[j] = 0.f;
    for (int k0 = 0; k0 < KR; k0 += 32) {
        for (int e = threadIdx.x; e < 64 * 32; e += blockDim.x) {
            const int r = e / 32, k = e % 32;
            As[r][k] = (r0 + r < M2) ? A[(int64_t)(r0 + r) * K + k0 + k] : 0.f;
            Bs[r][k] = (c0 + r < N) ? B[(int64_t)(c0 + r) * K + k0 + k] : 0.f;
            if (hilo) {
                Al[r][k] = (r0 + r < M2) ? A[(int64_t)(r0 + r) * K + KR + k0 + k] : 0.f;
                Bl[r][k] = (c0 + r < N) ? B[(int64_t)(c0 + r) * K + KR + k0 + k] : 0.f;
            }
        }
        __syncthreads();
        for (int k = 0; k < 32; ++k) {
            const float a = As[tr][k];
            if (hilo) {
                const float al = Al[tr][k];
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[j] += a * Bs[tc * 16 + j][k] + a * Bl[tc * 16 + j][k] + al * Bs[tc * 16 + j][k];
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[j] += a * Bs[tc * 16 + j][k];
            }
        }
        __syncthreads();
    }
    if (r0 + tr < M2)
        for (int j = 0; j < 16; ++j) {
            const int col = c0 + tc * 16 + j;
            if (col < N) C[(int64_t)col * ldc + r0 + tr] -= acc[j];
        }
}

int make_map(CUtensorMap* map, const float* ptr, int64_t inner, int64_t outer, int box_outer) {
    return encode_tensor_map_2d(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, ptr, (uint64_t)inner, (uint64_t)outer,
                                (uint64_t)inner * sizeof(float), BK, (uint32_t)box_outer, CU_TENSOR_MAP_SWIZZLE_128B);
}

}  // namespace

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int encode_tensor_map_2d(CUtensorMap* map, CUtensorMapDataType type, const void* base, uint64_t inner,
                         uint64_t outer, uint64_t row_stride_bytes, uint32_t box_inner, uint32_t box_outer,
                         CUtensorMapSwizzle swizzle) {
    if (!g_encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SIEB_TRY_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        SIEB_CHECK(fn && q == cudaDriverEntryPointSuccess, SIEB200_CUDA_ERROR,
                   "cuTensorMapEncodeTiled is not available from the driver");
        g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    const cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)outer};
    const cuuint64_t strides[1] = {(cuuint64_t)row_stride_bytes};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = g_encode(map, type, 2, const_cast<void*>(base), dims, strides, box, estr,
                                CU_TENSOR_MAP_INTERLEAVE_NONE, swizzle, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    SIEB_CHECK(r == CUDA_SUCCESS, SIEB200_CUDA_ERROR, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return SIEB200_OK;
}

struct GemmTC {
    unsigned* err = nullptr;
    int mode = 3;  // persistent kernel, reduction epilogue
    int c_slots = 4;  // C slots of the persistent kernel's epilogue (1 or 4)
    int lolo = 0;     // split operands: also the product A_lo B_lo^T
    bool attr_set = false;
    bool attr_set_p[8] = {};
    int sms = 148;
};

template <bool REDUCE, bool HILO, int CH>
int launch_one(unsigned grid, cudaStream_t stream, const CUtensorMap& ma, const CUtensorMap& mb,
               const CUtensorMap& mc, int M2, int N, int K, int shift0, int lolo, unsigned* err,
               bool& attr_set) {
    if (!attr_set) {
        SIEB_TRY_CUDA(cudaFuncSetAttribute(gemm_tf32_sub_persistent_kernel<REDUCE, HILO, CH>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, P_SMEM_BYTES));
        attr_set = true;
    }
    gemm_tf32_sub_persistent_kernel<REDUCE, HILO, CH><<<grid, P_THREADS, P_SMEM_BYTES, stream>>>(ma, mb, mc, M2, N,
                                                                                                K, shift0, lolo, err);
    return SIEB200_OK;
}

// variant bit 0: reduction epilogue, bit 1: split operands, bit 2: four C slots.
int launch_persistent(int variant, unsigned grid, cudaStream_t stream, const CUtensorMap& ma, const CUtensorMap& mb,
                      const CUtensorMap& mc, int M2, int N, int K, int shift0, int lolo, unsigned* err,
                      bool (&attr_set)[8]) {
    bool& a = attr_set[variant];
    switch (variant) {
        case 0: return launch_one<false, false, 1>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
        case 1: return launch_one<true, false, 1>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
        case 2: return launch_one<false, true, 1>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
        case 3: return launch_one<true, true, 1>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
        case 4: return launch_one<false, false, 4>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
        case 5: return launch_one<true, false, 4>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
        case 6: return launch_one<false, true, 4>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
        default: return launch_one<true, true, 4>(grid, stream, ma, mb, mc, M2, N, K, shift0, lolo, err, a);
    }
}

int gemm_tc_create(GemmTC** out) {
    GemmTC* g = new GemmTC();
    cudaError_t e = cudaMalloc(&g->err, sizeof(unsigned));
    if (e != cudaSuccess) {
        delete g;
        set_error(std::string("gemm workspace: ") + cudaGetErrorString(e));
        return SIEB200_CUDA_ERROR;
    }
    cudaMemset(g->err, 0, sizeof(unsigned));
    const char* env = getenv("SIEB200_GEMM_SIMT");
    if (env && env[0] == '1') g->mode = 0;
    const char* mode_env = getenv("SIEB200_GEMM_MODE");
    if (mode_env && mode_env[0] >= '0' && mode_env[0] <= '3' && mode_env[1] == 0) g->mode = mode_env[0] - '0';
    const char* slots_env = getenv("SIEB200_GEMM_C_SLOTS");
    if (slots_env && slots_env[0] == '1' && slots_env[1] == 0) g->c_slots = 1;
    const char* lolo_env = getenv("SIEB200_GEMM_LOLO");
    g->lolo = (lolo_env && lolo_env[0] == '1') ? 1 : 0;
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaGetLastError();
    *out = g;
    return SIEB200_OK;
}

void gemm_tc_destroy(GemmTC* g) {
    if (!g) return;
    if (g->err) cudaFree(g->err);
    delete g;
}

void gemm_tc_set_mode(GemmTC* g, int mode) { g->mode = mode; }

int gemm_tc_sub(GemmTC* g, cudaStream_t stream, float* C, int64_t ldc, const float* A, const float* B,
                int64_t M2, int64_t N, int K, int max_ctas, int layout, int64_t shift0) {
    SIEB_CHECK(K % BK == 0 && K > 0, SIEB200_INVALID_ARG, "GEMM K must be a positive multiple of 32");
    SIEB_CHECK(layout == 0 || (layout == 1 && K % (2 * BK) == 0), SIEB200_INVALID_ARG,
               "split-operand GEMM: K must be a positive multiple of 64");
    SIEB_CHECK(M2 > 0 && N > 0 && M2 < (1ll << 31) && N < (1ll << 31), SIEB200_INVALID_ARG, "GEMM size out of range");
    SIEB_CHECK(shift0 >= 0 && shift0 < N, SIEB200_INVALID_ARG, "GEMM first-row-tile column shift out of range");
    SIEB_CHECK(((uintptr_t)A % 16) == 0 && ((uintptr_t)B % 16) == 0, SIEB200_INVALID_ARG,
               "GEMM operands must be 16-byte aligned");
    if (g->mode == 0) {
        gemm_simt_sub_kernel<<<dim3((unsigned)((M2 + 63) / 64), (unsigned)((N + 63) / 64)), 256, 0, stream>>>(
            A, B, C, ldc, (int)M2, (int)N, K, layout, (int)shift0);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        return SIEB200_OK;
    }
    CUtensorMap ma, mb;
    SIEB_RETURN_IF(make_map(&ma, A, K, M2, BM));
    SIEB_RETURN_IF(make_map(&mb, B, K, N, BN));
    // The persistent kernel moves C by TMA: its base and column stride must
    // be 16-byte aligned (otherwise the per-tile kernel below is used).
    // The split-operand layout runs on the persistent kernel only.
    SIEB_CHECK(layout == 0 || (((uintptr_t)C % 16) == 0 && ((ldc * 4) % 16) == 0), SIEB200_INVALID_ARG,
               "split-operand GEMM: C and its column stride must be 16-byte aligned");
    if ((g->mode >= 2 || layout == 1) && ((uintptr_t)C % 16) == 0 && ((ldc * 4) % 16) == 0) {
        const int ch = g->c_slots;
        CUtensorMap mc;
        SIEB_RETURN_IF(encode_tensor_map_2d(&mc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, C, (uint64_t)M2, (uint64_t)N,
                                            (uint64_t)ldc * sizeof(float), BM, BN / ch, CU_TENSOR_MAP_SWIZZLE_NONE));
        const int64_t tiles = ((M2 + BM - 1) / BM) * ((N + BN - 1) / BN);
        const int cap = max_ctas > 0 ? std::min(max_ctas, g->sms) : g->sms;
        const unsigned grid = (unsigned)std::min<int64_t>(tiles, std::max(1, cap));
        const bool red = g->mode == 3;
        const int variant = (red ? 1 : 0) + (layout == 1 ? 2 : 0) + (ch == 4 ? 4 : 0);
        SIEB_RETURN_IF(launch_persistent(variant, grid, stream, ma, mb, mc, (int)M2, (int)N, K, (int)shift0,
                                         layout == 1 ? g->lolo : 0, g->err, g->attr_set_p));
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        return SIEB200_OK;
    }
    if (!g->attr_set) {
        SIEB_TRY_CUDA(cudaFuncSetAttribute(gemm_tf32_sub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           SMEM_BYTES));
        g->attr_set = true;
    }
    const dim3 grid((unsigned)((M2 + BM - 1) / BM), (unsigned)((N + BN - 1) / BN));
    gemm_tf32_sub_kernel<<<grid, 128, SMEM_BYTES, stream>>>(ma, mb, C, ldc, (int)M2, (int)N, K, (int)shift0, g->err);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

int gemm_tc_check(GemmTC* g, cudaStream_t stream) {
    unsigned e = 0;
    SIEB_TRY_CUDA(cudaMemcpyAsync(&e, g->err, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(stream));
    if (e != 0u) {
        set_error("tensor-core GEMM: a pipeline wait exceeded its bound");
        return SIEB200_TIMEOUT;
    }
    return SIEB200_OK;
}

}  // namespace sieb200
