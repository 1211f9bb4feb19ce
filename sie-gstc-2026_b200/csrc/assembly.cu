// Dense RWG-Galerkin impedance-matrix assembly (PEC T-EFIE / N-EFIE / N-MFIE,
// T-PMCHWT / N-PMCHWT / N-Muller, SIE-GSTC).
//
// Reference behaviour (paths relative to the SIE-GSTC project):
//   per face pair TL/TK      include/sie_mom/cuda/dunavant_quadrature.cuh:207-324
//   per face pair nTL/nTK    dunavant_quadrature.cuh:342-480 (surface form B),
//                            singular part 889-1040
//   RWG Gram (jump terms)    dunavant_quadrature.cuh:1261-1326
//   rotated-testing blocks   src/sie_mom/solvers/dielectric/dielectric_kernels.cu:155-500,
//                            src/sie_mom/solvers/pec_solver.cu:113-240
//   singular extraction      dunavant_quadrature.cuh:769-875,
//                            include/sie_mom/cuda/semi_analytic_integrals.cuh:35-92, 563-667
//   Green kernels            include/sie_mom/cuda/green_functions_utils.cuh:236-361
//   block placement          include/sie_mom/cuda/sie_kernels_assembly.cuh:156-272, 610-705,
//                            src/sie_mom/solvers/dielectric/dielectric_kernels.cu:23-149
//   GSTC jump-condition mass sie_kernels_assembly.cuh:460-594,
//                            include/sie_mom/cuda/gstc_tensor_utils.cuh:72-309,
//                            dunavant_quadrature.cuh:1422-1508
//
// B200 design. The reference runs one thread per face pair with 72 global
// complex atomics per pair. Here:
//   1. face_prep      one thread per face builds a geometry record and the
//                     face's quadrature points (double) once.
//   2. pair_regular   one CTA per test face; its 8 warps stream the source
//                     faces, one warp per face pair, lanes over the Q*Q point
//                     pairs. Instead of 9 RWG products per point pair, every
//                     lane accumulates 8 (TL) + 10 (TK) complex moments of the
//                     kernel in triangle-local coordinates; a warp butterfly
//                     reduces them and 9 lanes expand them into the 3x3 blocks:
//                       rho_m . rho_n  = (p-A_j).(q-B_i)
//                       (rho_m x rho_n) . R = (rho_m x rho_n) . (v_j - v_i),
//                     so the inner loop is bound by the Green-kernel
//                     evaluation (sqrt, division, sincos) on the FP64 pipe.
//   3. pair_singular  one warp per near pair (centroid distance below the
//                     threshold, decided in float as the reference does) adds
//                     the analytic (Wilton) part, lanes over outer points.
//   4. mass_face      GSTC only: one thread per (face, tensor).
//   5. gather         one thread per (test edge, source edge) sums the <= 2x2
//                     incident face pairs and writes every block of Z exactly
//                     once per slab: deterministic, no atomics.
// Face-pair blocks live in a workspace processed in slabs of test faces, so
// the largest meshes stream through a bounded buffer.

#include <cuda_runtime.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace sieb200 {

namespace {

constexpr int kMaxQ = 80;      // Dunavant rule 20 has 79 points
constexpr int kWarps = 8;      // warps per CTA in pair_regular
constexpr int kMaxLine = 20;   // Gauss-Legendre points of the nTL line form
constexpr double kPi = 3.14159265358979323846;

struct FaceGeom {
    d3 v[3];
    d3 c;        // centroid ((v0 + v1) + v2) / 3, as the reference forms it
    d3 fv[3];    // free vertex of local edge j
    d3 A[3];     // fv[j] - c
    double len[3];
    double area;
    int idx[3];
    int edge[3];
};

__device__ __forceinline__ d3 ldg3(const d3* p) {
    return mk3(__ldg(&p->x), __ldg(&p->y), __ldg(&p->z));
}

// Reference-exact (no FMA contraction) centroid and distance, so that the
// float threshold test takes the same branch as the reference kernels
// (sie_kernels_assembly.cuh:195-199).
__device__ __forceinline__ float centroid_distance(const FaceGeom& a, const FaceGeom& b) {
    const double dx = __dsub_rn(a.c.x, b.c.x), dy = __dsub_rn(a.c.y, b.c.y),
                 dz = __dsub_rn(a.c.z, b.c.z);
    const double s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return (float)__dsqrt_rn(s);
}

// Extraction test: the dielectric kernels compare the float-rounded centroid
// distance (dielectric_kernels.cu:201-206), the PEC N-EFIE / N-MFIE kernels
// the double distance against the float threshold (pec_solver.cu:134-136).
__device__ __forceinline__ bool near_pair(const FaceGeom& a, const FaceGeom& b, float thr, int exact) {
    if (!exact) return centroid_distance(a, b) < thr;
    const double dx = __dsub_rn(a.c.x, b.c.x), dy = __dsub_rn(a.c.y, b.c.y),
                 dz = __dsub_rn(a.c.z, b.c.z);
    const double s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
    return __dsqrt_rn(s) < (double)thr;
}

__global__ void face_prep_kernel(const double* __restrict__ V, const int* __restrict__ F,
                                 const int* __restrict__ FE, int nf, const float* __restrict__ qpts,
                                 int Q, FaceGeom* __restrict__ geom, d3* __restrict__ qp) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    FaceGeom g;
    for (int a = 0; a < 3; ++a) {
        g.idx[a] = F[3 * f + a];
        g.edge[a] = FE[3 * f + a];
        g.v[a] = mk3(V[3 * g.idx[a]], V[3 * g.idx[a] + 1], V[3 * g.idx[a] + 2]);
    }
    g.c = mk3(__ddiv_rn(__dadd_rn(__dadd_rn(g.v[0].x, g.v[1].x), g.v[2].x), 3.0),
              __ddiv_rn(__dadd_rn(__dadd_rn(g.v[0].y, g.v[1].y), g.v[2].y), 3.0),
              __ddiv_rn(__dadd_rn(__dadd_rn(g.v[0].z, g.v[1].z), g.v[2].z), 3.0));
    // mesh_geometry.cuh:51-80: local edge e runs A->B, free vertex opposite,
    // sign +1 iff global index of A > global index of B.
    const int EA[3] = {0, 1, 2}, EB[3] = {1, 2, 0}, EF[3] = {2, 0, 1};
    for (int e = 0; e < 3; ++e) {
        const d3 ev = g.v[EB[e]] - g.v[EA[e]];
        const double l = sqrt(ev.x * ev.x + ev.y * ev.y + ev.z * ev.z);
        g.len[e] = (g.idx[EA[e]] > g.idx[EB[e]] ? 1.0 : -1.0) * l;
        g.fv[e] = g.v[EF[e]];
        g.A[e] = g.fv[e] - g.c;
    }
    const d3 cr = cross3(g.v[1] - g.v[0], g.v[2] - g.v[0]);
    g.area = 0.5 * sqrt(dot3(cr, cr));
    geom[f] = g;
    // mesh_geometry.cuh:211-222 with float reference coordinates.
    for (int q = 0; q < Q; ++q) {
        const double xi = (double)qpts[2 * q], eta = (double)qpts[2 * q + 1];
        const double zeta = 1.0 - xi - eta;
        qp[(size_t)f * Q + q] = mk3(g.v[0].x * zeta + g.v[1].x * xi + g.v[2].x * eta,
                                    g.v[0].y * zeta + g.v[1].y * xi + g.v[2].y * eta,
                                    g.v[0].z * zeta + g.v[1].z * xi + g.v[2].z * eta);
    }
}

// Near pairs: count (list == nullptr) or fill.
__global__ void near_pairs_kernel(const FaceGeom* __restrict__ geom, int nf, float thr, int exact,
                                  int m0, int m1, unsigned long long* counter, int2* list,
                                  unsigned long long capacity) {
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long span = (long long)(m1 - m0) * nf;
    if (id >= span) return;
    const int m = m0 + (int)(id / nf), n = (int)(id % nf);
    if (near_pair(geom[m], geom[n], thr, exact)) {
        const unsigned long long slot = atomicAdd(counter, 1ull);
        if (list && slot < capacity) list[slot] = make_int2(m, n);
    }
}

template <int NK, bool TK>
struct Moments {
    cplx S0[NK], Sp[NK][3], Sq[NK][3], Spq[NK];
    cplx T0[TK ? NK : 1], Tp[TK ? NK : 1][3], Tq[TK ? NK : 1][3], Tpq[TK ? NK : 1][3];
};

__device__ __forceinline__ void warp_sum(double& v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
}
__device__ __forceinline__ void warp_sum(cplx& v) {
    warp_sum(v.re);
    warp_sum(v.im);
}

// One point pair: kernel values for wavenumber k (standard or extracted form)
// green_functions_utils.cuh:236-288 / 295-361. Returns G (TL kernel) and g
// with TK kernel = g * (r_p - r_q).
__device__ __forceinline__ void green_std(double R, double inv_R, double i4pR, double k, cplx& G,
                                          cplx& g) {
    double s, c;
    sincos(k * R, &s, &c);
    G = cx(c * i4pR, -s * i4pR);
    const cplx wg = cx(inv_R * G.re - k * G.im, inv_R * G.im + k * G.re);
    g = wg * inv_R;
}

__device__ __forceinline__ void green_reg(double R, double k, cplx& G, cplx& g) {
    if (R < 1e-9) {
        G = cx(0.0, -k / (4.0 * kPi));
        g = cx(0.0, 0.0);
        return;
    }
    const double i4p = 1.0 / (4.0 * kPi);
    const double inv_R = 1.0 / R, inv_R2 = inv_R * inv_R, inv_R3 = inv_R2 * inv_R;
    const double i4pR = i4p * inv_R;
    double s, c;
    sincos(k * R, &s, &c);
    G = cx((c - 1.0) * i4pR, -s * i4pR);
    cplx K = cx(inv_R3, k * inv_R2) * cx(c, -s);
    K.re += -(inv_R3 + k * k * 0.5 * inv_R);
    g = K * i4p;
}

template <int NK, bool TK>
__device__ __forceinline__ void accumulate(Moments<NK, TK>& M, const d3& pl, const d3& ql,
                                           double pq, const d3& pxq, double ww, int a,
                                           cplx G, cplx g) {
    const cplx Gw = G * ww;
    M.S0[a] += Gw;
    M.Sp[a][0] += Gw * pl.x; M.Sp[a][1] += Gw * pl.y; M.Sp[a][2] += Gw * pl.z;
    M.Sq[a][0] += Gw * ql.x; M.Sq[a][1] += Gw * ql.y; M.Sq[a][2] += Gw * ql.z;
    M.Spq[a] += Gw * pq;
    if (TK) {
        const cplx gw = g * ww;
        M.T0[a] += gw;
        M.Tp[a][0] += gw * pl.x; M.Tp[a][1] += gw * pl.y; M.Tp[a][2] += gw * pl.z;
        M.Tq[a][0] += gw * ql.x; M.Tq[a][1] += gw * ql.y; M.Tq[a][2] += gw * ql.z;
        M.Tpq[a][0] += gw * pxq.x; M.Tpq[a][1] += gw * pxq.y; M.Tpq[a][2] += gw * pxq.z;
    }
}

// Regular (or extracted-kernel) double quadrature of all face pairs (m, n)
// with m in [m0, m1). Output blocks: NB = NK (TL only) or 2*NK (TL then TK),
// each 3x3 complex, per pair at pairs[((m-m0)*nf + n) * NB*9].
// SPLIT: blockIdx.y picks one of the NK wavenumbers and the CTA accumulates
// that one only. The geometry of a point pair (R, 1/R, p.q, p x q) is then
// formed once per wavenumber instead of once, but the moments of one
// wavenumber (18 complex) fit in half the registers, so two CTAs share an SM
// and the FP64 pipe sees twice the warps; each wavenumber's sums run in the
// same order as without the split.
template <int NK, bool TK, bool SPLIT = false>
__global__ void __launch_bounds__(kWarps * 32, SPLIT ? 2 : 1)
pair_regular_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                    const float* __restrict__ qw_g, int Q, int nf, int m0, double k0, double k1,
                    float thr, cplx* __restrict__ pairs) {
    constexpr int NB = TK ? 2 * NK : NK;
    constexpr int NKC = SPLIT ? 1 : NK;  // wavenumbers accumulated by this CTA
    const int a_base = SPLIT ? (int)blockIdx.y : 0;
    __shared__ d3 s_tp[kMaxQ], s_tl[kMaxQ];
    __shared__ double s_w[kMaxQ];
    __shared__ d3 s_sp[kWarps][kMaxQ], s_sl[kWarps][kMaxQ];

    const int m = m0 + blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const FaceGeom& gm = geom[m];
    const d3 cm = gm.c;
    for (int t = threadIdx.x; t < Q; t += blockDim.x) {
        const d3 r = qp[(size_t)m * Q + t];
        s_tp[t] = r;
        s_tl[t] = r - cm;
        s_w[t] = (double)qw_g[t];
    }
    __syncthreads();
    const double kall[2] = {k0, k1};
    double kk[NKC];
#pragma unroll
    for (int a = 0; a < NKC; ++a) kk[a] = kall[a_base + a];
    const int QQ = Q * Q;

    for (int n = warp; n < nf; n += kWarps) {
        const FaceGeom& gn = geom[n];
        const d3 cn = gn.c;
        for (int t = lane; t < Q; t += 32) {
            const d3 r = ldg3(&qp[(size_t)n * Q + t]);
            s_sp[warp][t] = r;
            s_sl[warp][t] = r - cn;
        }
        __syncwarp();
        const bool regular = centroid_distance(gm, gn) < thr;  // warp-uniform
        const bool coinc = gm.idx[0] == gn.idx[0] && gm.idx[1] == gn.idx[1] &&
                           gm.idx[2] == gn.idx[2];

        Moments<NKC, TK> M;
#pragma unroll
        for (int a = 0; a < NKC; ++a) {
            M.S0[a] = cx(0, 0); M.Spq[a] = cx(0, 0);
#pragma unroll
            for (int c = 0; c < 3; ++c) { M.Sp[a][c] = cx(0, 0); M.Sq[a][c] = cx(0, 0); }
            if (TK) {
                M.T0[a] = cx(0, 0);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    M.Tp[a][c] = cx(0, 0); M.Tq[a][c] = cx(0, 0); M.Tpq[a][c] = cx(0, 0);
                }
            }
        }

        for (int idx = lane; idx < QQ; idx += 32) {
            const int p = idx / Q, q = idx - p * Q;
            const d3 rp = s_tp[p], rq = s_sp[warp][q];
            const d3 pl = s_tl[p], ql = s_sl[warp][q];
            const double ww = s_w[p] * s_w[q];
            const d3 Rv = rp - rq;
            const double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
            const double pq = dot3(pl, ql);
            const d3 pxq = TK ? cross3(pl, ql) : mk3(0, 0, 0);
            if (!regular) {
                if (R < 1e-12) continue;
                const double inv_R = 1.0 / R;
                const double i4pR = 1.0 / (4.0 * kPi * R);
#pragma unroll
                for (int a = 0; a < NKC; ++a) {
                    cplx G, g;
                    green_std(R, inv_R, i4pR, kk[a], G, g);
                    accumulate<NKC, TK>(M, pl, ql, pq, pxq, ww, a, G, g);
                }
            } else {
#pragma unroll
                for (int a = 0; a < NKC; ++a) {
                    cplx G, g;
                    green_reg(R, kk[a], G, g);
                    accumulate<NKC, TK>(M, pl, ql, pq, pxq, ww, a, G, g);
                }
            }
        }
        // Butterfly: every lane ends with the totals.
#pragma unroll
        for (int a = 0; a < NKC; ++a) {
            warp_sum(M.S0[a]); warp_sum(M.Spq[a]);
#pragma unroll
            for (int c = 0; c < 3; ++c) { warp_sum(M.Sp[a][c]); warp_sum(M.Sq[a][c]); }
            if (TK) {
                warp_sum(M.T0[a]);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    warp_sum(M.Tp[a][c]); warp_sum(M.Tq[a][c]); warp_sum(M.Tpq[a][c]);
                }
            }
        }
        if (lane < 9) {
            const int j = lane / 3, i = lane - 3 * j;
            const d3 A = gm.A[j], B = gn.A[i];
            const d3 d = gm.fv[j] - gn.fv[i];
            const double scale = gm.len[j] * gn.len[i];
            const double AB = dot3(A, B);
            cplx* out = pairs + ((size_t)blockIdx.x * nf + n) * (NB * 9);
#pragma unroll
            for (int a = 0; a < NKC; ++a) {
                // TL_ji = l_j l_i [ 1/4 (Spq - Sp.B - A.Sq + (A.B) S0) - S0 / k^2 ]
                cplx t = M.Spq[a];
                t = t - (M.Sp[a][0] * B.x + M.Sp[a][1] * B.y + M.Sp[a][2] * B.z);
                t = t - (M.Sq[a][0] * A.x + M.Sq[a][1] * A.y + M.Sq[a][2] * A.z);
                t += M.S0[a] * AB;
                const cplx tl = (t * 0.25 - M.S0[a] * (1.0 / (kk[a] * kk[a]))) * scale;
                out[(a_base + a) * 9 + lane] = tl;
                if (TK) {
                    cplx tk = cx(0, 0);
                    if (!coinc) {
                        // TK_ji = l_j l_i / 4 [ Tpq.d - (Tp x B).d - (A x Tq).d + ((A x B).d) T0 ]
                        const d3 BxD = cross3(B, d);   // (Tp x B).d = Tp . (B x d)
                        const d3 DxA = cross3(d, A);   // (A x Tq).d = Tq . (d x A)
                        const double axbd = dot3(cross3(A, B), d);
                        cplx u = M.Tpq[a][0] * d.x + M.Tpq[a][1] * d.y + M.Tpq[a][2] * d.z;
                        u = u - (M.Tp[a][0] * BxD.x + M.Tp[a][1] * BxD.y + M.Tp[a][2] * BxD.z);
                        u = u - (M.Tq[a][0] * DxA.x + M.Tq[a][1] * DxA.y + M.Tq[a][2] * DxA.z);
                        u += M.T0[a] * axbd;
                        tk = u * (0.25 * scale);
                    }
                    out[(NK + a_base + a) * 9 + lane] = tk;
                }
            }
        }
        __syncwarp();
    }
}

// The same double quadrature with a test point held per lane. Lane l works
// on test point p (G lanes per point when Q < 32, each taking every G-th
// source point) and sums over its source points only the moments that do not
// carry p: per wavenumber S0_p = sum w_q G, Sq_p = sum w_q G q, and for TK
// T0_p = sum w_q g, Tq_p = sum w_q g q (8 complex for both). The moments
// with p are folded in once per point,
//   S0 += w_p S0_p,  Sp += w_p S0_p p,  Sq += w_p Sq_p,  Spq += w_p p.Sq_p,
//   T0 += w_p T0_p,  Tp += w_p T0_p p,  Tq += w_p Tq_p,  Tpq += w_p p x Tq_p,
// reduced over the warp and accumulated in shared memory. Per point pair and
// wavenumber that is 20 FP64 accumulation instructions instead of 40 and no
// p.q or p x q, and the accumulators fit in half the registers (two CTAs per
// SM). Each moment is the same sum as in pair_regular_kernel in another
// order.
template <int NK, bool TK>
__global__ void __launch_bounds__(kWarps * 32, 2)
pair_regular_pq_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                       const float* __restrict__ qw_g, int Q, int nf, int m0, double k0, double k1,
                       float thr, cplx* __restrict__ pairs) {
    constexpr int NB = TK ? 2 * NK : NK;
    constexpr int NM = TK ? 18 : 8;  // complex moments per wavenumber
    __shared__ d3 s_tp[kMaxQ], s_tl[kMaxQ];
    __shared__ double s_w[kMaxQ];
    __shared__ d3 s_sp[kWarps][kMaxQ], s_sl[kWarps][kMaxQ];
    __shared__ cplx s_tot[kWarps][NK * NM];

    const int m = m0 + blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const FaceGeom& gm = geom[m];
    const d3 cm = gm.c;
    for (int t = threadIdx.x; t < Q; t += blockDim.x) {
        const d3 r = qp[(size_t)m * Q + t];
        s_tp[t] = r;
        s_tl[t] = r - cm;
        s_w[t] = (double)qw_g[t];
    }
    __syncthreads();
    const double kk[2] = {k0, k1};
    const int G = Q >= 32 ? 1 : 32 / Q;  // lanes per test point
    const int PL = 32 / G;               // test points per round
    const int lp = lane / G, lq = lane - (lane / G) * G;
    cplx* tot = s_tot[warp];

    for (int n = warp; n < nf; n += kWarps) {
        const FaceGeom& gn = geom[n];
        const d3 cn = gn.c;
        for (int t = lane; t < Q; t += 32) {
            const d3 r = ldg3(&qp[(size_t)n * Q + t]);
            s_sp[warp][t] = r;
            s_sl[warp][t] = r - cn;
        }
        for (int t = lane; t < NK * NM; t += 32) tot[t] = cx(0, 0);
        __syncwarp();
        const bool regular = centroid_distance(gm, gn) < thr;  // warp-uniform
        const bool coinc = gm.idx[0] == gn.idx[0] && gm.idx[1] == gn.idx[1] &&
                           gm.idx[2] == gn.idx[2];

        for (int p0 = 0; p0 < Q; p0 += PL) {
            const int p = p0 + lp;
            const bool act = p < Q;
            cplx S0[NK], Sq[NK][3], T0[TK ? NK : 1], Tq[TK ? NK : 1][3];
#pragma unroll
            for (int a = 0; a < NK; ++a) {
                S0[a] = cx(0, 0);
#pragma unroll
                for (int c = 0; c < 3; ++c) Sq[a][c] = cx(0, 0);
                if (TK) {
                    T0[a] = cx(0, 0);
#pragma unroll
                    for (int c = 0; c < 3; ++c) Tq[a][c] = cx(0, 0);
                }
            }
            if (act) {
                const d3 rp = s_tp[p];
                for (int q = lq; q < Q; q += G) {
                    const d3 rq = s_sp[warp][q], ql = s_sl[warp][q];
                    const double wq = s_w[q];
                    const d3 Rv = rp - rq;
                    const double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
                    cplx Gk[NK], gk[NK];
                    if (!regular) {
                        if (R < 1e-12) continue;
                        const double inv_R = 1.0 / R;
                        const double i4pR = 1.0 / (4.0 * kPi * R);
#pragma unroll
                        for (int a = 0; a < NK; ++a) green_std(R, inv_R, i4pR, kk[a], Gk[a], gk[a]);
                    } else {
#pragma unroll
                        for (int a = 0; a < NK; ++a) green_reg(R, kk[a], Gk[a], gk[a]);
                    }
#pragma unroll
                    for (int a = 0; a < NK; ++a) {
                        const cplx Gw = Gk[a] * wq;
                        S0[a] += Gw;
                        Sq[a][0] += Gw * ql.x; Sq[a][1] += Gw * ql.y; Sq[a][2] += Gw * ql.z;
                        if (TK) {
                            const cplx gw = gk[a] * wq;
                            T0[a] += gw;
                            Tq[a][0] += gw * ql.x; Tq[a][1] += gw * ql.y; Tq[a][2] += gw * ql.z;
                        }
                    }
                }
            }
            // Fold the test point in, reduce over the warp, accumulate.
            const d3 pl = act ? s_tl[p] : mk3(0, 0, 0);
            const double wp = act ? s_w[p] : 0.0;
            auto put = [&](int idx, cplx v) {
                warp_sum(v);
                if (lane == 0) tot[idx] += v;
            };
#pragma unroll
            for (int a = 0; a < NK; ++a) {
                const int b0 = a * NM;
                const cplx s0 = S0[a] * wp;
                const cplx sq[3] = {Sq[a][0] * wp, Sq[a][1] * wp, Sq[a][2] * wp};
                put(b0 + 0, s0);
                put(b0 + 1, s0 * pl.x); put(b0 + 2, s0 * pl.y); put(b0 + 3, s0 * pl.z);
                put(b0 + 4, sq[0]); put(b0 + 5, sq[1]); put(b0 + 6, sq[2]);
                put(b0 + 7, sq[0] * pl.x + sq[1] * pl.y + sq[2] * pl.z);
                if (TK) {
                    const cplx t0 = T0[a] * wp;
                    const cplx tq[3] = {Tq[a][0] * wp, Tq[a][1] * wp, Tq[a][2] * wp};
                    put(b0 + 8, t0);
                    put(b0 + 9, t0 * pl.x); put(b0 + 10, t0 * pl.y); put(b0 + 11, t0 * pl.z);
                    put(b0 + 12, tq[0]); put(b0 + 13, tq[1]); put(b0 + 14, tq[2]);
                    // p x Tq
                    put(b0 + 15, tq[2] * pl.y - tq[1] * pl.z);
                    put(b0 + 16, tq[0] * pl.z - tq[2] * pl.x);
                    put(b0 + 17, tq[1] * pl.x - tq[0] * pl.y);
                }
            }
        }
        __syncwarp();
        if (lane < 9) {
            const int j = lane / 3, i = lane - 3 * j;
            const d3 A = gm.A[j], B = gn.A[i];
            const d3 d = gm.fv[j] - gn.fv[i];
            const double scale = gm.len[j] * gn.len[i];
            const double AB = dot3(A, B);
            cplx* out = pairs + ((size_t)blockIdx.x * nf + n) * (NB * 9);
#pragma unroll
            for (int a = 0; a < NK; ++a) {
                const cplx* M = tot + a * NM;
                // TL_ji = l_j l_i [ 1/4 (Spq - Sp.B - A.Sq + (A.B) S0) - S0 / k^2 ]
                cplx t = M[7];
                t = t - (M[1] * B.x + M[2] * B.y + M[3] * B.z);
                t = t - (M[4] * A.x + M[5] * A.y + M[6] * A.z);
                t += M[0] * AB;
                out[a * 9 + lane] = (t * 0.25 - M[0] * (1.0 / (kk[a] * kk[a]))) * scale;
                if (TK) {
                    cplx tk = cx(0, 0);
                    if (!coinc) {
                        const d3 BxD = cross3(B, d);
                        const d3 DxA = cross3(d, A);
                        const double axbd = dot3(cross3(A, B), d);
                        cplx u = M[15] * d.x + M[16] * d.y + M[17] * d.z;
                        u = u - (M[9] * BxD.x + M[10] * BxD.y + M[11] * BxD.z);
                        u = u - (M[12] * DxA.x + M[13] * DxA.y + M[14] * DxA.z);
                        u += M[8] * axbd;
                        tk = u * (0.25 * scale);
                    }
                    out[(NK + a) * 9 + lane] = tk;
                }
            }
        }
        __syncwarp();
    }
}

// Lane slots used by pair_regular_pq_kernel for Q points: its lanes do useful
// work for this share of their iterations (1 for the flat kernel's Q x Q
// index space up to the last partial round).
inline double pq_lane_use(int Q) {
    const int G = Q >= 32 ? 1 : 32 / Q, PL = 32 / G;
    const int rounds = (Q + PL - 1) / PL, iters = (Q + G - 1) / G;
    return (double)Q * Q / (32.0 * rounds * iters);
}

// ------------------------------------------------------------ Wilton ----
struct Pots {
    double phi0, phi2, d;
    d3 phi1b, phi3b, r_pi;
};

__device__ __forceinline__ d3 normalize3(d3 a) {
    const double inv = 1.0 / sqrt(dot3(a, a));
    return a * inv;
}

// semi_analytic_integrals.cuh:35-92 and 563-667 in one pass.
__device__ Pots wilton(const d3 r, const d3 tri[3]) {
    Pots P;
    const d3 n = normalize3(cross3(tri[1] - tri[0], tri[2] - tri[0]));
    P.d = dot3(r - tri[0], n);
    P.r_pi = r - n * P.d;
    const double ad = fabs(P.d);
    const double eps9f = (double)1e-9f;
    P.phi0 = 0.0;
    P.phi2 = 0.0;
    P.phi1b = mk3(0, 0, 0);
    P.phi3b = mk3(0, 0, 0);
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const d3 vs = tri[e], ve = tri[(e + 1) % 3];
        const d3 th = normalize3(ve - vs);
        const d3 u = cross3(th, n);
        const d3 rs = vs - n * dot3(n, vs);
        const d3 re = ve - n * dot3(n, ve);
        const d3 to_s = rs - P.r_pi;
        const double su = dot3(to_s, u);
        const double p0 = fabs(su);
        const double orient = su >= 0.0 ? 1.0 : -1.0;
        const double lp = dot3(re - P.r_pi, th);
        const double lm = dot3(rs - P.r_pi, th);
        const double Pp = hypot(p0, lp), Pm = hypot(p0, lm);
        const double R0 = hypot(p0, ad);
        const double Rp = hypot(Pp, ad), Rm = hypot(Pm, ad);
        const double logt = (log(Rp) + log1p(lp / Rp)) - (log(Rm) + log1p(lm / Rm));
        double at = 0.0;
        if (ad > eps9f || ad > 1e-6)
            at = atan2(p0 * lp, R0 * R0 + ad * Rp) - atan2(p0 * lm, R0 * R0 + ad * Rm);
        if (p0 > eps9f) P.phi0 += orient * (p0 * logt - (ad > eps9f ? ad * at : 0.0));
        P.phi1b = P.phi1b + u * ((R0 * R0) * logt + (lp * Rp) - (lm * Rm));
        double term = 0.0;
        if (ad > 1e-6)
            term = (1.0 / ad) * at;
        else if (p0 > 1e-9)
            term = -((lp / (p0 * Pp)) - (lm / (p0 * Pm)));
        P.phi2 += orient * term;
        P.phi3b = P.phi3b - u * logt;
    }
    P.phi1b = P.phi1b * 0.5;
    return P;
}

__device__ __forceinline__ d3 psi1(const Pots& P, d3 fv) {
    return (P.phi1b + P.r_pi * P.phi0) - fv * P.phi0;
}

// semi_analytic_integrals.cuh:481-498 (k^2/2 formed in float).
__device__ __forceinline__ d3 upsilon(const Pots& P, d3 fv, d3 r, float k) {
    const d3 phi3 = P.phi3b + (P.r_pi - fv) * P.phi2;
    const d3 ps = psi1(P, fv);
    const float k2o2 = __fmul_rn(__fmul_rn(k, k), 0.5f);
    const d3 comb = phi3 + ps * (double)k2o2;
    return cross3(r - fv, comb) * -1.0;
}

// Singular (extracted) part of the near pairs, added to the pair blocks.
// dunavant_quadrature.cuh:769-875. Lanes over outer points p.
template <int NK>
__global__ void pair_singular_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                                     const float* __restrict__ qw_g, int Q, int nf, int m0,
                                     const int2* __restrict__ list, int count, double k0,
                                     double k1, bool with_tk, cplx* __restrict__ pairs) {
    const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp_global >= count) return;
    const int2 mn = list[warp_global];
    const FaceGeom gm = geom[mn.x];
    const FaceGeom gn = geom[mn.y];
    const bool coinc = gm.idx[0] == gn.idx[0] && gm.idx[1] == gn.idx[1] && gm.idx[2] == gn.idx[2];
    const double kk[2] = {k0, k1};
    double tl[NK][9], tk[NK][9];
#pragma unroll
    for (int a = 0; a < NK; ++a)
#pragma unroll
        for (int t = 0; t < 9; ++t) { tl[a][t] = 0.0; tk[a][t] = 0.0; }

    for (int p = lane; p < Q; p += 32) {
        const d3 rp = qp[(size_t)mn.x * Q + p];
        const double wp = (double)qw_g[p];
        const Pots P = wilton(rp, gn.v);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const d3 rm = rp - gm.fv[j];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const d3 ps = psi1(P, gn.fv[i]);
                const double db = 0.25 * dot3(rm, ps);
#pragma unroll
                for (int a = 0; a < NK; ++a) {
                    tl[a][j * 3 + i] += (db - 1.0 / (kk[a] * kk[a]) * P.phi0) * wp;
                    if (with_tk && !coinc) {
                        const d3 up = upsilon(P, gn.fv[i], rp, (float)kk[a]);
                        tk[a][j * 3 + i] += 0.25 * dot3(rm, up) * wp;
                    }
                }
            }
        }
    }
#pragma unroll
    for (int a = 0; a < NK; ++a)
#pragma unroll
        for (int t = 0; t < 9; ++t) { warp_sum(tl[a][t]); warp_sum(tk[a][t]); }
    if (lane < 9) {
        const int j = lane / 3, i = lane - 3 * j;
        const double as = 1.0 / (4.0 * kPi * gn.area);
        const double s = as * gm.len[j] * gn.len[i];
        const int NB = with_tk ? 2 * NK : NK;
        cplx* out = pairs + ((size_t)(mn.x - m0) * nf + mn.y) * (NB * 9);
        double tlv[NK], tkv[NK];
#pragma unroll
        for (int a = 0; a < NK; ++a) {
            // select entry `lane` without dynamic register indexing
            tlv[a] = 0.0; tkv[a] = 0.0;
#pragma unroll
            for (int t = 0; t < 9; ++t)
                if (t == lane) { tlv[a] = tl[a][t]; tkv[a] = tk[a][t]; }
            out[a * 9 + lane].re += tlv[a] * s;
            if (with_tk) out[(NK + a) * 9 + lane].re += tkv[a] * s;
        }
    }
}

// ---------------------------------------------- rotated (n x RWG) testing --
// Surface form B of nTL / nTK (dunavant_quadrature.cuh:342-480) with
// tau_mj = rho_mj x n_m and the TK kernel vector g R (R = r_p - r_q):
//   nTL = 1/4 (tau . rho_ni) G - 1/(2 k^2) tau . (g R),
//   nTK = 1/4 (tau x rho_ni) . (g R)   (not on the coincident face).
// With tau = t_p - t_j (t_p = p_l x n_m, t_j = A_j x n_m) and
// rho_ni = q_l - B_i, the nine RWG pairs follow from per-warp moments:
//   sum G tau.rho        = Stq - St.B - t_j.Sq + (t_j.B) S0
//   sum g tau.R          = TtR - t_j.TR
//   sum g (tau x rho).R  = U0 - B.V1 - t_j.V2 + (t_j x B).TR
// St = sum G t_p, Sq = sum G q_l, Stq = sum G t_p.q_l, TR = sum g R,
// TtR = sum g t_p.R, U0 = sum g (t_p x q_l).R, V1 = sum g R x t_p,
// V2 = sum g q_l x R.
template <int NK, bool NTK>
struct MomentsN {
    cplx S0[NK], St[NK][3], Sq[NK][3], Stq[NK];
    cplx TR[NK][3], TtR[NK];
    cplx U0[NTK ? NK : 1], V1[NTK ? NK : 1][3], V2[NTK ? NK : 1][3];
};

__device__ __forceinline__ d3 face_normal(const FaceGeom& g) {
    return normalize3(cross3(g.v[1] - g.v[0], g.v[2] - g.v[0]));
}

// The line form's unit normal: cross product divided by its length
// (dunavant_quadrature.cuh:521-525), and twice the area.
__device__ __forceinline__ d3 face_normal_div(const FaceGeom& g) {
    const d3 c = cross3(g.v[1] - g.v[0], g.v[2] - g.v[0]);
    const double l = sqrt(dot3(c, c));
    return mk3(c.x / l, c.y / l, c.z / l);
}

// semi_analytic_integrals.cuh:108-171 (calculate_phi_0, on the testing edges
// of the line form): an edge whose end is within 1e-9 of r is skipped, and on
// an edge's line (R0 < 1e-8) the end distances are regularised by 1e-8.
__device__ double phi0_line(const d3 r, const d3 tri[3]) {
    const d3 n = normalize3(cross3(tri[1] - tri[0], tri[2] - tri[0]));
    const double d = dot3(r - tri[0], n);
    const d3 r_pi = r - n * d;
    const double ad = fabs(d);
    double phi0 = 0.0;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
        const d3 vs = tri[e], ve = tri[(e + 1) % 3];
        const d3 th = normalize3(ve - vs);
        const d3 u = cross3(th, n);
        const d3 rs = vs - n * dot3(n, vs);
        const d3 re = ve - n * dot3(n, ve);
        const double su = dot3(rs - r_pi, u);
        const double p0 = fabs(su);
        const double orient = su >= 0.0 ? 1.0 : -1.0;
        const double lp = dot3(re - r_pi, th);
        const double lm = dot3(rs - r_pi, th);
        const double Pp = hypot(p0, lp), Pm = hypot(p0, lm);
        const double R0 = hypot(p0, ad);
        double Rp = hypot(Pp, ad), Rm = hypot(Pm, ad);
        if (Rp < 1e-9 || Rm < 1e-9) continue;
        if (R0 < 1e-8) {
            // Rounded product, then rounded sum, as the reference's
            // sqrt(pow(R, 2) + pow(eps, 2)): where 1e-16 is below half an ulp
            // of R^2 the regularisation has no effect and, on the edge line
            // beyond its start, log1p(-1) makes the reference's value
            // infinite; the same inputs give the same values here.
            Rp = sqrt(__dadd_rn(__dmul_rn(Rp, Rp), 1e-8 * 1e-8));
            Rm = sqrt(__dadd_rn(__dmul_rn(Rm, Rm), 1e-8 * 1e-8));
        }
        const double logt = (log(Rp) + log1p(lp / Rp)) - (log(Rm) + log1p(lm / Rm));
        double at = 0.0;
        if (ad > 1e-9) at = atan2(p0 * lp, R0 * R0 + ad * Rp) - atan2(p0 * lm, R0 * R0 + ad * Rm);
        phi0 += orient * (p0 * logt - ad * at);
    }
    return phi0;
}

// Regular (or extracted-kernel) double quadrature of the rotated-testing
// blocks of all face pairs (m, n), m in [m0, m1). Output per pair: nTL for
// each wavenumber, then (NTK) nTK for each, 3x3 complex each, in the slots
// pair_regular_kernel gives TL and TK.
// FORM_A: the area part of the line form A (dunavant_quadrature.cuh:492-567):
// nTL without the gradient term (pair_line_kernel adds the testing-edge line
// integral), n_m as the cross product divided by its length.
template <int NK, bool NTK, bool FORM_A>
__global__ void __launch_bounds__(kWarps * 32, 1)
pair_regular_n_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                      const float* __restrict__ qw_g, int Q, int nf, int m0, double k0, double k1,
                      float thr, int exact, cplx* __restrict__ pairs) {
    constexpr int NB = NTK ? 2 * NK : NK;
    __shared__ d3 s_tp[kMaxQ], s_tt[kMaxQ];
    __shared__ double s_w[kMaxQ];
    __shared__ d3 s_sp[kWarps][kMaxQ], s_sl[kWarps][kMaxQ];

    const int m = m0 + blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const FaceGeom& gm = geom[m];
    const d3 nm = FORM_A ? face_normal_div(gm) : face_normal(gm);
    for (int t = threadIdx.x; t < Q; t += blockDim.x) {
        const d3 r = qp[(size_t)m * Q + t];
        s_tp[t] = r;
        s_tt[t] = cross3(r - gm.c, nm);
        s_w[t] = (double)qw_g[t];
    }
    __syncthreads();
    const double kk[2] = {k0, k1};
    const int QQ = Q * Q;

    for (int n = warp; n < nf; n += kWarps) {
        const FaceGeom& gn = geom[n];
        const d3 cn = gn.c;
        for (int t = lane; t < Q; t += 32) {
            const d3 r = ldg3(&qp[(size_t)n * Q + t]);
            s_sp[warp][t] = r;
            s_sl[warp][t] = r - cn;
        }
        __syncwarp();
        const bool regular = near_pair(gm, gn, thr, exact);  // warp-uniform
        const bool coinc = gm.idx[0] == gn.idx[0] && gm.idx[1] == gn.idx[1] &&
                           gm.idx[2] == gn.idx[2];

        MomentsN<NK, NTK> M;
#pragma unroll
        for (int a = 0; a < NK; ++a) {
            M.S0[a] = cx(0, 0); M.Stq[a] = cx(0, 0); M.TtR[a] = cx(0, 0);
#pragma unroll
            for (int c = 0; c < 3; ++c) { M.St[a][c] = cx(0, 0); M.Sq[a][c] = cx(0, 0); M.TR[a][c] = cx(0, 0); }
            if (NTK) {
                M.U0[a] = cx(0, 0);
#pragma unroll
                for (int c = 0; c < 3; ++c) { M.V1[a][c] = cx(0, 0); M.V2[a][c] = cx(0, 0); }
            }
        }

        for (int idx = lane; idx < QQ; idx += 32) {
            const int p = idx / Q, q = idx - p * Q;
            const d3 rp = s_tp[p], rq = s_sp[warp][q];
            const d3 tp = s_tt[p], ql = s_sl[warp][q];
            const double ww = s_w[p] * s_w[q];
            const d3 Rv = rp - rq;
            const double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
            if (!regular && R < 1e-12) continue;
            const double tq = dot3(tp, ql), tR = dot3(tp, Rv);
            double u0 = 0.0;
            d3 v1 = mk3(0, 0, 0), v2 = mk3(0, 0, 0);
            if (NTK) {
                u0 = dot3(cross3(tp, ql), Rv);
                v1 = cross3(Rv, tp);
                v2 = cross3(ql, Rv);
            }
            const double inv_R = regular ? 0.0 : 1.0 / R;
            const double i4pR = regular ? 0.0 : 1.0 / (4.0 * kPi * R);
#pragma unroll
            for (int a = 0; a < NK; ++a) {
                cplx G, g;
                if (regular) green_reg(R, kk[a], G, g);
                else green_std(R, inv_R, i4pR, kk[a], G, g);
                const cplx Gw = G * ww, gw = g * ww;
                M.S0[a] += Gw;
                M.St[a][0] += Gw * tp.x; M.St[a][1] += Gw * tp.y; M.St[a][2] += Gw * tp.z;
                M.Sq[a][0] += Gw * ql.x; M.Sq[a][1] += Gw * ql.y; M.Sq[a][2] += Gw * ql.z;
                M.Stq[a] += Gw * tq;
                M.TR[a][0] += gw * Rv.x; M.TR[a][1] += gw * Rv.y; M.TR[a][2] += gw * Rv.z;
                M.TtR[a] += gw * tR;
                if (NTK) {
                    M.U0[a] += gw * u0;
                    M.V1[a][0] += gw * v1.x; M.V1[a][1] += gw * v1.y; M.V1[a][2] += gw * v1.z;
                    M.V2[a][0] += gw * v2.x; M.V2[a][1] += gw * v2.y; M.V2[a][2] += gw * v2.z;
                }
            }
        }
#pragma unroll
        for (int a = 0; a < NK; ++a) {
            warp_sum(M.S0[a]); warp_sum(M.Stq[a]); warp_sum(M.TtR[a]);
#pragma unroll
            for (int c = 0; c < 3; ++c) { warp_sum(M.St[a][c]); warp_sum(M.Sq[a][c]); warp_sum(M.TR[a][c]); }
            if (NTK) {
                warp_sum(M.U0[a]);
#pragma unroll
                for (int c = 0; c < 3; ++c) { warp_sum(M.V1[a][c]); warp_sum(M.V2[a][c]); }
            }
        }
        if (lane < 9) {
            const int j = lane / 3, i = lane - 3 * j;
            const d3 tj = cross3(gm.A[j], nm), B = gn.A[i];
            const double scale = gm.len[j] * gn.len[i];
            const double tjB = dot3(tj, B);
            const d3 tjxB = cross3(tj, B);
            cplx* out = pairs + ((size_t)blockIdx.x * nf + n) * (NB * 9);
#pragma unroll
            for (int a = 0; a < NK; ++a) {
                cplx s = M.Stq[a];
                s = s - (M.St[a][0] * B.x + M.St[a][1] * B.y + M.St[a][2] * B.z);
                s = s - (M.Sq[a][0] * tj.x + M.Sq[a][1] * tj.y + M.Sq[a][2] * tj.z);
                s += M.S0[a] * tjB;
                if (FORM_A) {
                    out[a * 9 + lane] = s * (0.25 * scale);
                } else {
                    const cplx t = M.TtR[a] - (M.TR[a][0] * tj.x + M.TR[a][1] * tj.y + M.TR[a][2] * tj.z);
                    out[a * 9 + lane] = (s * 0.25 + t * (-0.5 / (kk[a] * kk[a]))) * scale;
                }
                if (NTK) {
                    cplx u = cx(0, 0);
                    if (!coinc) {
                        u = M.U0[a];
                        u = u - (M.V1[a][0] * B.x + M.V1[a][1] * B.y + M.V1[a][2] * B.z);
                        u = u - (M.V2[a][0] * tj.x + M.V2[a][1] * tj.y + M.V2[a][2] * tj.z);
                        u += M.TR[a][0] * tjxB.x + M.TR[a][1] * tjxB.y + M.TR[a][2] * tjxB.z;
                        u = u * (0.25 * scale);
                    }
                    out[(NK + a) * 9 + lane] = u;
                }
            }
        }
        __syncwarp();
    }
}

// Singular (extracted) part of the rotated-testing blocks of the near pairs,
// added to the pair blocks. One warp per pair, lanes over outer points.
// Surface form B (dunavant_quadrature.cuh:889-1040), per outer point with
// phi_1 = phi_1b - d phi_0 n_n and the extracted gradient phi_3b - d phi_2 n_n:
//   nTL += 1/2 tau . (phi_1 + 1/2 R_i phi_0 + gradient / k^2)
//          (the gradient left out on the coincident face),
// then e_mj e_ni / (4 pi A_n). Line form A (1040-1179): nTL += 1/4 w tau . Psi_1
// on the area, scaled alike, plus the testing-edge sum
// sum_e sum_q L_e w_q (tau . nu_e) phi_0(r_eq) scaled by e_mj e_ni / (8 pi A_m A_n k^2)
// (lanes over the 3 NG edge points). Both forms:
//   nTK += 1/4 tau . Upsilon_coul (not on the coincident face).
template <int NK, bool FORM_A>
__global__ void pair_singular_n_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                                       const float* __restrict__ qw_g, int Q, int nf, int m0,
                                       const int2* __restrict__ list, int count, double k0,
                                       double k1, bool with_ntk, const float* __restrict__ gl_t,
                                       const float* __restrict__ gl_w, int NG, cplx* __restrict__ pairs) {
    const int warp_global = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp_global >= count) return;
    const int2 mn = list[warp_global];
    const FaceGeom gm = geom[mn.x];
    const FaceGeom gn = geom[mn.y];
    const bool coinc = gm.idx[0] == gn.idx[0] && gm.idx[1] == gn.idx[1] && gm.idx[2] == gn.idx[2];
    const d3 nm = FORM_A ? face_normal_div(gm) : face_normal(gm);
    const d3 nn = face_normal(gn);
    const double kk[2] = {k0, k1};
    double tl[NK][9], tk[NK][9];
#pragma unroll
    for (int a = 0; a < NK; ++a)
#pragma unroll
        for (int t = 0; t < 9; ++t) { tl[a][t] = 0.0; tk[a][t] = 0.0; }

    for (int p = lane; p < Q; p += 32) {
        const d3 rp = qp[(size_t)mn.x * Q + p];
        const double wp = (double)qw_g[p];
        const Pots P = wilton(rp, gn.v);
        const d3 phi1 = P.phi1b - nn * (P.d * P.phi0);
        const d3 grad = P.phi3b - nn * (P.d * P.phi2);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const d3 tau = cross3(rp - gm.fv[j], nm);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                if (FORM_A) {
                    const double an = 0.25 * wp * dot3(tau, psi1(P, gn.fv[i]));
#pragma unroll
                    for (int a = 0; a < NK; ++a) tl[a][j * 3 + i] += an;
                } else {
                    const d3 br = phi1 + ((rp - gn.fv[i]) * 0.5) * P.phi0;
#pragma unroll
                    for (int a = 0; a < NK; ++a) {
                        const d3 V = coinc ? br : br + grad * (1.0 / (kk[a] * kk[a]));
                        tl[a][j * 3 + i] += 0.5 * dot3(tau, V) * wp;
                    }
                }
                if (with_ntk && !coinc) {
#pragma unroll
                    for (int a = 0; a < NK; ++a) {
                        const d3 up = upsilon(P, gn.fv[i], rp, (float)kk[a]);
                        tk[a][j * 3 + i] += (FORM_A ? 0.25 * wp * dot3(tau, up) : 0.25 * dot3(tau, up) * wp);
                    }
                }
            }
        }
    }
    double line[3] = {0.0, 0.0, 0.0};
    if (FORM_A) {
        for (int it = lane; it < 3 * NG; it += 32) {
            const int e = it / NG, q = it - e * NG;
            const d3 vA = gm.v[e], vB = gm.v[e == 2 ? 0 : e + 1];
            const d3 E = vB - vA;
            const double Le = sqrt(dot3(E, E));
            const d3 c = cross3(E, nm);
            const d3 nu = mk3(c.x / Le, c.y / Le, c.z / Le);
            const double t = (double)gl_t[q], wl = (double)gl_w[q];
            const d3 req = mk3(vA.x + t * (vB.x - vA.x), vA.y + t * (vB.y - vA.y), vA.z + t * (vB.z - vA.z));
            const double ph0 = phi0_line(req, gn.v);
#pragma unroll
            for (int j = 0; j < 3; ++j) line[j] += Le * wl * dot3(cross3(req - gm.fv[j], nm), nu) * ph0;
        }
#pragma unroll
        for (int j = 0; j < 3; ++j) warp_sum(line[j]);
    }
#pragma unroll
    for (int a = 0; a < NK; ++a)
#pragma unroll
        for (int t = 0; t < 9; ++t) { warp_sum(tl[a][t]); warp_sum(tk[a][t]); }
    if (lane < 9) {
        const int j = lane / 3, i = lane - 3 * j;
        const double as = 1.0 / (4.0 * kPi * gn.area);
        const double s = as * gm.len[j] * gn.len[i];
        const int NB = with_ntk ? 2 * NK : NK;
        cplx* out = pairs + ((size_t)(mn.x - m0) * nf + mn.y) * (NB * 9);
        const double edges = gm.len[j] * gn.len[i];
        const double ls = FORM_A ? 1.0 / (8.0 * kPi * gm.area * gn.area) : 0.0;
        double lj = 0.0;
#pragma unroll
        for (int jj = 0; jj < 3; ++jj)
            if (jj == j) lj = line[jj];
#pragma unroll
        for (int a = 0; a < NK; ++a) {
            double tlv = 0.0, tkv = 0.0;
#pragma unroll
            for (int t = 0; t < 9; ++t)
                if (t == lane) { tlv = tl[a][t]; tkv = tk[a][t]; }
            if (FORM_A) {
                out[a * 9 + lane].re += tlv * (edges * as) + edges * ls * lj / (kk[a] * kk[a]);
                if (with_ntk) out[(NK + a) * 9 + lane].re += tkv * (edges * as);
            } else {
                out[a * 9 + lane].re += tlv * s;
                if (with_ntk) out[(NK + a) * 9 + lane].re += tkv * s;
            }
        }
    }
}

// Testing-edge line integral of the nTL form A (dunavant_quadrature.cuh:598-672),
// added to the nTL blocks of every face pair of the slab: for each test edge
// e (v_A -> v_B), Gauss-Legendre point t_q and source point p,
//   nTL_ji += l_j l_i (L_e / 2A_m) (tau_j(r_eq) . nu_e) G(r_eq, r_p) w_q w_p / k^2,
// the same for every source basis i. tau_j . nu_e is linear in t_q, so each
// warp (one face pair) accumulates sum w G and sum w t G per edge and
// wavenumber; 9 lanes expand them. Standard or extracted kernel as the pair's
// area quadrature.
template <int NK>
__global__ void __launch_bounds__(kWarps * 32)
pair_line_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                 const float* __restrict__ qw_g, int Q, int nf, int m0, double k0, double k1,
                 float thr, int exact, const float* __restrict__ gl_t, const float* __restrict__ gl_w,
                 int NG, int NB, cplx* __restrict__ pairs) {
    __shared__ double s_w[kMaxQ];
    __shared__ double s_t[20], s_wl[20];
    const int m = m0 + blockIdx.x;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = threadIdx.x; t < Q; t += blockDim.x) s_w[t] = (double)qw_g[t];
    for (int t = threadIdx.x; t < NG; t += blockDim.x) { s_t[t] = (double)gl_t[t]; s_wl[t] = (double)gl_w[t]; }
    __syncthreads();
    const FaceGeom& gm = geom[m];
    const d3 nm = face_normal_div(gm);
    const d3 cr = cross3(gm.v[1] - gm.v[0], gm.v[2] - gm.v[0]);
    const double twoA = sqrt(dot3(cr, cr));
    const double kk[2] = {k0, k1};
    const int items = NG * Q;
    for (int n = warp; n < nf; n += kWarps) {
        const FaceGeom& gn = geom[n];
        const bool regular = near_pair(gm, gn, thr, exact);  // warp-uniform
        cplx M0[3][NK], M1[3][NK];
#pragma unroll
        for (int e = 0; e < 3; ++e)
#pragma unroll
            for (int a = 0; a < NK; ++a) { M0[e][a] = cx(0, 0); M1[e][a] = cx(0, 0); }
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const d3 vA = gm.v[e], vB = gm.v[e == 2 ? 0 : e + 1];
            for (int it = lane; it < items; it += 32) {
                const int q = it / Q, p = it - q * Q;
                const double t = s_t[q];
                const d3 req = mk3(vA.x + t * (vB.x - vA.x), vA.y + t * (vB.y - vA.y), vA.z + t * (vB.z - vA.z));
                const d3 rq = ldg3(&qp[(size_t)n * Q + p]);
                const d3 Rv = req - rq;
                const double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
                if (!regular && R < 1e-12) continue;
                const double w = s_wl[q] * s_w[p];
                const double inv_R = regular ? 0.0 : 1.0 / R;
                const double i4pR = regular ? 0.0 : 1.0 / (4.0 * kPi * R);
#pragma unroll
                for (int a = 0; a < NK; ++a) {
                    cplx G, g;
                    if (regular) green_reg(R, kk[a], G, g);
                    else green_std(R, inv_R, i4pR, kk[a], G, g);
                    const cplx Gw = G * w;
                    M0[e][a] += Gw;
                    M1[e][a] += Gw * t;
                }
            }
        }
#pragma unroll
        for (int e = 0; e < 3; ++e)
#pragma unroll
            for (int a = 0; a < NK; ++a) { warp_sum(M0[e][a]); warp_sum(M1[e][a]); }
        if (lane < 9) {
            const int j = lane / 3, i = lane - 3 * j;
            cplx acc[NK];
#pragma unroll
            for (int a = 0; a < NK; ++a) acc[a] = cx(0, 0);
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                const d3 vA = gm.v[e], vB = gm.v[e == 2 ? 0 : e + 1];
                const d3 E = vB - vA;
                const double Le = sqrt(dot3(E, E));
                const d3 c = cross3(E, nm);
                const d3 nu = mk3(c.x / Le, c.y / Le, c.z / Le);
                const double geomf = Le / twoA;
                // tau_j(r_eq) . nu_e = c0 + t c1
                const double c0 = dot3(cross3(vA - gm.fv[j], nm), nu);
                const double c1 = dot3(cross3(E, nm), nu);
#pragma unroll
                for (int a = 0; a < NK; ++a) acc[a] += (M0[e][a] * c0 + M1[e][a] * c1) * geomf;
            }
            const double scale = gm.len[j] * gn.len[i];
            cplx* out = pairs + ((size_t)blockIdx.x * nf + n) * (NB * 9);
#pragma unroll
            for (int a = 0; a < NK; ++a) out[a * 9 + lane] += acc[a] * (scale / (kk[a] * kk[a]));
        }
        __syncwarp();
    }
}

// RWG Gram block <f_j, f_i> of each face (dunavant_quadrature.cuh:1261-1326)
// with the reference's float dot product, weight and scale. One thread per
// face, gram[9 f + 3 j + i].
__global__ void gram_face_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                                 const float* __restrict__ qw_g, int Q, int nf, double* __restrict__ gram) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const FaceGeom& g = geom[f];
    double R[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) R[e] = 0.0;
    for (int p = 0; p < Q; ++p) {
        const float wp = qw_g[p];
        const d3 rp = qp[(size_t)f * Q + p];
        d3 rho[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) rho[i] = rp - g.fv[i];
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const double d = __dadd_rn(__dadd_rn(__dmul_rn(rho[j].x, rho[i].x), __dmul_rn(rho[j].y, rho[i].y)),
                                           __dmul_rn(rho[j].z, rho[i].z));
                R[j * 3 + i] += (double)__fmul_rn(wp, (float)d);
            }
    }
    const float area = (float)g.area;
    const float sc = __fdiv_rn(1.f, __fmul_rn(4.f, area));
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float fs = __fmul_rn(__fmul_rn(sc, (float)g.len[j]), (float)g.len[i]);
            gram[(size_t)f * 9 + j * 3 + i] = R[j * 3 + i] * (double)fs;
        }
}

// ------------------------------------------------------------ GSTC mass --
// Mass block of tensor t (0..3: the Y blocks ee, em, me, mm after the perp
// transform; 4..7 the Z blocks) of face g for the 2x2 tensor block
// (t00 t01; t10 t11): out[j*3+i] for local test edge j and source edge i.
// Linear in the four tensor entries.
__device__ void mass_tensor_block(const FaceGeom& g, const d3* __restrict__ qpf, const float* __restrict__ qw_g,
                                  int Q, int basis, int t, cplx t00, cplx t01, cplx t10, cplx t11,
                                  cplx (&out)[9]) {
    // Frame: gstc_tensor_utils.cuh:72-147.
    d3 u, w;
    if (basis == 0) {
        const d3 e1 = g.v[1] - g.v[0], e2 = g.v[2] - g.v[0];
        const d3 nn = cross3(e1, e2);
        const double l1 = sqrt(dot3(e1, e1)), ln = sqrt(dot3(nn, nn));
        if (l1 < 1e-20 || ln < 1e-20) {
            u = mk3(1, 0, 0); w = mk3(0, 1, 0);
        } else {
            const d3 nh = nn * (1.0 / ln);
            u = e1 * (1.0 / l1);
            w = cross3(nh, u);
        }
    } else {
        const d3 c = mk3((g.v[0].x + g.v[1].x + g.v[2].x) / 3.0, (g.v[0].y + g.v[1].y + g.v[2].y) / 3.0,
                         (g.v[0].z + g.v[1].z + g.v[2].z) / 3.0);
        const double r = sqrt(dot3(c, c));
        if (r < 1e-12) {
            u = mk3(1, 0, 0); w = mk3(0, 1, 0);
        } else {
            double ct = c.z / r;
            ct = ct > 1.0 ? 1.0 : (ct < -1.0 ? -1.0 : ct);
            const double th = acos(ct), ph = atan2(c.y, c.x);
            const double cth = cos(th), sth = sin(th), cph = cos(ph), sph = sin(ph);
            u = mk3(cth * cph, cth * sph, -sth);
            w = mk3(-sph, cph, 0.0);
        }
    }
    // Lift the 2x2 block (gstc_tensor_utils.cuh:184-238).
    const double uc[3] = {u.x, u.y, u.z}, wc[3] = {w.x, w.y, w.z};
    cplx T[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            cplx s = cx(0, 0);
            s += t00 * (uc[i] * uc[j]);
            s += t01 * (uc[i] * wc[j]);
            s += t10 * (wc[i] * uc[j]);
            s += t11 * (wc[i] * wc[j]);
            T[i][j] = s;
        }
    if (t < 4) {
        // Y_perp = -[n]x Y [n]x with float-cast entries (gstc_tensor_utils.cuh:269-309).
        const d3 n = normalize3(cross3(g.v[1] - g.v[0], g.v[2] - g.v[0]));
        const double N[3][3] = {{0.0, (double)(float)(-n.z), (double)(float)n.y},
                                {(double)(float)n.z, 0.0, (double)(float)(-n.x)},
                                {(double)(float)(-n.y), (double)(float)n.x, 0.0}};
        cplx tmp[3][3];
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                cplx s = cx(0, 0);
#pragma unroll
                for (int k = 0; k < 3; ++k) s += T[r][k] * N[k][c];
                tmp[r][c] = s;
            }
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                cplx s = cx(0, 0);
#pragma unroll
                for (int k = 0; k < 3; ++k) s += tmp[k][c] * N[r][k];
                T[r][c] = cx(-s.re, -s.im);
            }
    }
    // Mass quadrature with float geometry (dunavant_quadrature.cuh:1422-1508).
    const float area = (float)g.area;
    float el[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) el[i] = (float)g.len[i];
    cplx R[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) R[e] = cx(0, 0);
    for (int p = 0; p < Q; ++p) {
        const double wp = (double)qw_g[p];
        const d3 rp = qpf[p];
        d3 rho[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) rho[i] = rp - g.fv[i];
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const cplx tx = T[0][0] * rho[i].x + (T[0][1] * rho[i].y + T[0][2] * rho[i].z);
                const cplx ty = T[1][0] * rho[i].x + (T[1][1] * rho[i].y + T[1][2] * rho[i].z);
                const cplx tz = T[2][0] * rho[i].x + (T[2][1] * rho[i].y + T[2][2] * rho[i].z);
                const cplx ig = tx * rho[j].x + (ty * rho[j].y + tz * rho[j].z);
                R[j * 3 + i] += ig * wp;
            }
    }
    const float sc = __fdiv_rn(1.f, __fmul_rn(4.f, area));
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const float fs = __fmul_rn(__fmul_rn(sc, el[j]), el[i]);
            out[j * 3 + i] = R[j * 3 + i] * (double)fs;
        }
}

// One thread per (face, tensor t in 0..7).
__global__ void mass_face_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                                 const float* __restrict__ qw_g, int Q, int nf,
                                 const cplx* __restrict__ tensors, int uniform, int basis,
                                 cplx* __restrict__ mass) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nf * 8) return;
    const int f = id >> 3, t = id & 7;
    const cplx* tp = tensors + (uniform ? 0 : (size_t)f * 32) + (t >= 4 ? 16 : 0);
    const int blk = t & 3, r0 = (blk >> 1) * 2, c0 = (blk & 1) * 2;
    cplx out[9];
    mass_tensor_block(geom[f], qp + (size_t)f * Q, qw_g, Q, basis, t, tp[r0 * 4 + c0], tp[r0 * 4 + c0 + 1],
                      tp[(r0 + 1) * 4 + c0], tp[(r0 + 1) * 4 + c0 + 1], out);
#pragma unroll
    for (int e = 0; e < 9; ++e) mass[((size_t)f * 8 + t) * 9 + e] = out[e];
}

// A_M'' block pattern of the 8 mass values of one (test, source) edge pair
// with the 1/2 and 1/8 factors and the eta0 scales of the M rows/columns
// (sie_kernels_assembly.cuh:565-592), added into the 4x4 region block.
__device__ __forceinline__ void add_mass_pattern(const cplx (&mv)[8], double me, double me2, cplx (&blk)[4][4]) {
    const cplx Yee = mv[0], Yem = mv[1], Yme = mv[2], Ymm = mv[3];
    const cplx Zee = mv[4], Zem = mv[5], Zme = mv[6], Zmm = mv[7];
    const double f = 0.5, fq = 0.125;
    const cplx ap = Zee * f + Ymm * fq, am = Zee * f - Ymm * fq;
    const cplx bp = Zem * f + Yme * fq, bm = Zem * f - Yme * fq;
    const cplx cp = Zme * f + Yem * fq, cm = Zme * f - Yem * fq;
    const cplx dp = Zmm * f + Yee * fq, dm = Zmm * f - Yee * fq;
    const double s1 = 1.0, se_ = me, s2 = me2;
    blk[0][0] += ap * s1; blk[0][1] += bm * se_; blk[0][2] += am * s1; blk[0][3] += bp * se_;
    blk[1][0] += cm * se_; blk[1][1] += dp * s2; blk[1][2] += cp * se_; blk[1][3] += dm * s2;
    blk[2][0] += am * s1; blk[2][1] += bp * se_; blk[2][2] += ap * s1; blk[2][3] += bm * se_;
    blk[3][0] += cp * se_; blk[3][1] += dm * s2; blk[3][2] += cm * se_; blk[3][3] += dp * s2;
}

// Adjoint contraction for the GSTC tensors: s[f*32 + k] = lambda^H
// (dZ / d record[f][k]) x, record[f] = (Lambda, Lambda^{-1}) row-major.
// Z depends on the record only through the face's own mass blocks, and
// linearly, so dZ / d entry is the mass block of a unit entry placed by the
// A_M'' pattern on the face's 3 x 3 local edge pairs. One thread per (face, t).
__global__ void tensor_grad_kernel(const FaceGeom* __restrict__ geom, const d3* __restrict__ qp,
                                   const float* __restrict__ qw_g, int Q, int nf, int ne,
                                   const int* __restrict__ FE, int basis, double me, double me2,
                                   const cplx* __restrict__ lam, const cplx* __restrict__ x,
                                   cplx* __restrict__ s_out) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nf * 8) return;
    const int f = id >> 3, t = id & 7;
    // Pattern coefficients of tensor t: the 4x4 region block of a unit value.
    cplx mv[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) mv[k] = cx(k == t ? 1.0 : 0.0, 0.0);
    cplx C[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) C[r][c] = cx(0, 0);
    add_mass_pattern(mv, me, me2, C);
    // G[j][i] = sum_{r,c} C[r][c] conj(lambda[e_j + r E]) x[e_i + c E].
    const int64_t E = ne;
    int e[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) e[k] = FE[3 * f + k];
    cplx G[9];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            cplx acc = cx(0, 0);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const cplx lv = lam[e[j] + r * E];
                const cplx lc = cx(lv.re, -lv.im);
#pragma unroll
                for (int c = 0; c < 4; ++c) acc += C[r][c] * (lc * x[e[i] + c * E]);
            }
            G[j * 3 + i] = acc;
        }
    const int blk = t & 3, r0 = (blk >> 1) * 2, c0 = (blk & 1) * 2;
    const FaceGeom g = geom[f];
#pragma unroll 1
    for (int ab = 0; ab < 4; ++ab) {
        const cplx one = cx(1, 0), zero = cx(0, 0);
        cplx out[9];
        mass_tensor_block(g, qp + (size_t)f * Q, qw_g, Q, basis, t, ab == 0 ? one : zero, ab == 1 ? one : zero,
                          ab == 2 ? one : zero, ab == 3 ? one : zero, out);
        cplx sacc = cx(0, 0);
#pragma unroll
        for (int k = 0; k < 9; ++k) sacc += G[k] * out[k];
        const int a = ab >> 1, b = ab & 1;
        s_out[(size_t)f * 32 + (t >= 4 ? 16 : 0) + (r0 + a) * 4 + (c0 + b)] = sacc;
    }
}

// ------------------------------------------------------------ gather ----
struct GatherParams {
    int formulation;
    int variant;  // 0 tangential testing; 1 N-EFIE / N-PMCHWT; 2 N-MFIE / N-Muller
    int nf, ne;
    int m0, m1;
    int NB;
    cplx c_jj[2], c_mm[2];
    double s_jm, s_mm;
    double me, me2;  // mass scales (float eta0, eta0^2)
    // N-Muller (dielectric_kernels.cu:433-488): z_jj = w_em[1] nTL2 - w_em[0] nTL1
    // (w_em = omega eps mu), z_jm = eps2 nTK2 - eps1 nTK1 - eps_f G,
    // z_mj = mu2 nTK2 - mu1 nTK1 - mu_f G on the same face.
    double w_em[2], eps[2], mu[2], eps_f, mu_f;
    const double* gram;  // RWG Gram blocks (N-MFIE, N-Muller), 9 per face
};

// The region block (1x1 PEC, 2x2 PMCHWT, 4x4 GSTC) of Z at test edge te and
// source edge se from the face-pair blocks of the test faces in [m0, m1);
// false when te has no incident face in the slab.
__device__ __forceinline__ bool edge_pair_block(const cplx* __restrict__ pairs, const cplx* __restrict__ mass,
                                                const int* __restrict__ inc, const GatherParams& P, int te, int se,
                                                cplx (&blk)[4][4]) {
    const int it[2] = {inc[2 * te], inc[2 * te + 1]};
    const int is[2] = {inc[2 * se], inc[2 * se + 1]};
    bool any = false;
#pragma unroll
    for (int a = 0; a < 2; ++a)
        if (it[a] >= 0 && it[a] / 3 >= P.m0 && it[a] / 3 < P.m1) any = true;
    if (!any) return false;

    cplx acc[4] = {cx(0, 0), cx(0, 0), cx(0, 0), cx(0, 0)};
    cplx mass_acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) mass_acc[k] = cx(0, 0);
    bool has_mass = false;
    double gram_acc = 0.0;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        if (it[a] < 0) continue;
        const int m = it[a] / 3, j = it[a] - 3 * m;
        if (m < P.m0 || m >= P.m1) continue;
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            if (is[b] < 0) continue;
            const int n = is[b] / 3, i = is[b] - 3 * n;
            const cplx* pb = pairs + ((size_t)(m - P.m0) * P.nf + n) * (P.NB * 9) + j * 3 + i;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < P.NB) acc[k] += pb[k * 9];
            if (P.formulation == SIEB200_GSTC && m == n) {
                has_mass = true;
                const cplx* mb = mass + (size_t)m * 72 + j * 3 + i;
#pragma unroll
                for (int k = 0; k < 8; ++k) mass_acc[k] += mb[k * 9];
            }
            if (P.variant == 2 && m == n) gram_acc += P.gram[(size_t)m * 9 + j * 3 + i];
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) blk[r][c] = cx(0, 0);
    if (P.formulation == SIEB200_PEC_EFIE && P.variant == 2) {
        // N-MFIE (pec_solver.cu:171-240): 1/2 Gram on the same face, - nTK2.
        blk[0][0] = cx(0.5 * gram_acc, 0.0) - acc[1];
    } else if (P.formulation == SIEB200_PEC_EFIE) {
        blk[0][0] = P.c_jj[1] * acc[0];
    } else if (P.formulation == SIEB200_PMCHWT && P.variant == 2) {
        // acc: nTL1, nTL2, nTK1, nTK2.
        const cplx jj = acc[1] * cx(0.0, P.w_em[1]) - acc[0] * cx(0.0, P.w_em[0]);
        const cplx jm = acc[3] * P.eps[1] - acc[2] * P.eps[0] - cx(P.eps_f * gram_acc, 0.0);
        const cplx mj = acc[3] * P.mu[1] - acc[2] * P.mu[0] - cx(P.mu_f * gram_acc, 0.0);
        blk[0][0] = jj;
        blk[0][1] = jm * P.s_jm;
        blk[1][0] = mj * P.s_jm;
        blk[1][1] = jj * (-P.s_mm);
    } else if (P.formulation == SIEB200_PMCHWT) {
        // acc: TL1, TL2, TK1, TK2
        const cplx tk = acc[2] + acc[3];
        const cplx jm = tk * P.s_jm;
        blk[0][0] = P.c_jj[0] * acc[0] + P.c_jj[1] * acc[1];
        blk[0][1] = jm;
        blk[1][0] = cx(-jm.re, -jm.im);
        blk[1][1] = (P.c_mm[0] * acc[0] + P.c_mm[1] * acc[1]) * P.s_mm;
    } else {
#pragma unroll
        for (int reg = 0; reg < 2; ++reg) {
            const cplx tl = acc[reg], tk = acc[2 + reg];
            const cplx jm = tk * P.s_jm;
            const int o = 2 * reg;
            blk[o][o] = P.c_jj[reg] * tl;
            blk[o][o + 1] = jm;
            blk[o + 1][o] = cx(-jm.re, -jm.im);
            blk[o + 1][o + 1] = P.c_mm[reg] * tl;
        }
        if (has_mass) add_mass_pattern(mass_acc, P.me, P.me2, blk);
    }
    return true;
}

__device__ __forceinline__ int region_count(int formulation) {
    return formulation == SIEB200_PEC_EFIE ? 1 : (formulation == SIEB200_PMCHWT ? 2 : 4);
}

// One thread per (test edge te, source edge se); te fastest for coalesced
// column-major stores. Sums the incident face pairs with the test face in
// [m0, m1) and adds into Z (zeroed before the first slab).
__global__ void gather_kernel(const cplx* __restrict__ pairs, const cplx* __restrict__ mass,
                              const int* __restrict__ inc, GatherParams P, cplx* __restrict__ Z,
                              int64_t ldz) {
    const int te = blockIdx.x * blockDim.x + threadIdx.x;
    const int se = blockIdx.y * blockDim.y + threadIdx.y;
    if (te >= P.ne || se >= P.ne) return;
    cplx blk[4][4];
    if (!edge_pair_block(pairs, mass, inc, P, te, se, blk)) return;
    const int64_t E = P.ne;
    const int nr = region_count(P.formulation);
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (c < nr && r < nr) Z[(te + r * E) + (se + c * E) * ldz] += blk[r][c];
}

// Matrix-free product: y += (the slab's rows of Z) x without storing Z. One
// warp per test edge: lanes stride over the source edges, each forming the
// same region block as gather_kernel, then a warp reduction; the warp owns
// its y entries, and slabs run in order, so the sum is deterministic.
__global__ void gather_matvec_kernel(const cplx* __restrict__ pairs, const cplx* __restrict__ mass,
                                     const int* __restrict__ inc, GatherParams P, const cplx* __restrict__ x,
                                     cplx* __restrict__ y) {
    const int te = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (te >= P.ne) return;  // warp-uniform
    const int64_t E = P.ne;
    const int nr = region_count(P.formulation);
    cplx acc[4] = {cx(0, 0), cx(0, 0), cx(0, 0), cx(0, 0)};
    bool mine = false;
    for (int se = lane; se < P.ne; se += 32) {
        cplx blk[4][4];
        if (!edge_pair_block(pairs, mass, inc, P, te, se, blk)) break;  // same answer for every se
        mine = true;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (c >= nr) break;
            const cplx xv = x[se + c * E];
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[r] += blk[r][c] * xv;  // rows >= nr of blk are zero
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        double re = acc[r].re, im = acc[r].im;
#pragma unroll
        for (int o = 16; o >= 1; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        acc[r] = cx(re, im);
    }
    mine = __any_sync(0xffffffffu, mine);
    if (mine && lane == 0) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
            if (r < nr) y[te + r * E] += acc[r];
    }
}

}  // namespace

int64_t system_dimension(int formulation, int64_t ne) {
    return formulation == SIEB200_PEC_EFIE ? ne : (formulation == SIEB200_PMCHWT ? 2 * ne : 4 * ne);
}

// Mesh, rule and incidences to the device, then the per-face geometry
// records and quadrature points (shared by assembly and the adjoint
// contraction).
static int prepare_faces(sieb200_ctx* ctx, const sieb200_mesh& mesh, const float* pts, const float* wts, int Q,
                         FaceGeom** geom_out, d3** qp_out, float** dw_out, int** dFE_out) {
    const int nf = (int)mesh.num_faces, ne = (int)mesh.num_edges, nv = (int)mesh.num_vertices;
    cudaStream_t st = ctx->stream;
    // Edge -> (face*3 + local edge) incidences; at most two per edge.
    std::vector<int> inc(2 * (size_t)ne, -1);
    for (int f = 0; f < nf; ++f)
        for (int le = 0; le < 3; ++le) {
            const int e = mesh.faces_edges[3 * f + le];
            SIEB_CHECK(e >= 0 && e < ne, SIEB200_INVALID_ARG, "faces_edges entry out of range");
            if (inc[2 * e] < 0) inc[2 * e] = 3 * f + le;
            else if (inc[2 * e + 1] < 0) inc[2 * e + 1] = 3 * f + le;
            else {
                set_error("non-manifold mesh: an edge is shared by more than two faces");
                return SIEB200_INVALID_ARG;
            }
        }

    // Upload mesh, rule, incidences.
    const size_t vbytes = sizeof(double) * 3 * nv, fbytes = sizeof(int) * 3 * nf;
    SIEB_RETURN_IF(ctx->faces.reserve(vbytes + 2 * fbytes + 16 * 3));
    char* fb = ctx->faces.as<char>();
    double* dV = reinterpret_cast<double*>(fb);
    int* dF = reinterpret_cast<int*>(fb + ((vbytes + 15) / 16) * 16);
    int* dFE = dF + 3 * nf + 4;
    SIEB_TRY_CUDA(cudaMemcpyAsync(dV, mesh.vertices, vbytes, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dF, mesh.faces, fbytes, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dFE, mesh.faces_edges, fbytes, cudaMemcpyHostToDevice, st));
    SIEB_RETURN_IF(ctx->qw.reserve(sizeof(float) * (3 * kMaxQ + 2 * kMaxLine)));
    float* dpts = ctx->qw.as<float>();
    float* dw = dpts + 2 * kMaxQ;
    SIEB_TRY_CUDA(cudaMemcpyAsync(dpts, pts, sizeof(float) * 2 * Q, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dw, wts, sizeof(float) * Q, cudaMemcpyHostToDevice, st));
    SIEB_RETURN_IF(ctx->inc.reserve(sizeof(int) * inc.size()));
    SIEB_TRY_CUDA(cudaMemcpyAsync(ctx->inc.ptr, inc.data(), sizeof(int) * inc.size(),
                                  cudaMemcpyHostToDevice, st));

    SIEB_RETURN_IF(ctx->geom.reserve(sizeof(FaceGeom) * nf));
    SIEB_RETURN_IF(ctx->qpts.reserve(sizeof(d3) * (size_t)nf * Q));
    FaceGeom* geom = ctx->geom.as<FaceGeom>();
    d3* qp = ctx->qpts.as<d3>();
    *geom_out = geom;
    *qp_out = qp;
    *dw_out = dw;
    *dFE_out = dFE;
    face_prep_kernel<<<(nf + 127) / 128, 128, 0, st>>>(dV, dF, dFE, nf, dpts, Q, geom, qp);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());

    return SIEB200_OK;
}

// Assembly of Z (dx == nullptr) or, matrix-free, y = Z x with the same face
// pair blocks contracted against x slab by slab instead of written to Z.
static int assemble_or_apply(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                             const double* host_tensors, cplx* dZ, int64_t ldz, const cplx* dx, cplx* dy) {
    AssemblyParams ap;
    SIEB_RETURN_IF(make_assembly_params(opt, &ap));
    const int nf = (int)mesh.num_faces, ne = (int)mesh.num_edges, nv = (int)mesh.num_vertices;
    (void)nv;
    const int64_t N = system_dimension(opt.formulation, ne);
    SIEB_CHECK(dx || ldz >= N, SIEB200_INVALID_ARG, "leading dimension of Z is smaller than N");
    float pts[2 * kMaxQ], wts[kMaxQ];
    const int Q = expand_rule(opt.quadrature_rule, pts, wts);
    SIEB_CHECK(Q > 0 && Q <= kMaxQ, SIEB200_INVALID_ARG, "Dunavant quadrature rule must be in [1, 20]");
    cudaStream_t st = ctx->stream;

    FaceGeom* geom = nullptr;
    d3* qp = nullptr;
    float* dw = nullptr;
    int* dFE = nullptr;
    SIEB_RETURN_IF(prepare_faces(ctx, mesh, pts, wts, Q, &geom, &qp, &dw, &dFE));

    // GSTC mass blocks.
    cplx* dmass = nullptr;
    if (opt.formulation == SIEB200_GSTC) {
        const size_t ntens = opt.tensors_are_uniform ? 32 : (size_t)nf * 32;
        SIEB_RETURN_IF(ctx->tens.reserve(sizeof(cplx) * ntens));
        SIEB_TRY_CUDA(cudaMemcpyAsync(ctx->tens.ptr, host_tensors, sizeof(cplx) * ntens,
                                      cudaMemcpyHostToDevice, st));
        SIEB_RETURN_IF(ctx->mass.reserve(sizeof(cplx) * 72 * (size_t)nf));
        dmass = ctx->mass.as<cplx>();
        mass_face_kernel<<<(nf * 8 + 127) / 128, 128, 0, st>>>(
            geom, qp, dw, Q, nf, ctx->tens.as<cplx>(), opt.tensors_are_uniform, ap.basis, dmass);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
    }

    // RWG Gram blocks for the jump terms of N-MFIE and N-Muller.
    const int variant = ap.variant;
    double* dgram = nullptr;
    if (variant == 2) {
        SIEB_RETURN_IF(ctx->mass.reserve(sizeof(double) * 9 * (size_t)nf));
        dgram = ctx->mass.as<double>();
        gram_face_kernel<<<(nf + 127) / 128, 128, 0, st>>>(geom, qp, dw, Q, nf, dgram);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
    }

    // Slabs of test faces bounded by the pair-block workspace. Blocks per
    // pair: TL (or nTL) per wavenumber, then TK (or nTK) where the
    // formulation uses it (all but T-EFIE and N-EFIE).
    const bool tk = !(opt.formulation == SIEB200_PEC_EFIE && variant != 2);
    const int NK = ap.nk;
    const int NB = tk ? 2 * NK : NK;
    const int exact = (opt.formulation == SIEB200_PEC_EFIE && variant != 0) ? 1 : 0;
    // Line form A of nTL (N-EFIE, N-PMCHWT, N-Muller): Gauss-Legendre rule on
    // [0, 1] after the Dunavant rule in the rule buffer.
    const int NG = ap.line_points;
    const bool form_a = NG > 0;
    float* dgl = ctx->qw.as<float>() + 3 * kMaxQ;
    if (form_a) {
        float glt[2 * kMaxLine];
        SIEB_CHECK(NG <= kMaxLine && gauss_legendre_rule_f(NG, glt, glt + kMaxLine) == NG, SIEB200_INVALID_ARG,
                   "Gauss-Legendre point count must be in [1, 20]");
        SIEB_TRY_CUDA(cudaMemcpyAsync(dgl, glt, sizeof(glt), cudaMemcpyHostToDevice, st));
    }
    const size_t pair_bytes = sizeof(cplx) * 9 * NB;
    size_t budget = (size_t)8 << 30;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget = std::min(budget, free_b / 3);
    int slab = (int)std::max<size_t>(1, std::min<size_t>(nf, budget / (pair_bytes * nf)));
    SIEB_RETURN_IF(ctx->pairs.reserve(pair_bytes * (size_t)slab * nf));
    cplx* pairs = ctx->pairs.as<cplx>();
    SIEB_RETURN_IF(ctx->counter.reserve(sizeof(unsigned long long)));
    unsigned long long* counter = ctx->counter.as<unsigned long long>();

    if (dx)
        SIEB_TRY_CUDA(cudaMemsetAsync(dy, 0, sizeof(cplx) * N, st));
    else
        SIEB_TRY_CUDA(cudaMemset2DAsync(dZ, sizeof(cplx) * ldz, 0, sizeof(cplx) * N, N, st));

    GatherParams gp;
    gp.formulation = opt.formulation;
    gp.nf = nf;
    gp.ne = ne;
    gp.NB = NB;
    gp.c_jj[0] = ap.c_jj[0]; gp.c_jj[1] = ap.c_jj[1];
    gp.c_mm[0] = ap.c_mm[0]; gp.c_mm[1] = ap.c_mm[1];
    gp.s_jm = ap.s_jm; gp.s_mm = ap.s_mm;
    gp.me = ap.mass_eta0; gp.me2 = ap.mass_eta0_sq;
    gp.variant = variant;
    for (int r = 0; r < 2; ++r) { gp.w_em[r] = ap.w_em[r]; gp.eps[r] = ap.eps[r]; gp.mu[r] = ap.mu[r]; }
    gp.eps_f = ap.eps_f; gp.mu_f = ap.mu_f;
    gp.gram = dgram;

    // SIEB200_ASM_SPLIT=1: the two-wavenumber regular pass as one CTA per
    // (face, wavenumber), two CTAs per SM. It raises the FP64 pipe's busy
    // share (51 % against 47 %) but issues 37 % more instructions (the pair
    // geometry twice), so the default is one CTA per face over both.
    const char* split_env = getenv("SIEB200_ASM_SPLIT");
    const bool split_wavenumbers = split_env && split_env[0] == '1';
    // Test point per lane (pair_regular_pq_kernel) where its lanes stay busy
    // (>= 75 % of their iterations); SIEB200_ASM_PER_POINT=0 keeps the flat
    // point-pair kernel everywhere.
    const char* pp_env = getenv("SIEB200_ASM_PER_POINT");
    const bool per_point = !(pp_env && pp_env[0] == '0') && pq_lane_use(Q) >= 0.75;
    for (int m0 = 0; m0 < nf; m0 += slab) {
        const int m1 = std::min(nf, m0 + slab);
        const int rows = m1 - m0;
        if (variant != 0 && opt.formulation == SIEB200_PEC_EFIE && !tk && form_a)
            pair_regular_n_kernel<1, false, true><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[1], ap.k[1], ap.threshold, exact, pairs);
        else if (variant != 0 && opt.formulation == SIEB200_PEC_EFIE && !tk)
            pair_regular_n_kernel<1, false, false><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[1], ap.k[1], ap.threshold, exact, pairs);
        else if (variant != 0 && opt.formulation == SIEB200_PEC_EFIE)
            pair_regular_n_kernel<1, true, false><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[1], ap.k[1], ap.threshold, exact, pairs);
        else if (variant != 0 && form_a)
            pair_regular_n_kernel<2, true, true><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[0], ap.k[1], ap.threshold, exact, pairs);
        else if (variant != 0)
            pair_regular_n_kernel<2, true, false><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[0], ap.k[1], ap.threshold, exact, pairs);
        else if (opt.formulation == SIEB200_PEC_EFIE && per_point)
            pair_regular_pq_kernel<1, false><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[1], ap.k[1], ap.threshold, pairs);
        else if (opt.formulation == SIEB200_PEC_EFIE)
            pair_regular_kernel<1, false><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[1], ap.k[1], ap.threshold, pairs);
        else if (split_wavenumbers)
            pair_regular_kernel<2, true, true><<<dim3(rows, 2), kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[0], ap.k[1], ap.threshold, pairs);
        else if (per_point)
            pair_regular_pq_kernel<2, true><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[0], ap.k[1], ap.threshold, pairs);
        else
            pair_regular_kernel<2, true><<<rows, kWarps * 32, 0, st>>>(
                geom, qp, dw, Q, nf, m0, ap.k[0], ap.k[1], ap.threshold, pairs);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        if (form_a) {
            if (NK == 1)
                pair_line_kernel<1><<<rows, kWarps * 32, 0, st>>>(geom, qp, dw, Q, nf, m0, ap.k[1], ap.k[1],
                                                                  ap.threshold, exact, dgl, dgl + kMaxLine, NG,
                                                                  NB, pairs);
            else
                pair_line_kernel<2><<<rows, kWarps * 32, 0, st>>>(geom, qp, dw, Q, nf, m0, ap.k[0], ap.k[1],
                                                                  ap.threshold, exact, dgl, dgl + kMaxLine, NG,
                                                                  NB, pairs);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
        }

        // Near-pair list of this slab: count, size, fill.
        const long long span = (long long)rows * nf;
        const int nb = (int)((span + 255) / 256);
        SIEB_TRY_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
        near_pairs_kernel<<<nb, 256, 0, st>>>(geom, nf, ap.threshold, exact, m0, m1, counter, nullptr, 0);
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        unsigned long long count = 0;
        SIEB_TRY_CUDA(cudaMemcpyAsync(&count, counter, sizeof(count), cudaMemcpyDeviceToHost, st));
        SIEB_TRY_CUDA(cudaStreamSynchronize(st));
        if (count > 0) {
            SIEB_RETURN_IF(ctx->near_list.reserve(sizeof(int2) * count));
            SIEB_TRY_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
            near_pairs_kernel<<<nb, 256, 0, st>>>(geom, nf, ap.threshold, exact, m0, m1, counter,
                                                  ctx->near_list.as<int2>(), count);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
            const int threads = 128;
            const int blocks = (int)((count * 32 + threads - 1) / threads);
            if (variant != 0 && opt.formulation == SIEB200_PEC_EFIE && form_a)
                pair_singular_n_kernel<1, true><<<blocks, threads, 0, st>>>(
                    geom, qp, dw, Q, nf, m0, ctx->near_list.as<int2>(), (int)count, ap.k[1],
                    ap.k[1], tk, dgl, dgl + kMaxLine, NG, pairs);
            else if (variant != 0 && opt.formulation == SIEB200_PEC_EFIE)
                pair_singular_n_kernel<1, false><<<blocks, threads, 0, st>>>(
                    geom, qp, dw, Q, nf, m0, ctx->near_list.as<int2>(), (int)count, ap.k[1],
                    ap.k[1], tk, dgl, dgl + kMaxLine, 0, pairs);
            else if (variant != 0 && form_a)
                pair_singular_n_kernel<2, true><<<blocks, threads, 0, st>>>(
                    geom, qp, dw, Q, nf, m0, ctx->near_list.as<int2>(), (int)count, ap.k[0],
                    ap.k[1], true, dgl, dgl + kMaxLine, NG, pairs);
            else if (variant != 0)
                pair_singular_n_kernel<2, false><<<blocks, threads, 0, st>>>(
                    geom, qp, dw, Q, nf, m0, ctx->near_list.as<int2>(), (int)count, ap.k[0],
                    ap.k[1], true, dgl, dgl + kMaxLine, 0, pairs);
            else if (opt.formulation == SIEB200_PEC_EFIE)
                pair_singular_kernel<1><<<blocks, threads, 0, st>>>(
                    geom, qp, dw, Q, nf, m0, ctx->near_list.as<int2>(), (int)count, ap.k[1],
                    ap.k[1], false, pairs);
            else
                pair_singular_kernel<2><<<blocks, threads, 0, st>>>(
                    geom, qp, dw, Q, nf, m0, ctx->near_list.as<int2>(), (int)count, ap.k[0],
                    ap.k[1], true, pairs);
            SIEB_NOTE_LAUNCH();
            SIEB_TRY_CUDA(cudaGetLastError());
        }
        gp.m0 = m0;
        gp.m1 = m1;
        if (dx) {
            gather_matvec_kernel<<<(ne + 7) / 8, 256, 0, st>>>(pairs, dmass, ctx->inc.as<int>(), gp, dx, dy);
        } else {
            const dim3 gb(32, 8), gg((ne + 31) / 32, (ne + 7) / 8);
            gather_kernel<<<gg, gb, 0, st>>>(pairs, dmass, ctx->inc.as<int>(), gp, dZ, ldz);
        }
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
    }
    return SIEB200_OK;
}

int assemble_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                    const double* host_tensors, cplx* dZ, int64_t ldz) {
    return assemble_or_apply(ctx, mesh, opt, host_tensors, dZ, ldz, nullptr, nullptr);
}

int matvec_free_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                       const double* host_tensors, const cplx* dx, cplx* dy) {
    return assemble_or_apply(ctx, mesh, opt, host_tensors, nullptr, 0, dx, dy);
}

int tensor_gradient_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                           const cplx* d_lam, const cplx* d_x, cplx* d_s) {
    SIEB_CHECK(opt.formulation == SIEB200_GSTC, SIEB200_INVALID_ARG,
               "the tensor gradient exists for the GSTC formulation only");
    AssemblyParams ap;
    SIEB_RETURN_IF(make_assembly_params(opt, &ap));
    const int nf = (int)mesh.num_faces, ne = (int)mesh.num_edges;
    float pts[2 * kMaxQ], wts[kMaxQ];
    const int Q = expand_rule(opt.quadrature_rule, pts, wts);
    SIEB_CHECK(Q > 0 && Q <= kMaxQ, SIEB200_INVALID_ARG, "Dunavant quadrature rule must be in [1, 20]");
    FaceGeom* geom = nullptr;
    d3* qp = nullptr;
    float* dw = nullptr;
    int* dFE = nullptr;
    SIEB_RETURN_IF(prepare_faces(ctx, mesh, pts, wts, Q, &geom, &qp, &dw, &dFE));
    tensor_grad_kernel<<<(nf * 8 + 127) / 128, 128, 0, ctx->stream>>>(geom, qp, dw, Q, nf, ne, dFE, ap.basis,
                                                                       ap.mass_eta0, ap.mass_eta0_sq, d_lam, d_x,
                                                                       d_s);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

// ------------------------------------------------ surface-integral fields
// The positive surface-integral terms at observation points,
//   Q_E = j w mu L[J] + K[M],   Q_H = -K[J] + j w eps L[M]
// (surface_current_fields.hpp:12-44, kernel sie_kernels_utils.cuh:21-140).

// G and grad G of the field evaluation (green_functions_utils.cuh:142-221):
// standard, or with the static and k^2/2 terms extracted.
__device__ __forceinline__ void field_green(d3 r1, d3 r2, double k, bool regular, cplx& G, cplx g[3]) {
    const d3 Rv = r1 - r2;
    const double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
    if (!regular) {
        if (R < 1e-12) {
            G = cx(0.0, 0.0);
            g[0] = g[1] = g[2] = cx(0.0, 0.0);
            return;
        }
        const double inv_R = 1.0 / R;
        const double i4pR = 1.0 / (4.0 * kPi * R);
        double s, c;
        sincos(k * R, &s, &c);
        G = cx(c * i4pR, -s * i4pR);
        const cplx wg = cx(inv_R, k) * G;
        g[0] = wg * (Rv.x * inv_R);
        g[1] = wg * (Rv.y * inv_R);
        g[2] = wg * (Rv.z * inv_R);
    } else {
        if (R < 1e-6) {
            G = cx(0.0, -k / (4.0 * kPi));
            g[0] = g[1] = g[2] = cx(0.0, 0.0);
            return;
        }
        const double i4p = 1.0 / (4.0 * kPi);
        const double inv_R = 1.0 / R, inv_R2 = inv_R * inv_R, inv_R3 = inv_R2 * inv_R;
        double s, c;
        sincos(k * R, &s, &c);
        G = cx((c - 1.0) * (i4p * inv_R), -s * (i4p * inv_R));
        cplx Kr = cx(inv_R3, k * inv_R2) * cx(c, -s);
        Kr.re += -(inv_R3 + k * k * 0.5 * inv_R);
        const cplx sc = Kr * i4p;
        g[0] = sc * Rv.x;
        g[1] = sc * Rv.y;
        g[2] = sc * Rv.z;
    }
}

struct FieldConsts {
    cplx cJ, cM, cJh, cMh;   // j w mu, 1, -1, j w eps
    float k;                 // the wavenumber as the quadrature helpers receive it
    float k_sq_inv;          // 1 / k^2 in float
    float threshold;         // 0.1 lambda in float
};

// One CTA of 256 threads per observation point; threads take faces
// f = t, t + 256, ...; per face the three half-RWG integrals
// (dunavant_quadrature.cuh:1634-1705, plus the Wilton part of :1719-1770
// when the face centroid is within 0.1 lambda), folded into E and H; a warp
// butterfly and one pass over the warps in a fixed order sum them.
__global__ void __launch_bounds__(256) surface_fields_kernel(const FaceGeom* __restrict__ geom,
                                                            const d3* __restrict__ qp,
                                                            const float* __restrict__ qw, int Q, int nf,
                                                            const d3* __restrict__ obs,
                                                            const cplx* __restrict__ J,
                                                            const cplx* __restrict__ M, FieldConsts fc,
                                                            cplx* __restrict__ E, cplx* __restrict__ H) {
    const d3 r = obs[blockIdx.x];
    const double kd = (double)fc.k;
    cplx e[3] = {cx(0, 0), cx(0, 0), cx(0, 0)}, h[3] = {cx(0, 0), cx(0, 0), cx(0, 0)};
    for (int f = threadIdx.x; f < nf; f += blockDim.x) {
        const FaceGeom g = geom[f];
        // float distance from the centroid, formed without contraction
        const double dx = __dsub_rn(r.x, g.c.x), dy = __dsub_rn(r.y, g.c.y), dz = __dsub_rn(r.z, g.c.z);
        const float dist = (float)__dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                                                       __dmul_rn(dz, dz)));
        const bool near = dist < fc.threshold;
        cplx L[3][3], K[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) { L[i][c] = cx(0, 0); K[i][c] = cx(0, 0); }
        for (int q = 0; q < Q; ++q) {
            const d3 rq = qp[(size_t)f * Q + q];
            const double w = (double)qw[q];
            cplx G, gg[3];
            field_green(r, rq, kd, near, G, gg);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const d3 rho = rq - g.fv[i];
                const double rc[3] = {rho.x, rho.y, rho.z};
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    L[i][c] += ((G * rc[c]) * 0.5 + gg[c] * (double)(-fc.k_sq_inv)) * w;
                const cplx cr[3] = {gg[2] * rho.y - gg[1] * rho.z, gg[0] * rho.z - gg[2] * rho.x,
                                    gg[1] * rho.x - gg[0] * rho.y};
#pragma unroll
                for (int c = 0; c < 3; ++c) K[i][c] += (cr[c] * 0.5) * w;
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const double el = (double)(float)g.len[i];
#pragma unroll
            for (int c = 0; c < 3; ++c) { L[i][c] = L[i][c] * el; K[i][c] = K[i][c] * el; }
        }
        if (near) {
            const float A = (float)g.area;
            const float base = __fdiv_rn(1.0f, __fmul_rn(__fmul_rn(8.0f, (float)kPi), A));
            const Pots P = wilton(r, g.v);
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const d3 fv = g.fv[i];
                const d3 Rf = r - fv;
                const d3 phi3 = P.phi3b + (P.r_pi - fv) * P.phi2;
                const d3 Lin = (psi1(P, fv) - (Rf * 0.5) * P.phi0) + (phi3 - Rf * P.phi2) * (double)fc.k_sq_inv;
                const d3 Kv = upsilon(P, fv, r, fc.k);
                const double ls = (double)__fmul_rn((float)g.len[i], base);
                const d3 Lv = Lin * 2.0;
                L[i][0] += cx(Lv.x * ls, 0.0); L[i][1] += cx(Lv.y * ls, 0.0); L[i][2] += cx(Lv.z * ls, 0.0);
                K[i][0] += cx(Kv.x * ls, 0.0); K[i][1] += cx(Kv.y * ls, 0.0); K[i][2] += cx(Kv.z * ls, 0.0);
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int ed = g.edge[i];
            const cplx je = J[ed], me = M ? M[ed] : cx(0, 0);
            const cplx wEJ = fc.cJ * je, wEM = fc.cM * me, wHJ = fc.cJh * je, wHM = fc.cMh * me;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                e[c] += wEJ * L[i][c];
                e[c] += wEM * K[i][c];
                h[c] += wHJ * K[i][c];
                h[c] += wHM * L[i][c];
            }
        }
    }
    __shared__ double part[8][12];
    double v[12] = {e[0].re, e[0].im, e[1].re, e[1].im, e[2].re, e[2].im,
                    h[0].re, h[0].im, h[1].re, h[1].im, h[2].re, h[2].im};
#pragma unroll
    for (int j = 0; j < 12; ++j) warp_sum(v[j]);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < 12; ++j) part[warp][j] = v[j];
    __syncthreads();
    if (threadIdx.x < 12) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w][threadIdx.x];
        double* out = reinterpret_cast<double*>(threadIdx.x < 6 ? E : H) + 6 * (size_t)blockIdx.x;
        out[threadIdx.x % 6] = t;
    }
}

int surface_fields_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const double* j_cur, const double* m_cur,
                          int64_t nobs, const double* points, double frequency_hz, double eps_r, double mu_r,
                          double eps0, double mu0, int rule, double* E_out, double* H_out) {
    auto fin = [](double x) { return std::isfinite(x); };
    SIEB_CHECK(frequency_hz > 0 && fin(frequency_hz), SIEB200_INVALID_ARG,
               "field-evaluation frequency must be positive and finite");
    SIEB_CHECK(eps_r > 0 && mu_r > 0 && fin(eps_r) && fin(mu_r), SIEB200_INVALID_ARG,
               "field-evaluation relative permittivity and permeability must be positive and finite");
    SIEB_CHECK(eps0 > 0 && mu0 > 0 && fin(eps0) && fin(mu0), SIEB200_INVALID_ARG,
               "field-evaluation vacuum constants must be positive and finite");
    SIEB_CHECK(rule >= 1 && rule <= 20, SIEB200_INVALID_ARG, "Dunavant quadrature rule must be in [1, 20]");
    SIEB_CHECK(nobs >= 0 && nobs < (1ll << 31), SIEB200_INVALID_ARG, "observation point count out of range");
    for (int64_t p = 0; p < nobs; ++p)
        SIEB_CHECK(fin(points[3 * p]) && fin(points[3 * p + 1]) && fin(points[3 * p + 2]), SIEB200_INVALID_ARG,
                   "non-finite observation point at index " + std::to_string(p));
    if (nobs == 0) return SIEB200_OK;
    SIEB_CHECK(mesh.num_vertices > 0 && mesh.num_faces > 0 && mesh.num_edges > 0, SIEB200_INVALID_ARG,
               "field-evaluation mesh must contain vertices, faces, and edges");
    const int nf = (int)mesh.num_faces, ne = (int)mesh.num_edges;
    float pts[2 * kMaxQ], wts[kMaxQ];
    const int Q = expand_rule(rule, pts, wts);
    SIEB_CHECK(Q > 0 && Q <= kMaxQ, SIEB200_INVALID_ARG, "Dunavant quadrature rule must be in [1, 20]");
    cudaStream_t st = ctx->stream;
    FaceGeom* geom = nullptr;
    d3* qp = nullptr;
    float* dw = nullptr;
    int* dFE = nullptr;
    SIEB_RETURN_IF(prepare_faces(ctx, mesh, pts, wts, Q, &geom, &qp, &dw, &dFE));

    // surface_current_fields.cu:96-112 (medium constants) and :255-275 (coefficients).
    const double pi = std::acos(-1.0);
    const double omega = 2.0 * pi * frequency_hz;
    const double eps = eps_r * eps0, mu = mu_r * mu0;
    const double k = omega * std::sqrt(mu * eps);
    FieldConsts fc;
    fc.cJ = cx(0.0, omega * mu);
    fc.cM = cx(1.0, 0.0);
    fc.cJh = cx(-1.0, 0.0);
    fc.cMh = cx(0.0, omega * eps);
    fc.k = (float)k;
    volatile float kf = fc.k;  // float arithmetic as written, no contraction
    fc.k_sq_inv = 1.f / (kf * kf);
    volatile float lambda = (float)((double)(2.0f * (float)M_PI) / k);
    fc.threshold = 0.1f * lambda;

    DeviceBuffer buf;
    const size_t b_obs = sizeof(d3) * (size_t)nobs, b_cur = sizeof(cplx) * (size_t)ne;
    const size_t b_out = sizeof(cplx) * 3 * (size_t)nobs;
    SIEB_RETURN_IF(buf.reserve(b_obs + 2 * b_cur + 2 * b_out));
    char* b = buf.as<char>();
    d3* dobs = reinterpret_cast<d3*>(b);
    cplx* dJ = reinterpret_cast<cplx*>(b + b_obs);
    cplx* dM = m_cur ? dJ + ne : nullptr;
    cplx* dE = reinterpret_cast<cplx*>(b + b_obs + 2 * b_cur);
    cplx* dH = dE + 3 * (size_t)nobs;
    SIEB_TRY_CUDA(cudaMemcpyAsync(dobs, points, b_obs, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dJ, j_cur, b_cur, cudaMemcpyHostToDevice, st));
    if (m_cur) SIEB_TRY_CUDA(cudaMemcpyAsync(dM, m_cur, b_cur, cudaMemcpyHostToDevice, st));
    surface_fields_kernel<<<(unsigned)nobs, 256, 0, st>>>(geom, qp, dw, Q, nf, dobs, dJ, dM, fc, dE, dH);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    SIEB_TRY_CUDA(cudaMemcpyAsync(E_out, dE, b_out, cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(H_out, dH, b_out, cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    return SIEB200_OK;
}

}  // namespace sieb200
