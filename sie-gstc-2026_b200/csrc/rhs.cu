// Right-hand sides (tested incident fields) and far-field projection.
//
// RHS reference: include/sie_mom/cuda/dunavant_quadrature.cuh:1543-1611 (RWG
// testing with float edge lengths and weights), source functors
// include/sie_mom/excitation/source_functors.cuh:14-130, placements
// src/sie_mom/solvers/pec_solver.cu:242-264 (PEC),
// src/sie_mom/solvers/dielectric/dielectric_solver.cu:399-530 (T-PMCHWT,
// N-PMCHWT, N-Muller), pec_solver.cu:365-388 (T-EFIE, N-EFIE, N-MFIE) and
// include/sie_mom/cuda/sie_kernels_utils.cuh:184-232 (SIE-GSTC). The rotated
// variants test with rho x n_m (dunavant_quadrature.cuh:1569-1593).
//
// One thread per (face, source) computes the face's three tested values;
// one thread per (edge, source) gathers the <= 2 incident faces and places
// them, so every column is produced without atomics.
//
// Far field: applications/anisotropic_gstc_sphere/plot_far_field.py:88-220.
// One CTA per direction reduces exp(+j k0 r_hat . r_q) c(q) over the F*7
// weighted basis samples.

#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "common.cuh"

namespace sieb200 {

struct DevSource {
    int kind;  // 0 plane wave, 1 dipole
    int region;
    int is_magnetic;
    double a[3], b[3];
    double k, eta;
    // placement: rows get v_E * se and v_H * sh at offsets oe, oh (in units of
    // E; a negative offset places nothing)
    double se, sh;
    int oe, oh;
    int rotated;  // n x RWG testing (dunavant_quadrature.cuh:1569-1593)
};

namespace {

__device__ void source_fields(const DevSource& s, d3 r, cplx E[3], cplx H[3]) {
    if (s.kind == 0) {
        const d3 kh = mk3(s.b[0], s.b[1], s.b[2]);
        const double kdr = dot3(kh, r) * s.k;
        double sn, cs;
        sincos(-kdr, &sn, &cs);
        const cplx ph = cx(cs, sn);
        E[0] = ph * s.a[0];
        E[1] = ph * s.a[1];
        E[2] = ph * s.a[2];
        const double ie = 1.0 / s.eta;
        H[0] = (E[2] * kh.y - E[1] * kh.z) * ie;
        H[1] = (E[0] * kh.z - E[2] * kh.x) * ie;
        H[2] = (E[1] * kh.x - E[0] * kh.y) * ie;
        return;
    }
    const d3 p = mk3(s.a[0], s.a[1], s.a[2]);
    const d3 Rv = r - mk3(s.b[0], s.b[1], s.b[2]);
    const double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
    if (R < 1e-6) {
        for (int c = 0; c < 3; ++c) { E[c] = cx(0, 0); H[c] = cx(0, 0); }
        return;
    }
    const d3 Rh = mk3(Rv.x / R, Rv.y / R, Rv.z / R);
    const double Rdp = Rh.x * p.x + Rh.y * p.y + Rh.z * p.z;
    const d3 Rxp = mk3(Rh.y * p.z - Rh.z * p.y, Rh.z * p.x - Rh.x * p.z, Rh.x * p.y - Rh.y * p.x);
    const d3 tri = mk3(Rxp.y * Rh.z - Rxp.z * Rh.y, Rxp.z * Rh.x - Rxp.x * Rh.z,
                       Rxp.x * Rh.y - Rxp.y * Rh.x);
    double sn, cs;
    sincos(-s.k * R, &sn, &cs);
    const cplx ph = cx(cs, sn);
    const double t1 = (s.k * s.k) / R, t2r = 1.0 / (R * R * R), t2i = s.k / (R * R);
    const double tv[3] = {3.0 * Rh.x * Rdp - p.x, 3.0 * Rh.y * Rdp - p.y, 3.0 * Rh.z * Rdp - p.z};
    const double trc[3] = {tri.x, tri.y, tri.z};
    const double rxp[3] = {Rxp.x, Rxp.y, Rxp.z};
    const cplx hc = cx(-(s.k * s.k) / (s.eta * R), s.k / (s.eta * R * R)) * ph;
    for (int c = 0; c < 3; ++c) {
        const cplx Ec = cx(t1 * trc[c] + tv[c] * t2r, tv[c] * t2i) * ph;
        const cplx Hc = cx(hc.re * -rxp[c], hc.im * -rxp[c]);
        if (s.is_magnetic) {
            E[c] = cx(Hc.re * -s.eta, Hc.im * -s.eta);
            H[c] = cx(Ec.re / s.eta, Ec.im / s.eta);
        } else {
            E[c] = Ec;
            H[c] = Hc;
        }
    }
}

__global__ void rhs_face_kernel(const double* __restrict__ V, const int* __restrict__ F, int nf,
                                const float* __restrict__ qpts, const float* __restrict__ qw,
                                int Q, const DevSource* __restrict__ src, int nsrc,
                                cplx* __restrict__ out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (f >= nf || s >= nsrc) return;
    const DevSource S = src[s];
    int idx[3];
    d3 v[3];
    for (int a = 0; a < 3; ++a) {
        idx[a] = F[3 * f + a];
        v[a] = mk3(V[3 * idx[a]], V[3 * idx[a] + 1], V[3 * idx[a] + 2]);
    }
    const int EA[3] = {0, 1, 2}, EB[3] = {1, 2, 0}, EF[3] = {2, 0, 1};
    float el[3];
    d3 fv[3];
    d3 nm = mk3(0, 0, 0);
    if (S.rotated) {
        const d3 cr = cross3(v[1] - v[0], v[2] - v[0]);
        nm = cr * (1.0 / sqrt(dot3(cr, cr)));
    }
    for (int e = 0; e < 3; ++e) {
        const d3 ev = v[EB[e]] - v[EA[e]];
        const double l = sqrt(ev.x * ev.x + ev.y * ev.y + ev.z * ev.z);
        el[e] = (float)((idx[EA[e]] > idx[EB[e]] ? 1.0 : -1.0) * l);
        fv[e] = v[EF[e]];
    }
    cplx ve[3] = {cx(0, 0), cx(0, 0), cx(0, 0)}, vh[3] = {cx(0, 0), cx(0, 0), cx(0, 0)};
    for (int p = 0; p < Q; ++p) {
        const double wp = (double)qw[p];
        const double xi = (double)qpts[2 * p], eta = (double)qpts[2 * p + 1];
        const double zeta = 1.0 - xi - eta;
        const d3 rp = mk3(v[0].x * zeta + v[1].x * xi + v[2].x * eta,
                          v[0].y * zeta + v[1].y * xi + v[2].y * eta,
                          v[0].z * zeta + v[1].z * xi + v[2].z * eta);
        cplx E[3], H[3];
        source_fields(S, rp, E, H);
        for (int i = 0; i < 3; ++i) {
            const d3 t = S.rotated ? cross3(rp - fv[i], nm) : rp - fv[i];
            const cplx de = cx(t.x * E[0].re + t.y * E[1].re + t.z * E[2].re,
                               t.x * E[0].im + t.y * E[1].im + t.z * E[2].im);
            const cplx dh = cx(t.x * H[0].re + t.y * H[1].re + t.z * H[2].re,
                               t.x * H[0].im + t.y * H[1].im + t.z * H[2].im);
            ve[i] += de * wp;
            vh[i] += dh * wp;
        }
    }
    cplx* o = out + ((size_t)s * nf + f) * 6;
    for (int i = 0; i < 3; ++i) {
        const double sc = (double)__fmul_rn(0.5f, el[i]);
        o[i] = ve[i] * sc;
        o[3 + i] = vh[i] * sc;
    }
}

// Incident E and H of one source at observation points
// (compute_incident_field_kernel, src/sie_mom/excitation/excitation.cu:140-156):
// the same source functors as the right-hand sides, one thread per point.
__global__ void incident_fields_kernel(const double* __restrict__ pts, int64_t n, const DevSource* __restrict__ src,
                                       cplx* __restrict__ E, cplx* __restrict__ H) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const DevSource S = *src;
    cplx e[3], h[3];
    source_fields(S, mk3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), e, h);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        E[3 * i + c] = e[c];
        H[3 * i + c] = h[c];
    }
}

__global__ void rhs_gather_kernel(const cplx* __restrict__ face_vals, const int* __restrict__ inc,
                                  int nf, int ne, const DevSource* __restrict__ src, int nsrc,
                                  int64_t N, cplx* __restrict__ B, int64_t ldb) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int s = blockIdx.y;
    if (e >= ne || s >= nsrc) return;
    const DevSource S = src[s];
    cplx ve = cx(0, 0), vh = cx(0, 0);
    for (int a = 0; a < 2; ++a) {
        const int fi = inc[2 * e + a];
        if (fi < 0) continue;
        const int f = fi / 3, le = fi - 3 * f;
        const cplx* o = face_vals + ((size_t)s * nf + f) * 6;
        ve += o[le];
        vh += o[3 + le];
    }
    cplx* col = B + (int64_t)s * ldb;
    // Column zeroing happens before launch; each (row) is owned by one thread.
    if (S.oe >= 0) col[e + (int64_t)S.oe * ne] = ve * S.se;
    if (S.oh >= 0) col[e + (int64_t)S.oh * ne] = vh * S.sh;
}

// ------------------------------------------------------------ far field --
__global__ void ff_samples_kernel(const double* __restrict__ V, const int* __restrict__ F,
                                  const int* __restrict__ FE, int nf, const cplx* __restrict__ jc,
                                  const cplx* __restrict__ mc, d3* __restrict__ rq,
                                  cplx* __restrict__ cj, cplx* __restrict__ cm) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    // plot_far_field.py:88-115 rule (double): centroid, then two 3-orbits.
    const double s15 = sqrt(15.0);
    const double a1 = (6.0 - s15) / 21.0, w1 = (155.0 - s15) / 1200.0;
    const double a2 = (6.0 + s15) / 21.0, w2 = (155.0 + s15) / 1200.0;
    const double nodes[7][2] = {{1.0 / 3.0, 1.0 / 3.0}, {a1, a1}, {1.0 - 2.0 * a1, a1},
                                {a1, 1.0 - 2.0 * a1}, {a2, a2}, {1.0 - 2.0 * a2, a2},
                                {a2, 1.0 - 2.0 * a2}};
    const double wq[7] = {0.225, w1, w1, w1, w2, w2, w2};
    int idx[3];
    d3 v[3];
    for (int a = 0; a < 3; ++a) {
        idx[a] = F[3 * f + a];
        v[a] = mk3(V[3 * idx[a]], V[3 * idx[a] + 1], V[3 * idx[a] + 2]);
    }
    d3 r[7];
    for (int q = 0; q < 7; ++q) {
        const double xi = nodes[q][0], eta = nodes[q][1], zeta = 1.0 - xi - eta;
        r[q] = v[0] * zeta + v[1] * xi + v[2] * eta;
        rq[f * 7 + q] = r[q];
    }
    const int EA[3] = {0, 1, 2}, EB[3] = {1, 2, 0}, EF[3] = {2, 0, 1};
    cplx accj[7][3], accm[7][3];
    for (int q = 0; q < 7; ++q)
        for (int c = 0; c < 3; ++c) { accj[q][c] = cx(0, 0); accm[q][c] = cx(0, 0); }
    for (int le = 0; le < 3; ++le) {
        const d3 ev = v[EB[le]] - v[EA[le]];
        const double len = (idx[EA[le]] > idx[EB[le]] ? 1.0 : -1.0) * sqrt(dot3(ev, ev));
        const int e = FE[3 * f + le];
        const cplx coj = jc[e] * (0.5 * len);
        const cplx com = mc ? mc[e] * (0.5 * len) : cx(0, 0);
        for (int q = 0; q < 7; ++q) {
            const d3 rho = r[q] - v[EF[le]];
            const double rr[3] = {rho.x, rho.y, rho.z};
            for (int c = 0; c < 3; ++c) {
                accj[q][c] += coj * (wq[q] * rr[c]);
                accm[q][c] += com * (wq[q] * rr[c]);
            }
        }
    }
    for (int q = 0; q < 7; ++q)
        for (int c = 0; c < 3; ++c) {
            cj[(f * 7 + q) * 3 + c] = accj[q][c];
            cm[(f * 7 + q) * 3 + c] = accm[q][c];
        }
}

// Far-field operator as a matrix: rows (F_theta of direction d, then F_phi),
// columns (J of edge e, then M of edge e), row-major with 2*ne columns, so
// that [F_theta; F_phi] = A [J; M] with the same radiation vectors and
// coefficients as ff_samples_kernel / ff_directions_kernel. One thread per
// (direction, edge); the edge's incident faces and the 7-point rule are
// evaluated on the fly.
__global__ void ff_matrix_kernel(const double* __restrict__ V, const int* __restrict__ F,
                                 const int* __restrict__ inc, int ne, int64_t ndir, double k0, double eta0,
                                 const double* __restrict__ rh, const double* __restrict__ th,
                                 const double* __restrict__ ph, cplx* __restrict__ A) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t d = blockIdx.y;
    if (e >= ne) return;
    const double s15 = sqrt(15.0);
    const double a1 = (6.0 - s15) / 21.0, w1 = (155.0 - s15) / 1200.0;
    const double a2 = (6.0 + s15) / 21.0, w2 = (155.0 + s15) / 1200.0;
    const double nodes[7][2] = {{1.0 / 3.0, 1.0 / 3.0}, {a1, a1}, {1.0 - 2.0 * a1, a1},
                                {a1, 1.0 - 2.0 * a1}, {a2, a2}, {1.0 - 2.0 * a2, a2},
                                {a2, 1.0 - 2.0 * a2}};
    const double wq[7] = {0.225, w1, w1, w1, w2, w2, w2};
    const int EA[3] = {0, 1, 2}, EB[3] = {1, 2, 0}, EF[3] = {2, 0, 1};
    const d3 r = mk3(rh[3 * d], rh[3 * d + 1], rh[3 * d + 2]);
    cplx N[3] = {cx(0, 0), cx(0, 0), cx(0, 0)};
    for (int a = 0; a < 2; ++a) {
        const int fi = inc[2 * e + a];
        if (fi < 0) continue;
        const int f = fi / 3, le = fi - 3 * f;
        int idx[3];
        d3 v[3];
        for (int b = 0; b < 3; ++b) {
            idx[b] = F[3 * f + b];
            v[b] = mk3(V[3 * idx[b]], V[3 * idx[b] + 1], V[3 * idx[b] + 2]);
        }
        const d3 ev = v[EB[le]] - v[EA[le]];
        const double len = (idx[EA[le]] > idx[EB[le]] ? 1.0 : -1.0) * sqrt(dot3(ev, ev));
        for (int q = 0; q < 7; ++q) {
            const double xi = nodes[q][0], eta = nodes[q][1], zeta = 1.0 - xi - eta;
            const d3 rq = v[0] * zeta + v[1] * xi + v[2] * eta;
            const d3 rho = rq - v[EF[le]];
            double sn, cs;
            sincos(k0 * dot3(r, rq), &sn, &cs);
            const double wgt = 0.5 * len * wq[q];
            const cplx ph_ = cx(cs * wgt, sn * wgt);
            N[0] += ph_ * rho.x;
            N[1] += ph_ * rho.y;
            N[2] += ph_ * rho.z;
        }
    }
    const double* t = th + 3 * d;
    const double* p = ph + 3 * d;
    const cplx nt = N[0] * t[0] + N[1] * t[1] + N[2] * t[2];
    const cplx np = N[0] * p[0] + N[1] * p[1] + N[2] * p[2];
    const cplx coeff = cx(0.0, -k0 / (4.0 * 3.14159265358979323846));
    const int64_t cols = 2 * (int64_t)ne;
    A[d * cols + e] = coeff * (nt * eta0);
    A[(ndir + d) * cols + e] = coeff * (np * eta0);
    A[d * cols + ne + e] = coeff * np;
    A[(ndir + d) * cols + ne + e] = cx(0, 0) - coeff * nt;
}

__global__ void ff_directions_kernel(const d3* __restrict__ rq, const cplx* __restrict__ cj,
                                     const cplx* __restrict__ cm, int64_t M, double k0, double eta0,
                                     const double* __restrict__ rh, const double* __restrict__ th,
                                     const double* __restrict__ ph, cplx* __restrict__ ft,
                                     cplx* __restrict__ fp, double* __restrict__ U) {
    const int d = blockIdx.x;
    const d3 r = mk3(rh[3 * d], rh[3 * d + 1], rh[3 * d + 2]);
    cplx acc[6];
    for (int c = 0; c < 6; ++c) acc[c] = cx(0, 0);
    for (int64_t i = threadIdx.x; i < M; i += blockDim.x) {
        const double phase = k0 * dot3(r, rq[i]);
        double sn, cs;
        sincos(phase, &sn, &cs);
        const cplx e = cx(cs, sn);
        for (int c = 0; c < 3; ++c) {
            acc[c] += e * cj[i * 3 + c];
            acc[3 + c] += e * cm[i * 3 + c];
        }
    }
    __shared__ cplx red[6][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = 0; c < 6; ++c) {
        double re = acc[c].re, im = acc[c].im;
        for (int o = 16; o > 0; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (lane == 0) red[c][warp] = cx(re, im);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        cplx Nv[3], Lv[3];
        for (int c = 0; c < 3; ++c) {
            Nv[c] = cx(0, 0);
            Lv[c] = cx(0, 0);
            for (int w = 0; w < nw; ++w) {
                Nv[c] += red[c][w];
                Lv[c] += red[3 + c][w];
            }
        }
        const double* t = th + 3 * d;
        const double* p = ph + 3 * d;
        const cplx nt = Nv[0] * t[0] + Nv[1] * t[1] + Nv[2] * t[2];
        const cplx np = Nv[0] * p[0] + Nv[1] * p[1] + Nv[2] * p[2];
        const cplx lt = Lv[0] * t[0] + Lv[1] * t[1] + Lv[2] * t[2];
        const cplx lp = Lv[0] * p[0] + Lv[1] * p[1] + Lv[2] * p[2];
        const cplx coeff = cx(0.0, -k0 / (4.0 * 3.14159265358979323846));
        const cplx a = coeff * (nt * eta0 + lp);
        const cplx b = coeff * (np * eta0 - lt);
        ft[d] = a;
        fp[d] = b;
        U[d] = (a.re * a.re + a.im * a.im + b.re * b.re + b.im * b.im) / (2.0 * eta0);
    }
}

}  // namespace

// Host: physical constants of one source, bound from its region's medium
// (src/sie_mom/excitation/excitation.cu:110-137) and the formulation's
// placement scales.
int prepare_sources(const sieb200_options& opt, const sieb200_source* sources, int nsrc,
                    std::vector<DevSource>* out) {
    const double pi = std::acos(-1.0);
    out->clear();
    for (int s = 0; s < nsrc; ++s) {
        const sieb200_source& in = sources[s];
        DevSource d{};
        SIEB_CHECK(in.kind == 0 || in.kind == 1, SIEB200_INVALID_ARG, "source kind must be 0 (plane wave) or 1 (dipole)");
        SIEB_CHECK(in.region == 1 || in.region == 2, SIEB200_INVALID_ARG, "source region must be interior or exterior");
        const double eps_r = in.region == 1 ? opt.eps_r_interior : opt.eps_r_exterior;
        const double mu_r = in.region == 1 ? opt.mu_r_interior : opt.mu_r_exterior;
        SIEB_CHECK(eps_r > 0 && mu_r > 0, SIEB200_INVALID_ARG, "source relative permittivity and permeability must be positive");
        const double eps = eps_r * opt.vacuum_permittivity, mu = mu_r * opt.vacuum_permeability;
        const double omega = 2.0 * pi * opt.frequency_hz;
        d.k = omega * std::sqrt(mu * eps);
        d.eta = std::sqrt(mu / eps);
        d.kind = in.kind;
        d.region = in.region;
        d.is_magnetic = in.is_magnetic;
        for (int c = 0; c < 3; ++c) { d.a[c] = in.a[c]; d.b[c] = in.b[c]; }
        for (int c = 0; c < 3; ++c)
            SIEB_CHECK(std::isfinite(in.a[c]) && std::isfinite(in.b[c]), SIEB200_INVALID_ARG,
                       "source vectors must be finite");
        if (in.kind == 0) {
            // excitation.cu:45-60: unit direction, transverse amplitude.
            const double dn = std::hypot(in.b[0], in.b[1], in.b[2]);
            const double an = std::hypot(in.a[0], in.a[1], in.a[2]);
            SIEB_CHECK(dn > 0 && std::isfinite(dn), SIEB200_INVALID_ARG, "plane-wave direction magnitude must be positive and finite");
            SIEB_CHECK(an > 0 && std::isfinite(an), SIEB200_INVALID_ARG, "plane-wave amplitude magnitude must be positive and finite");
            for (int c = 0; c < 3; ++c) d.b[c] = in.b[c] / dn;
            const double lf = d.b[0] * in.a[0] / an + d.b[1] * in.a[1] / an + d.b[2] * in.a[2] / an;
            SIEB_CHECK(std::abs(lf) <= 64.0 * 2.220446049250313e-16, SIEB200_INVALID_ARG,
                       "plane-wave electric amplitude must be transverse to propagation");
        } else {
            const double mn = std::hypot(in.a[0], in.a[1], in.a[2]);
            SIEB_CHECK(mn > 0 && std::isfinite(mn), SIEB200_INVALID_ARG, "dipole moment magnitude must be positive and finite");
        }
        d.rotated = opt.variant != SIEB200_VARIANT_T;
        if (opt.formulation == SIEB200_PEC_EFIE) {
            SIEB_CHECK(in.region == 2, SIEB200_INVALID_ARG, "PEC solver requires an exterior (region 2) source");
            if (opt.variant == SIEB200_VARIANT_N_JUMP) {
                // N-MFIE: +<f x n, H_inc> (pec_solver.cu:372-377).
                d.se = 0.0; d.sh = 1.0; d.oe = -1; d.oh = 0;
            } else {
                d.se = 1.0; d.sh = 0.0; d.oe = 0; d.oh = -1;
            }
        } else if (opt.formulation == SIEB200_PMCHWT && opt.variant == SIEB200_VARIANT_N_JUMP) {
            // N-Muller: eps V_E and -mu eta0 V_H of the source region
            // (dielectric_solver.cu:461-489).
            const double eta0 = std::sqrt(opt.vacuum_permeability / opt.vacuum_permittivity);
            d.se = eps_r * opt.vacuum_permittivity;
            d.sh = -(mu_r * opt.vacuum_permeability) * eta0;
            d.oe = 0; d.oh = 1;
        } else if (opt.formulation == SIEB200_PMCHWT) {
            const double eta0 = std::sqrt(opt.vacuum_permeability / opt.vacuum_permittivity);
            const double sign = in.region == 2 ? 1.0 : -1.0;
            d.se = sign; d.sh = sign * eta0; d.oe = 0; d.oh = 1;
        } else {
            const float mu0f = (float)opt.vacuum_permeability, eps0f = (float)opt.vacuum_permittivity;
            const double eta0 = std::sqrt((double)mu0f / (double)eps0f);
            d.se = 1.0; d.sh = eta0;
            d.oe = in.region == 1 ? 0 : 2;
            d.oh = d.oe + 1;
        }
        out->push_back(d);
    }
    return SIEB200_OK;
}

int assemble_rhs_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                        const sieb200_source* sources, int nsrc, cplx* dB, int64_t ldb) {
    std::vector<DevSource> ds;
    SIEB_RETURN_IF(prepare_sources(opt, sources, nsrc, &ds));
    const int nf = (int)mesh.num_faces, ne = (int)mesh.num_edges, nv = (int)mesh.num_vertices;
    const int64_t N = system_dimension(opt.formulation, ne);
    float pts[160], wts[80];
    const int Q = expand_rule(opt.quadrature_rule, pts, wts);
    SIEB_CHECK(Q > 0, SIEB200_INVALID_ARG, "Dunavant quadrature rule must be in [1, 20]");
    cudaStream_t st = ctx->stream;
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
    const size_t vbytes = sizeof(double) * 3 * nv, fbytes = sizeof(int) * 3 * nf;
    const size_t ibytes = sizeof(int) * inc.size();
    const size_t sbytes = sizeof(DevSource) * nsrc;
    const size_t off_f = ((vbytes + 255) / 256) * 256;
    const size_t off_i = off_f + ((fbytes + 255) / 256) * 256;
    const size_t off_s = off_i + ((ibytes + 255) / 256) * 256;
    const size_t off_q = off_s + ((sbytes + 255) / 256) * 256;
    SIEB_RETURN_IF(ctx->srcbuf.reserve(off_q + sizeof(float) * 240));
    char* base = ctx->srcbuf.as<char>();
    double* dV = reinterpret_cast<double*>(base);
    int* dF = reinterpret_cast<int*>(base + off_f);
    int* dinc = reinterpret_cast<int*>(base + off_i);
    DevSource* dsrc = reinterpret_cast<DevSource*>(base + off_s);
    float* dq = reinterpret_cast<float*>(base + off_q);
    SIEB_TRY_CUDA(cudaMemcpyAsync(dV, mesh.vertices, vbytes, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dF, mesh.faces, fbytes, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dinc, inc.data(), ibytes, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dsrc, ds.data(), sbytes, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dq, pts, sizeof(float) * 2 * Q, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dq + 160, wts, sizeof(float) * Q, cudaMemcpyHostToDevice, st));
    SIEB_RETURN_IF(ctx->rhsbuf.reserve(sizeof(cplx) * 6 * (size_t)nf * nsrc));
    SIEB_TRY_CUDA(cudaMemset2DAsync(dB, sizeof(cplx) * ldb, 0, sizeof(cplx) * N, nsrc, st));
    rhs_face_kernel<<<dim3((nf + 127) / 128, nsrc), 128, 0, st>>>(dV, dF, nf, dq, dq + 160, Q, dsrc,
                                                                  nsrc, ctx->rhsbuf.as<cplx>());
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    rhs_gather_kernel<<<dim3((ne + 127) / 128, nsrc), 128, 0, st>>>(
        ctx->rhsbuf.as<cplx>(), dinc, nf, ne, dsrc, nsrc, N, dB, ldb);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

// evaluate_incident_fields (src/sie_mom/excitation/excitation.cu:158-210):
// host points in, host E and H (3 complex per point) out; the source's k and
// eta are bound from its region's medium as for the right-hand sides.
int incident_fields_device(sieb200_ctx* ctx, const sieb200_options& opt, const sieb200_source& source, int64_t n,
                           const double* points, double* E_out, double* H_out) {
    std::vector<DevSource> ds;
    SIEB_RETURN_IF(prepare_sources(opt, &source, 1, &ds));
    for (int64_t i = 0; i < 3 * n; ++i)
        SIEB_CHECK(std::isfinite(points[i]), SIEB200_INVALID_ARG, "incident-field observation point must be finite");
    if (n == 0) return SIEB200_OK;
    cudaStream_t st = ctx->stream;
    const size_t pbytes = sizeof(double) * 3 * (size_t)n, fbytes = sizeof(cplx) * 3 * (size_t)n;
    const size_t off_s = ((pbytes + 255) / 256) * 256;
    const size_t off_e = off_s + 256, off_h = off_e + ((fbytes + 255) / 256) * 256;
    DeviceBuffer buf;
    SIEB_RETURN_IF(buf.reserve(off_h + fbytes));
    char* b = buf.as<char>();
    SIEB_TRY_CUDA(cudaMemcpyAsync(b, points, pbytes, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + off_s, ds.data(), sizeof(DevSource), cudaMemcpyHostToDevice, st));
    incident_fields_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
        reinterpret_cast<const double*>(b), n, reinterpret_cast<const DevSource*>(b + off_s),
        reinterpret_cast<cplx*>(b + off_e), reinterpret_cast<cplx*>(b + off_h));
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    SIEB_TRY_CUDA(cudaMemcpyAsync(E_out, b + off_e, fbytes, cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(H_out, b + off_h, fbytes, cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    return SIEB200_OK;
}

int far_field_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const double* j_cur,
                     const double* m_cur, double k0, double eta0, int64_t ndir, const double* rh,
                     const double* th, const double* ph, double* f_theta, double* f_phi,
                     double* intensity) {
    const int nf = (int)mesh.num_faces, ne = (int)mesh.num_edges, nv = (int)mesh.num_vertices;
    cudaStream_t st = ctx->stream;
    const int64_t M = (int64_t)nf * 7;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += ((bytes + 255) / 256) * 256; return o; };
    const size_t oV = take(sizeof(double) * 3 * nv), oF = take(sizeof(int) * 3 * nf),
                 oFE = take(sizeof(int) * 3 * nf), oJ = take(sizeof(cplx) * ne),
                 oM = take(sizeof(cplx) * ne), oRq = take(sizeof(d3) * M),
                 oCj = take(sizeof(cplx) * 3 * M), oCm = take(sizeof(cplx) * 3 * M),
                 oDir = take(sizeof(double) * 9 * ndir), oOut = take(sizeof(cplx) * 2 * ndir),
                 oU = take(sizeof(double) * ndir);
    DeviceBuffer buf;
    SIEB_RETURN_IF(buf.reserve(off));
    char* b = buf.as<char>();
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oV, mesh.vertices, sizeof(double) * 3 * nv, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oF, mesh.faces, sizeof(int) * 3 * nf, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oFE, mesh.faces_edges, sizeof(int) * 3 * nf, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oJ, j_cur, sizeof(cplx) * ne, cudaMemcpyHostToDevice, st));
    if (m_cur) SIEB_TRY_CUDA(cudaMemcpyAsync(b + oM, m_cur, sizeof(cplx) * ne, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oDir, rh, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oDir + sizeof(double) * 3 * ndir, th, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oDir + sizeof(double) * 6 * ndir, ph, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, st));
    ff_samples_kernel<<<(nf + 127) / 128, 128, 0, st>>>(
        reinterpret_cast<double*>(b + oV), reinterpret_cast<int*>(b + oF),
        reinterpret_cast<int*>(b + oFE), nf, reinterpret_cast<cplx*>(b + oJ),
        m_cur ? reinterpret_cast<cplx*>(b + oM) : nullptr, reinterpret_cast<d3*>(b + oRq),
        reinterpret_cast<cplx*>(b + oCj), reinterpret_cast<cplx*>(b + oCm));
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    if (ndir > 0) {
        double* dd = reinterpret_cast<double*>(b + oDir);
        ff_directions_kernel<<<(unsigned)ndir, 256, 0, st>>>(
            reinterpret_cast<d3*>(b + oRq), reinterpret_cast<cplx*>(b + oCj),
            reinterpret_cast<cplx*>(b + oCm), M, k0, eta0, dd, dd + 3 * ndir, dd + 6 * ndir,
            reinterpret_cast<cplx*>(b + oOut), reinterpret_cast<cplx*>(b + oOut) + ndir,
            reinterpret_cast<double*>(b + oU));
        SIEB_NOTE_LAUNCH();
        SIEB_TRY_CUDA(cudaGetLastError());
        SIEB_TRY_CUDA(cudaMemcpyAsync(f_theta, b + oOut, sizeof(cplx) * ndir, cudaMemcpyDeviceToHost, st));
        SIEB_TRY_CUDA(cudaMemcpyAsync(f_phi, b + oOut + sizeof(cplx) * ndir, sizeof(cplx) * ndir, cudaMemcpyDeviceToHost, st));
        SIEB_TRY_CUDA(cudaMemcpyAsync(intensity, b + oU, sizeof(double) * ndir, cudaMemcpyDeviceToHost, st));
    }
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    return SIEB200_OK;
}

int far_field_matrix_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, double k0, double eta0, int64_t ndir,
                            const double* rh, const double* th, const double* ph, cplx* dA) {
    const int nf = (int)mesh.num_faces, ne = (int)mesh.num_edges, nv = (int)mesh.num_vertices;
    cudaStream_t st = ctx->stream;
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
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += ((bytes + 255) / 256) * 256; return o; };
    const size_t oV = take(sizeof(double) * 3 * nv), oF = take(sizeof(int) * 3 * nf),
                 oI = take(sizeof(int) * 2 * ne), oDir = take(sizeof(double) * 9 * ndir);
    DeviceBuffer buf;
    SIEB_RETURN_IF(buf.reserve(off));
    char* b = buf.as<char>();
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oV, mesh.vertices, sizeof(double) * 3 * nv, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oF, mesh.faces, sizeof(int) * 3 * nf, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(b + oI, inc.data(), sizeof(int) * 2 * ne, cudaMemcpyHostToDevice, st));
    double* dd = reinterpret_cast<double*>(b + oDir);
    SIEB_TRY_CUDA(cudaMemcpyAsync(dd, rh, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dd + 3 * ndir, th, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, st));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dd + 6 * ndir, ph, sizeof(double) * 3 * ndir, cudaMemcpyHostToDevice, st));
    ff_matrix_kernel<<<dim3((unsigned)((ne + 127) / 128), (unsigned)ndir), 128, 0, st>>>(
        reinterpret_cast<double*>(b + oV), reinterpret_cast<int*>(b + oF), reinterpret_cast<int*>(b + oI), ne,
        ndir, k0, eta0, dd, dd + 3 * ndir, dd + 6 * ndir, dA);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    return SIEB200_OK;
}

}  // namespace sieb200
