// Surface-parameter record preparation on the device: the per-face checks
// and inversion of prepare_tensor_records (src/sie_mom/gstc/tensor_io.py:17-132)
// as one kernel, one thread per face, FP64 throughout. The host binding
// (sieb200/records.py) reduces the per-face diagnostics and raises the
// reference's errors in the reference's order.
//
// Per face, with eta the reference impedance and M the physical 4x4 map:
//   balanced B = M with the electric block x eta and the magnetic block / eta;
//   scale = max |B_ij| (at least the smallest normal double);
//   defects relative to scale: reciprocity (B_ee - B_ee^T, B_mm - B_mm^T,
//   B_me + B_em^T), skew-Hermitian (B + B^H), off-diagonal entries;
//   singular values of B by one-sided (Hestenes) Jacobi rotations on its
//   columns, which keeps the small singular values to high relative accuracy
//   (the test s_min <= 4 eps s_max needs them);
//   B^-1 by Gaussian elimination with partial pivoting, the physical inverse
//   (electric block x eta, magnetic / eta), the balanced inverse rebuilt
//   from it as the reference does, and the Frobenius residuals
//   max(|B Bi - I|, |Bi B - I|) and |M M^-1 - I|.
// Outputs: records (M row-major, then M^-1) and 8 doubles of diagnostics.

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>

#include "common.cuh"

namespace sieb200 {

namespace {

struct C {
    double r, i;
};
__host__ __device__ inline C cadd(C a, C b) { return {a.r + b.r, a.i + b.i}; }
__host__ __device__ inline C csub(C a, C b) { return {a.r - b.r, a.i - b.i}; }
__host__ __device__ inline C cmul(C a, C b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__host__ __device__ inline C cconj(C a) { return {a.r, -a.i}; }
__host__ __device__ inline C cscale(C a, double s) { return {a.r * s, a.i * s}; }
__host__ __device__ inline double cabs2(C a) { return a.r * a.r + a.i * a.i; }
__host__ __device__ inline double cabsv(C a) { return hypot(a.r, a.i); }
__host__ __device__ inline C cdiv(C a, C b) {
    // Smith's division
    if (fabs(b.r) >= fabs(b.i)) {
        const double t = b.i / b.r, d = b.r + b.i * t;
        return {(a.r + a.i * t) / d, (a.i - a.r * t) / d};
    }
    const double t = b.r / b.i, d = b.i + b.r * t;
    return {(a.r * t + a.i) / d, (a.i * t - a.r) / d};
}
__host__ __device__ inline bool cfinite(C a) { return isfinite(a.r) && isfinite(a.i); }

}  // namespace

// Diagnostics per face and their flag bits (read by sieb200/records.py).
enum { D_RECIP = 0, D_SKEW, D_OFFDIAG, D_SMAX, D_SMIN, D_RES, D_PRES, D_FLAGS, D_COUNT };
enum { F_BALANCED_NONFINITE = 1, F_SINGULAR_PIVOT = 2, F_INVERSE_NONFINITE = 4, F_BAL_INVERSE_NONFINITE = 8 };

// One face: mp (16 complex, row-major map) -> out (32 complex record) and
// d (D_COUNT diagnostics). Host-callable as well, for checks of the
// arithmetic against numpy.
__host__ __device__ void prepare_record_face(const double* mp, double eta, double* out, double* d) {
    using std::fmax;
    using std::fmin;
    C M[4][4], B[4][4];
    unsigned flags = 0;
    double scale = 0.0;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            M[r][c] = {mp[2 * (4 * r + c)], mp[2 * (4 * r + c) + 1]};
            const double s = (r < 2 && c < 2) ? eta : 1.0;
            B[r][c] = cscale(M[r][c], s);
            if (r >= 2 && c >= 2) B[r][c] = {M[r][c].r / eta, M[r][c].i / eta};
            if (!cfinite(B[r][c])) flags |= F_BALANCED_NONFINITE;
            scale = fmax(scale, cabsv(B[r][c]));
        }
    scale = fmax(scale, DBL_MIN);
    // reciprocity: B_ee - B_ee^T, B_mm - B_mm^T, B_me + B_em^T
    double recip = 0.0, skew = 0.0, offd = 0.0;
    {
        double dee = 0, dmm = 0, dme = 0;
        for (int r = 0; r < 2; ++r)
            for (int c = 0; c < 2; ++c) {
                dee = fmax(dee, cabsv(csub(B[r][c], B[c][r])));
                dmm = fmax(dmm, cabsv(csub(B[2 + r][2 + c], B[2 + c][2 + r])));
                dme = fmax(dme, cabsv(cadd(B[2 + r][c], B[c][2 + r])));
            }
        recip = fmax(dee, fmax(dmm, dme)) / scale;
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) {
                skew = fmax(skew, cabsv(cadd(B[r][c], cconj(B[c][r]))));
                if (r != c) offd = fmax(offd, cabsv(B[r][c]));
            }
        skew /= scale;
        offd /= scale;
    }
    // singular values: one-sided Jacobi on the columns of B
    double smax = 0.0, smin = 0.0;
    {
        C U[4][4];  // U[col][row]
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) U[c][r] = B[r][c];
        for (int sweep = 0; sweep < 40; ++sweep) {
            bool rotated = false;
            for (int p = 0; p < 3; ++p)
                for (int q = p + 1; q < 4; ++q) {
                    double a = 0.0, b = 0.0;
                    C g = {0.0, 0.0};
                    for (int r = 0; r < 4; ++r) {
                        a += cabs2(U[p][r]);
                        b += cabs2(U[q][r]);
                        g = cadd(g, cmul(cconj(U[p][r]), U[q][r]));
                    }
                    const double gn = cabsv(g);
                    if (!(gn > 1e-16 * sqrt(a * b)) || gn == 0.0) continue;
                    rotated = true;
                    // rotate column q by the phase of g so the 2 x 2 Gram is real,
                    // then the real Jacobi rotation that zeroes its off-diagonal
                    const C ph = {g.r / gn, -g.i / gn};  // conj(g) / |g|
                    const double zeta = (b - a) / (2.0 * gn);
                    const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                    const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
                    for (int r = 0; r < 4; ++r) {
                        const C up = U[p][r];
                        const C v = cmul(U[q][r], ph);
                        U[p][r] = csub(cscale(up, cs), cscale(v, sn));
                        U[q][r] = cadd(cscale(up, sn), cscale(v, cs));
                    }
                }
            if (!rotated) break;
        }
        smax = 0.0;
        smin = INFINITY;
        for (int c = 0; c < 4; ++c) {
            double nrm = 0.0;
            for (int r = 0; r < 4; ++r) nrm += cabs2(U[c][r]);
            nrm = sqrt(nrm);
            smax = fmax(smax, nrm);
            smin = fmin(smin, nrm);
        }
    }
    // B^-1 by Gaussian elimination with partial pivoting on [B | I]
    C X[4][4];
    {
        C A[4][8];
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 8; ++c) A[r][c] = c < 4 ? B[r][c] : C{c - 4 == r ? 1.0 : 0.0, 0.0};
        for (int k = 0; k < 4; ++k) {
            int piv = k;
            double best = cabsv(A[k][k]);
            for (int r = k + 1; r < 4; ++r) {
                const double v = cabsv(A[r][k]);
                if (v > best) { best = v; piv = r; }
            }
            if (!(best > 0.0)) {
                flags |= F_SINGULAR_PIVOT;
                best = 1.0;
            }
            if (piv != k)
                for (int c = 0; c < 8; ++c) {
                    const C t = A[k][c];
                    A[k][c] = A[piv][c];
                    A[piv][c] = t;
                }
            for (int r = k + 1; r < 4; ++r) {
                const C l = (flags & F_SINGULAR_PIVOT) ? C{0.0, 0.0} : cdiv(A[r][k], A[k][k]);
                for (int c = k; c < 8; ++c) A[r][c] = csub(A[r][c], cmul(l, A[k][c]));
            }
        }
        for (int c = 0; c < 4; ++c)
            for (int r = 3; r >= 0; --r) {
                C s = A[r][4 + c];
                for (int k = r + 1; k < 4; ++k) s = csub(s, cmul(A[r][k], X[k][c]));
                X[r][c] = (flags & F_SINGULAR_PIVOT) ? C{0.0, 0.0} : cdiv(s, A[r][r]);
            }
    }
    // physical inverse, then the balanced inverse rebuilt from it
    C Inv[4][4], Bi[4][4];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            Inv[r][c] = X[r][c];
            if (r < 2 && c < 2) Inv[r][c] = cscale(X[r][c], eta);
            if (r >= 2 && c >= 2) Inv[r][c] = {X[r][c].r / eta, X[r][c].i / eta};
            if (!cfinite(Inv[r][c])) flags |= F_INVERSE_NONFINITE;
            Bi[r][c] = Inv[r][c];
            if (r < 2 && c < 2) Bi[r][c] = {Inv[r][c].r / eta, Inv[r][c].i / eta};
            if (r >= 2 && c >= 2) Bi[r][c] = cscale(Inv[r][c], eta);
            if (!cfinite(Bi[r][c])) flags |= F_BAL_INVERSE_NONFINITE;
        }
    double r1 = 0.0, r2 = 0.0, rp = 0.0;
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            C s1 = {r == c ? -1.0 : 0.0, 0.0}, s2 = s1, s3 = s1;
            for (int k = 0; k < 4; ++k) {
                s1 = cadd(s1, cmul(B[r][k], Bi[k][c]));
                s2 = cadd(s2, cmul(Bi[r][k], B[k][c]));
                s3 = cadd(s3, cmul(M[r][k], Inv[k][c]));
            }
            r1 += cabs2(s1);
            r2 += cabs2(s2);
            rp += cabs2(s3);
        }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            out[2 * (4 * r + c)] = M[r][c].r;
            out[2 * (4 * r + c) + 1] = M[r][c].i;
            out[32 + 2 * (4 * r + c)] = Inv[r][c].r;
            out[32 + 2 * (4 * r + c) + 1] = Inv[r][c].i;
        }
    d[D_RECIP] = recip;
    d[D_SKEW] = skew;
    d[D_OFFDIAG] = offd;
    d[D_SMAX] = smax;
    d[D_SMIN] = smin;
    d[D_RES] = fmax(sqrt(r1), sqrt(r2));
    d[D_PRES] = sqrt(rp);
    d[D_FLAGS] = (double)flags;
}

namespace {
__global__ void records_kernel(int64_t faces, const double* __restrict__ maps, double eta,
                               double* __restrict__ records, double* __restrict__ diag) {
    const int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= faces) return;
    prepare_record_face(maps + f * 32, eta, records + f * 64, diag + f * D_COUNT);
}
}  // namespace

int prepare_records_device(sieb200_ctx* ctx, int64_t faces, const double* maps, double eta, double* records,
                           double* diag) {
    if (faces == 0) return SIEB200_OK;
    const int threads = 128;
    records_kernel<<<(unsigned)((faces + threads - 1) / threads), threads, 0, ctx->stream>>>(faces, maps, eta,
                                                                                            records, diag);
    SIEB_NOTE_LAUNCH();
    SIEB_TRY_CUDA(cudaGetLastError());
    return SIEB200_OK;
}

}  // namespace sieb200
