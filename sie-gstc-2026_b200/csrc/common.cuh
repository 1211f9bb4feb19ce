// Shared types and helpers of the sieb200 CUDA library (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/sieb200.h"

namespace sieb200 {

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
struct Status {
    int code;
    std::string msg;
};

#define SIEB_TRY_CUDA(expr)                                                              \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess) {                                                          \
            ::sieb200::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));    \
            return _e == cudaErrorMemoryAllocation ? SIEB200_OUT_OF_MEMORY                \
                                                   : SIEB200_CUDA_ERROR;                  \
        }                                                                                 \
    } while (0)

#define SIEB_CHECK(cond, code, msg)               \
    do {                                          \
        if (!(cond)) {                            \
            ::sieb200::set_error(msg);            \
            return (code);                        \
        }                                         \
    } while (0)

#define SIEB_RETURN_IF(st)          \
    do {                            \
        int _s = (st);              \
        if (_s != SIEB200_OK) return _s; \
    } while (0)

// Process-wide count of kernels this library has launched (host side).
void note_launch();
void note_launches(long long n);  // n launches replayed from a CUDA graph
long long launch_count();
#define SIEB_NOTE_LAUNCH() ::sieb200::note_launch()

// ------------------------------------------------------------------ math
struct cplx {
    double re, im;
};

__host__ __device__ inline cplx cx(double r, double i) { return {r, i}; }
__host__ __device__ inline cplx operator+(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ inline cplx operator-(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
__host__ __device__ inline cplx operator*(cplx a, cplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ inline cplx operator*(cplx a, double s) { return {a.re * s, a.im * s}; }
__host__ __device__ inline cplx& operator+=(cplx& a, cplx b) {
    a.re += b.re;
    a.im += b.im;
    return a;
}

struct d3 {
    double x, y, z;
};
__host__ __device__ inline d3 mk3(double x, double y, double z) { return {x, y, z}; }
__host__ __device__ inline d3 operator+(d3 a, d3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ inline d3 operator-(d3 a, d3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ inline d3 operator*(d3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ inline double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline d3 cross3(d3 a, d3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// ------------------------------------------------------------------ context
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    int reserve(size_t n);  // grows, never shrinks; contents not preserved
    void release();
    template <class T>
    T* as() const { return static_cast<T*>(ptr); }
    ~DeviceBuffer() { release(); }
};

}  // namespace sieb200

namespace sieb200 {
// Event-pair profiler of selected kernels on the context stream.
struct KernelProfile {
    int64_t launches = 0;
    double ms = 0.0, flops = 0.0, bytes = 0.0;
};
struct Profiler {
    bool enabled = false;
    struct Pending {
        int kernel;
        cudaEvent_t a, b;
        double flops, bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;  // events reused across collections
    static constexpr int kKinds = 8;
    KernelProfile k[kKinds];
    // Optional timeline: every span's start and end relative to `base`,
    // recorded on the context stream when the timeline was switched on.
    struct Span {
        int kernel;
        float start_ms, end_ms;
    };
    bool timeline = false;
    cudaEvent_t base = nullptr;
    std::vector<Span> spans;
    // Returns an event pair recorded around a launch (nullptr events when off).
    void begin(cudaStream_t s, int kernel, double flops, double bytes, cudaEvent_t* end_out);
    void end(cudaStream_t s, cudaEvent_t e);
    void collect();  // synchronizes the recorded events and accumulates
};
}  // namespace sieb200

struct sieb200_ctx {
    int device = 0;
    sieb200::Profiler prof;
    cudaStream_t stream = nullptr;
    void* cusolver = nullptr;  // cusolverDnHandle_t, created on first use
    int sm_count = 0;
    // Assembly workspaces (reused across calls).
    sieb200::DeviceBuffer faces, geom, qpts, qw, pairs, near_list, counter, inc, mass, zbuf,
        rhsbuf, srcbuf, tens;
};

namespace sieb200 {

// Physical scalars of one assembly, already rounded the way the reference
// kernels see them (their float kernel arguments).
struct AssemblyParams {
    int formulation = 0;
    int nk = 1;                 // wavenumbers evaluated (1 for PEC, 2 otherwise)
    double k[2] = {0, 0};       // float-valued
    float threshold = 0.f;      // float centroid-distance threshold
    // PEC: Z = c_tl[1] * TL2.
    // PMCHWT: jj = c_jj[0] TL1 + c_jj[1] TL2; jm = s_jm (TK1+TK2); mj = -jm;
    //         mm = s_mm (c_mm[0] TL1 + c_mm[1] TL2).
    // GSTC:  per region r: jj = c_jj[r] TL_r, jm = s_jm TK_r, mj = -jm, mm = c_mm[r] TL_r.
    cplx c_jj[2] = {}, c_mm[2] = {};
    double s_jm = 0, s_mm = 1;
    // GSTC mass-block scales (float eta0 and eta0^2).
    double mass_eta0 = 1, mass_eta0_sq = 1;
    int basis = 0;
    // Testing variant: 0 tangential (T-EFIE, T-PMCHWT, GSTC); 1 rotated
    // n x RWG (N-EFIE, N-PMCHWT; nTL/nTK in the TL/TK slots, same placement);
    // 2 N-MFIE (1/2 Gram - nTK2) or N-Muller (below).
    int variant = 0;
    // N-Muller: w_em[r] = omega eps_r mu_r, eps/mu per region (float-valued),
    // eps_f/mu_f their float means; s_jm = eta0, s_mm = eta0^2 as for PMCHWT.
    double w_em[2] = {0, 0}, eps[2] = {0, 0}, mu[2] = {0, 0};
    double eps_f = 0, mu_f = 0;
    // Gauss-Legendre points of the nTL line form A; 0 for the surface form B.
    int line_points = 0;
};

int make_assembly_params(const sieb200_options& opt, AssemblyParams* out);
int expand_rule(int rule, float* pts, float* w);  // returns Q or -1
int gauss_legendre_rule_f(int n, float* t, float* w);  // returns n or -1

// Assembly on the context stream into a device column-major N x N matrix.
int assemble_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                    const double* host_tensors, cplx* dZ, int64_t ldz);
// y = Z x without storing Z (device vectors of length N), Z as assemble_device builds it.
int matvec_free_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                       const double* host_tensors, const cplx* dx, cplx* dy);
// s[f*32 + k] = lambda^H (dZ / d record[f][k]) x for the GSTC system (device
// vectors of length 4 ne, s: num_faces x 32).
int surface_fields_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const double* j_cur, const double* m_cur,
                          int64_t nobs, const double* points, double frequency_hz, double eps_r, double mu_r,
                          double eps0, double mu0, int rule, double* E_out, double* H_out);
int tensor_gradient_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                           const cplx* d_lam, const cplx* d_x, cplx* d_s);
int assemble_rhs_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const sieb200_options& opt,
                        const sieb200_source* sources, int nsrc, cplx* dB, int64_t ldb);

int64_t system_dimension(int formulation, int64_t num_edges);

}  // namespace sieb200
