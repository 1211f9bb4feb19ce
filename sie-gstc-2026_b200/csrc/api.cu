// C ABI of the sieb200 library: validation, orchestration and the
// reference-compatible physical parameters. Declarations and the reference
// interface each entry point replaces are in include/sieb200.h.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <thread>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "dense.cuh"
#include "gemm_tc.cuh"

namespace sieb200 {

int far_field_matrix_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, double k0, double eta0, int64_t ndir,
                            const double* rh, const double* th, const double* ph, cplx* dA);
int far_field_device(sieb200_ctx* ctx, const sieb200_mesh& mesh, const double* j_cur,
                     const double* m_cur, double k0, double eta0, int64_t ndir, const double* rh,
                     const double* th, const double* ph, double* f_theta, double* f_phi,
                     double* intensity);
int incident_fields_device(sieb200_ctx* ctx, const sieb200_options& opt, const sieb200_source& source, int64_t n,
                           const double* points, double* E_out, double* H_out);
int prepare_records_device(sieb200_ctx* ctx, int64_t faces, const double* maps, double eta, double* records,
                           double* diag);

namespace {
thread_local std::string g_last_error;

struct Orbit {
    int mult;
    double a, b, c, w;
};
struct Rule {
    int n;
    Orbit o[19];
};
// Dunavant (1985) rules 1-20 as orbits; see gen_dunavant_table.py.
const Rule kRules[20] = {
#include "dunavant_table.inc"
};
// Gauss-Legendre rules 1-20 on [0, 1]; see gen_gauss_legendre_table.py.
#include "gauss_legendre_table.inc"

using Clock = std::chrono::steady_clock;
double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void note_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void Profiler::begin(cudaStream_t s, int kernel, double flops, double bytes, cudaEvent_t* end_out) {
    *end_out = nullptr;
    if (!enabled) return;
    Pending p{kernel, nullptr, nullptr, flops, bytes};
    auto take = [&](cudaEvent_t* e) {
        if (!pool.empty()) {
            *e = pool.back();
            pool.pop_back();
            return true;
        }
        return cudaEventCreate(e) == cudaSuccess;
    };
    if (!take(&p.a)) {
        cudaGetLastError();
        return;
    }
    if (!take(&p.b)) {
        pool.push_back(p.a);
        cudaGetLastError();
        return;
    }
    cudaEventRecord(p.a, s);
    pending.push_back(p);
    *end_out = p.b;
}

void Profiler::end(cudaStream_t s, cudaEvent_t e) {
    if (e) cudaEventRecord(e, s);
}

void Profiler::collect() {
    for (Pending& p : pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            KernelProfile& kp = k[p.kernel];
            kp.launches += 1;
            kp.ms += ms;
            kp.flops += p.flops;
            kp.bytes += p.bytes;
            float t0 = 0.f, t1 = 0.f;
            if (timeline && base && cudaEventElapsedTime(&t0, base, p.a) == cudaSuccess &&
                cudaEventElapsedTime(&t1, base, p.b) == cudaSuccess)
                spans.push_back(Span{p.kernel, t0, t1});
        }
        pool.push_back(p.a);
        pool.push_back(p.b);
    }
    pending.clear();
    cudaGetLastError();
}

int DeviceBuffer::reserve(size_t n) {
    if (n <= bytes && ptr) return SIEB200_OK;
    release();
    if (n == 0) n = 16;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) {
        ptr = nullptr;
        bytes = 0;
        cudaGetLastError();
        set_error(std::string("device allocation of ") + std::to_string(n) +
                  " bytes failed: " + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? SIEB200_OUT_OF_MEMORY : SIEB200_CUDA_ERROR;
    }
    bytes = n;
    return SIEB200_OK;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

// Gauss-Legendre rule with n points on [0, 1], nodes ascending, rounded to
// float as the solvers upload it (pec_solver.cu:67-75,
// dielectric/dielectric_solver.cu:179-197). Returns n, or -1.
int gauss_legendre_rule_f(int n, float* t, float* w) {
    if (n < 1 || n > 20) return -1;
    const int off = n * (n - 1) / 2;
    for (int q = 0; q < n; ++q) {
        t[q] = (float)kGaussLegendreNodes[off + q];
        w[q] = (float)kGaussLegendreWeights[off + q];
    }
    return n;
}

// Expansion order of src/sie_mom/quadrature/triangle_dunavant_rule.cpp:135-256
// (orbit by orbit: 1-orbits once; 3-orbits as (a,b),(b,c),(c,a); 6-orbits
// additionally the swapped pairs), rounded to float as
// include/sie_mom/quadrature/triangle_dunavant_rule.hpp:95-100 does.
int expand_rule(int rule, float* pts, float* w) {
    if (rule < 1 || rule > 20) return -1;
    const Rule& r = kRules[rule - 1];
    int o = 0;
    for (int s = 0; s < r.n; ++s) {
        const double t[3] = {r.o[s].a, r.o[s].b, r.o[s].c};
        const int reps = r.o[s].mult == 1 ? 1 : 3;
        for (int k = 0; k < reps; ++k, ++o) {
            pts[2 * o] = (float)t[k];
            pts[2 * o + 1] = (float)t[(k + 1) % 3];
            w[o] = (float)r.o[s].w;
        }
        if (r.o[s].mult == 6)
            for (int k = 0; k < 3; ++k, ++o) {
                pts[2 * o] = (float)t[(k + 1) % 3];
                pts[2 * o + 1] = (float)t[k];
                w[o] = (float)r.o[s].w;
            }
    }
    return o;
}

// Kernel arguments as the reference hands them to its float-parameter
// kernels (src/sie_mom/solvers/pec_solver.cu:338-359,
// dielectric/dielectric_solver.cu:312-321, gstc_sie.cu:281-290, 311-312),
// and the scalar factors the kernels then form from them.
int make_assembly_params(const sieb200_options& o, AssemblyParams* ap) {
    const double pi = std::acos(-1.0);
    const double omega = 2.0 * pi * o.frequency_hz;
    const double e1 = o.eps_r_interior * o.vacuum_permittivity, m1 = o.mu_r_interior * o.vacuum_permeability;
    const double e2 = o.eps_r_exterior * o.vacuum_permittivity, m2 = o.mu_r_exterior * o.vacuum_permeability;
    const double k1 = omega * std::sqrt(m1 * e1), k2 = omega * std::sqrt(m2 * e2);
    const float omf = (float)omega, mu0f = (float)o.vacuum_permeability, eps0f = (float)o.vacuum_permittivity;
    ap->formulation = o.formulation;
    ap->basis = o.basis;
    ap->variant = o.variant;
    // The line form A integrates nTL along the testing edges for N-EFIE,
    // N-PMCHWT and N-Muller; N-MFIE has no nTL (pec_solver.cu:215-218).
    const bool line_integrated = o.formulation == SIEB200_PEC_EFIE ? o.variant == SIEB200_VARIANT_N
                                                                  : o.variant != SIEB200_VARIANT_T;
    ap->line_points = (o.ntl_form == SIEB200_NTL_LINE && line_integrated) ? o.line_quadrature_points : 0;
    if (o.formulation == SIEB200_PEC_EFIE) {
        const double lambda0 = 2.0 * pi / (omega * std::sqrt(o.vacuum_permeability * o.vacuum_permittivity));
        ap->threshold = (float)(o.singularity_threshold_lambda0 * lambda0);
        ap->nk = 1;
        ap->k[0] = ap->k[1] = (double)(float)k2;
        if (o.variant == 1) {
            // N-EFIE: j * (omega * mu2) from the float kernel arguments omega and
            // mu2 = mu_r2 mu0 (pec_solver.cu:163, 346-349).
            const float ce = omf * (float)m2;
            ap->c_jj[1] = cx(0.0, (double)ce);
        } else {
            // c_efie = j * (omega * mu_r2 * mu0) in float (sie_kernels_assembly.cuh:690).
            const float ce = omf * (float)o.mu_r_exterior * mu0f;
            ap->c_jj[1] = cx(0.0, (double)ce);
        }
        return SIEB200_OK;
    }
    ap->nk = 2;
    ap->k[0] = (double)(float)k1;
    ap->k[1] = (double)(float)k2;
    const float mu1f = (float)o.mu_r_interior * mu0f, mu2f = (float)o.mu_r_exterior * mu0f;
    const float ep1f = (float)o.eps_r_interior * eps0f, ep2f = (float)o.eps_r_exterior * eps0f;
    const float eta0f = sqrtf(mu0f / eps0f);
    if (o.formulation == SIEB200_PMCHWT) {
        const double lambda0 = 2.0 * pi / (omega * std::sqrt(o.vacuum_permeability * o.vacuum_permittivity));
        ap->threshold = (float)(o.singularity_threshold_lambda0 * lambda0);
        // dielectric_kernels.cu:104-141.
        ap->c_jj[0] = cx(0.0, (double)omf * (double)mu1f);
        ap->c_jj[1] = cx(0.0, (double)omf * (double)mu2f);
        ap->c_mm[0] = cx(0.0, (double)omf * (double)ep1f);
        ap->c_mm[1] = cx(0.0, (double)omf * (double)ep2f);
        ap->s_jm = (double)eta0f;
        ap->s_mm = (double)(eta0f * eta0f);
        // N-Muller (dielectric_kernels.cu:443-488).
        const float epf[2] = {ep1f, ep2f}, muf[2] = {mu1f, mu2f};
        for (int r = 0; r < 2; ++r) {
            ap->w_em[r] = ((double)omf * (double)epf[r]) * (double)muf[r];
            ap->eps[r] = (double)epf[r];
            ap->mu[r] = (double)muf[r];
        }
        ap->eps_f = (double)((ep1f + ep2f) / 2.0f);
        ap->mu_f = (double)((mu1f + mu2f) / 2.0f);
        return SIEB200_OK;
    }
    // SIE-GSTC (gstc_sie.hpp:73-100; sie_kernels_assembly.cuh:225-231; sie_scaling.cuh:48-61).
    const double c0 = 1.0 / std::sqrt(o.vacuum_permeability * o.vacuum_permittivity);
    ap->threshold = (float)(o.singularity_threshold_lambda0 * c0 / o.frequency_hz);
    const double eta0 = (double)eta0f;  // float sqrt of a float quotient under nvcc
    ap->c_jj[0] = cx(0.0, (double)omf * (double)mu1f);
    ap->c_jj[1] = cx(0.0, (double)omf * (double)mu2f);
    ap->c_mm[0] = cx(0.0, (double)omf * (eta0 * eta0 * (double)ep1f));
    ap->c_mm[1] = cx(0.0, (double)omf * (eta0 * eta0 * (double)ep2f));
    ap->s_jm = eta0;
    ap->s_mm = 1.0;
    ap->mass_eta0 = (double)eta0f;
    ap->mass_eta0_sq = (double)(eta0f * eta0f);
    return SIEB200_OK;
}

int assemble_rhs_device(sieb200_ctx*, const sieb200_mesh&, const sieb200_options&,
                        const sieb200_source*, int, cplx*, int64_t);

namespace {

int validate(const sieb200_mesh* mesh, const sieb200_options* o, const double* tensors,
             bool need_tensors = true) {
    SIEB_CHECK(mesh && o, SIEB200_INVALID_ARG, "mesh and options must not be null");
    SIEB_CHECK(mesh->vertices && mesh->faces && mesh->faces_edges && mesh->num_vertices > 0 &&
                   mesh->num_faces > 0 && mesh->num_edges > 0,
               SIEB200_INVALID_ARG, "SIE mesh must contain vertices, faces, and edges");
    SIEB_CHECK(o->formulation >= 0 && o->formulation <= 2, SIEB200_INVALID_ARG, "unknown formulation");
    SIEB_CHECK(o->frequency_hz > 0 && std::isfinite(o->frequency_hz), SIEB200_INVALID_ARG,
               "SIE frequency must be positive");
    SIEB_CHECK(o->eps_r_interior > 0 && o->mu_r_interior > 0 && o->eps_r_exterior > 0 &&
                   o->mu_r_exterior > 0,
               SIEB200_INVALID_ARG, "relative permittivities and permeabilities must be positive");
    SIEB_CHECK(o->vacuum_permittivity > 0 && o->vacuum_permeability > 0, SIEB200_INVALID_ARG,
               "vacuum permittivity and permeability must be positive");
    SIEB_CHECK(o->quadrature_rule >= 1 && o->quadrature_rule <= 20, SIEB200_INVALID_ARG,
               "Dunavant quadrature rule must be in [1, 20]");
    SIEB_CHECK(o->singularity_threshold_lambda0 > 0, SIEB200_INVALID_ARG,
               "singularity threshold in lambda0 must be positive");
    SIEB_CHECK(o->basis == 0 || o->basis == 1, SIEB200_INVALID_ARG, "unsupported GSTC basis type");
    SIEB_CHECK(o->variant >= SIEB200_VARIANT_T && o->variant <= SIEB200_VARIANT_N_JUMP, SIEB200_INVALID_ARG,
               "unknown formulation variant");
    SIEB_CHECK(o->formulation != SIEB200_GSTC || o->variant == SIEB200_VARIANT_T, SIEB200_INVALID_ARG,
               "the SIE-GSTC formulation has no testing variants");
    SIEB_CHECK(o->ntl_form == SIEB200_NTL_SURFACE || o->ntl_form == SIEB200_NTL_LINE, SIEB200_INVALID_ARG,
               "unknown nTL integral form");
    if (o->ntl_form == SIEB200_NTL_LINE) {
        // pec_solver.cu:91-97 and dielectric_solver.cu:116-125: the line form
        // needs a line-integrated nTL and a 1-20 point Gauss-Legendre rule.
        SIEB_CHECK(o->formulation != SIEB200_PEC_EFIE || o->variant == SIEB200_VARIANT_N, SIEB200_INVALID_ARG,
                   "line nTL form requires N-EFIE");
        SIEB_CHECK(o->formulation != SIEB200_PMCHWT || o->variant != SIEB200_VARIANT_T, SIEB200_INVALID_ARG,
                   "line nTL form requires N-PMCHWT or N-Muller formulation");
        SIEB_CHECK(o->formulation != SIEB200_GSTC, SIEB200_INVALID_ARG,
                   "the SIE-GSTC formulation has no nTL line form");
        SIEB_CHECK(o->line_quadrature_points >= 1 && o->line_quadrature_points <= 20, SIEB200_INVALID_ARG,
                   "Gauss-Legendre point count must be in [1, 20]");
    }
    const int64_t N = system_dimension(o->formulation, mesh->num_edges);
    SIEB_CHECK(N <= std::numeric_limits<int>::max(), SIEB200_OVERFLOW,
               "SIE matrix dimension exceeds the int limit of the dense solvers");
    for (int64_t i = 0; i < 3 * mesh->num_faces; ++i) {
        SIEB_CHECK(mesh->faces[i] >= 0 && mesh->faces[i] < mesh->num_vertices, SIEB200_INVALID_ARG,
                   "face vertex index out of range");
        SIEB_CHECK(mesh->faces_edges[i] >= 0 && mesh->faces_edges[i] < mesh->num_edges,
                   SIEB200_INVALID_ARG, "faces_edges entry out of range");
    }
    for (int64_t i = 0; i < 3 * mesh->num_vertices; ++i)
        SIEB_CHECK(std::isfinite(mesh->vertices[i]), SIEB200_INVALID_ARG, "mesh vertices must be finite");
    if (o->formulation == SIEB200_GSTC && need_tensors) {
        SIEB_CHECK(tensors != nullptr, SIEB200_INVALID_ARG, "GSTC tensor records are required");
        const int64_t count = (o->tensors_are_uniform ? 1 : mesh->num_faces) * 64;
        for (int64_t i = 0; i < count; ++i)
            SIEB_CHECK(std::isfinite(tensors[i]), SIEB200_NONFINITE, "GSTC tensors must be finite");
    }
    return SIEB200_OK;
}

// Physical currents from the scaled solution: M blocks x eta0 (double, from
// the double vacuum constants), finite check, per-block maximum
// (gstc_sie.cu:459-503, dielectric_solver.cu:594-738).
int finish_currents(const sieb200_options& o, int64_t ne, double* x, sieb200_metrics* m) {
    const double eta0 = std::sqrt(o.vacuum_permeability / o.vacuum_permittivity);
    const int blocks = o.formulation == SIEB200_PEC_EFIE ? 1 : (o.formulation == SIEB200_PMCHWT ? 2 : 4);
    for (int b = 0; b < blocks; ++b) {
        const bool magnetic = (b % 2) == 1;
        double mx = 0.0;
        for (int64_t e = 0; e < ne; ++e) {
            double* v = x + 2 * (b * ne + e);
            if (magnetic) { v[0] *= eta0; v[1] *= eta0; }
            if (!std::isfinite(v[0]) || !std::isfinite(v[1])) {
                set_error("non-finite physical current coefficient at index " + std::to_string(b * ne + e));
                return SIEB200_NONFINITE;
            }
            mx = std::max(mx, std::hypot(v[0], v[1]));
        }
        if (m) m->maximum_coefficient[b] = mx;
    }
    return SIEB200_OK;
}

double host_norm(const double* v, int64_t n) {
    long double s = 0.0L;
    for (int64_t i = 0; i < 2 * n; ++i) s += (long double)v[i] * v[i];
    return std::sqrt((double)s);
}

// Shared driver: assemble Z and the columns, factor/solve with the chosen
// method, residual against an intact FP64 Z, physical currents.
int solve_dense_common(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* o,
                       const double* tensors, const sieb200_source* sources, int ncols,
                       const int* col_of_source, int nsrc, double* out, sieb200_metrics* metrics) {
    SIEB_RETURN_IF(validate(mesh, o, tensors));
    SIEB_CHECK(ctx, SIEB200_INVALID_ARG, "context must not be null");
    SIEB_CHECK(ncols > 0, SIEB200_INVALID_ARG, "at least one excitation case is required");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    const int64_t ne = mesh->num_edges;
    const int64_t N = system_dimension(o->formulation, ne);
    const int method = o->solver;
    SIEB_CHECK(method >= 0 && method <= 3, SIEB200_INVALID_ARG, "unsupported solver method");
    cudaStream_t st = ctx->stream;

    DeviceBuffer Zb, Zcopy, Bb, Srcb, Xb, Rb;
    SIEB_RETURN_IF(Zb.reserve(sizeof(cplx) * N * N));
    const auto t_asm = Clock::now();
    SIEB_RETURN_IF(assemble_device(ctx, *mesh, *o, tensors, Zb.as<cplx>(), N));
    SIEB_RETURN_IF(Srcb.reserve(sizeof(cplx) * N * nsrc));
    SIEB_RETURN_IF(assemble_rhs_device(ctx, *mesh, *o, sources, nsrc, Srcb.as<cplx>(), N));
    // Columns: sum of the sources of each case (their rows are disjoint).
    std::vector<double> hsrc(2 * N * nsrc), hb(2 * N * ncols, 0.0);
    SIEB_TRY_CUDA(cudaMemcpyAsync(hsrc.data(), Srcb.ptr, sizeof(cplx) * N * nsrc, cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    const double asm_s = seconds_since(t_asm);
    for (int s = 0; s < nsrc; ++s)
        for (int64_t i = 0; i < 2 * N; ++i) hb[2 * N * col_of_source[s] + i] += hsrc[2 * N * s + i];
    std::vector<double> rhs_norm(ncols);
    for (int c = 0; c < ncols; ++c) {
        rhs_norm[c] = host_norm(hb.data() + 2 * N * c, N);
        if (!(rhs_norm[c] > 0.0) || !std::isfinite(rhs_norm[c])) {
            set_error("case " + std::to_string(c) + ": incident RHS norm must be finite and nonzero");
            return SIEB200_INVALID_ARG;
        }
    }
    SIEB_RETURN_IF(Bb.reserve(sizeof(cplx) * N * ncols));
    SIEB_TRY_CUDA(cudaMemcpyAsync(Bb.ptr, hb.data(), sizeof(cplx) * N * ncols, cudaMemcpyHostToDevice, st));

    const bool in_place = method == SIEB200_SOLVER_LU_CUSOLVER;
    if (o->compute_residual && in_place) {
        SIEB_RETURN_IF(Zcopy.reserve(sizeof(cplx) * N * N));
        SIEB_TRY_CUDA(cudaMemcpyAsync(Zcopy.ptr, Zb.ptr, sizeof(cplx) * N * N, cudaMemcpyDeviceToDevice, st));
    }
    DenseSolver solver;
    solver.ctx = ctx;
    solver.n = N;
    solver.method = method;
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    const auto t_fac = Clock::now();
    int stt = solver.factorize(Zb.as<double>(), N);
    if (stt == SIEB200_OK) SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    const double fac_s = seconds_since(t_fac);
    if (stt != SIEB200_OK) { mixed_release(&solver); return stt; }
    const auto t_sol = Clock::now();
    int iters = 0;
    stt = solver.solve(ncols, Bb.as<double>(), N, false, o->tolerance, o->max_iterations, &iters);
    if (stt == SIEB200_OK) SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    const double sol_s = seconds_since(t_sol);
    if (stt != SIEB200_OK && stt != SIEB200_NOT_CONVERGED) { mixed_release(&solver); return stt; }
    const int solve_status = stt;

    std::vector<double> hx(2 * N * ncols);
    SIEB_TRY_CUDA(cudaMemcpyAsync(hx.data(), Bb.ptr, sizeof(cplx) * N * ncols, cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));

    std::vector<double> abs_res(ncols, 0.0);
    double res_s = 0.0;
    if (o->compute_residual) {
        const auto t_res = Clock::now();
        const double* Zr = in_place ? Zcopy.as<double>() : Zb.as<double>();
        DeviceBuffer scratch;
        std::vector<double> hr(2 * N);
        if (ncols >= 2) {
            // every column at once: R = B - Z X (one FP64 complex GEMM)
            SIEB_RETURN_IF(Rb.reserve(sizeof(cplx) * N * ncols));
            SIEB_TRY_CUDA(cudaMemcpyAsync(Rb.ptr, hb.data(), sizeof(cplx) * N * ncols, cudaMemcpyHostToDevice, st));
            SIEB_RETURN_IF(zgemm_device(st, N, ncols, N, reinterpret_cast<const cplx*>(Zr), N, Bb.as<cplx>(), N,
                                        Rb.as<cplx>(), N, cx(-1, 0), cx(1, 0)));
            std::vector<double> hR(2 * N * ncols);
            SIEB_TRY_CUDA(cudaMemcpyAsync(hR.data(), Rb.ptr, sizeof(cplx) * N * ncols, cudaMemcpyDeviceToHost, st));
            SIEB_TRY_CUDA(cudaStreamSynchronize(st));
            for (int c = 0; c < ncols; ++c) abs_res[c] = host_norm(hR.data() + 2 * N * c, N);
        } else {
        SIEB_RETURN_IF(Rb.reserve(sizeof(cplx) * N * 2));
        for (int c = 0; c < ncols; ++c) {
            cplx* r = Rb.as<cplx>();
            SIEB_TRY_CUDA(cudaMemcpyAsync(r, hb.data() + 2 * N * c, sizeof(cplx) * N, cudaMemcpyHostToDevice, st));
            // r = -b + Z x  (sign irrelevant for the norm)
            SIEB_RETURN_IF(gemv_device(ctx, N, Zr, N, 0, Bb.as<cplx>() + N * c, -1.0, r, scratch));
            SIEB_TRY_CUDA(cudaMemcpyAsync(hr.data(), r, sizeof(cplx) * N, cudaMemcpyDeviceToHost, st));
            SIEB_TRY_CUDA(cudaStreamSynchronize(st));
            abs_res[c] = host_norm(hr.data(), N);
        }
        }
        res_s = seconds_since(t_res);
    }
    mixed_release(&solver);

    for (int c = 0; c < ncols; ++c) {
        sieb200_metrics* m = metrics ? metrics + c : nullptr;
        if (m) {
            std::memset(m, 0, sizeof(*m));
            m->matrix_dimension = N;
            m->dense_matrix_bytes = (int64_t)(sizeof(cplx) * N * N);
            m->assembly_seconds = asm_s;
            m->factorization_seconds = fac_s;
            m->solve_seconds = sol_s;
            m->residual_seconds = res_s;
            m->residual_computed = o->compute_residual ? 1 : 0;
            m->rhs_norm = rhs_norm[c];
            m->absolute_residual = abs_res[c];
            m->relative_residual = o->compute_residual ? abs_res[c] / rhs_norm[c] : 0.0;
            m->refinement_iterations = iters;
            m->solver = method;
        }
        SIEB_RETURN_IF(finish_currents(*o, ne, hx.data() + 2 * N * c, m));
    }
    std::memcpy(out, hx.data(), sizeof(double) * 2 * N * ncols);
    return solve_status;
}

// ------------------------------------------------------------ batched sweep
// Device buffers a sweep lane keeps across its instances (largest first, so
// they are sized once and never freed mid-sweep: cudaFree would stall the
// other lanes' streams).
struct LaneBuffers {
    DeviceBuffer Z, B, Src, R, scratch;
};

// One SIE-GSTC instance on a lane's own context: assembly, factorization
// (trailing GEMM on at most sm_cap SMs), refined solve, FP64 residual,
// physical currents. The same steps as solve_dense_common, without the
// per-call allocations.
int lane_solve(sieb200_ctx* ctx, DenseSolver& solver, LaneBuffers& lb, const sieb200_sweep_instance& in,
               int sm_cap) {
    const sieb200_options* o = &in.opt;
    SIEB_CHECK(o->formulation == SIEB200_GSTC, SIEB200_INVALID_ARG, "sweep instances must be SIE-GSTC systems");
    SIEB_RETURN_IF(validate(&in.mesh, o, in.tensors));
    SIEB_CHECK(in.currents_out, SIEB200_INVALID_ARG, "sweep instance output must not be null");
    std::vector<sieb200_source> src;
    for (int slot = 0; slot < 2; ++slot) {
        if (in.source[slot].kind < 0) continue;
        SIEB_CHECK(in.source[slot].region == slot + 1, SIEB200_INVALID_ARG,
                   "sweep instance excitation does not match its regional slot");
        src.push_back(in.source[slot]);
    }
    SIEB_CHECK(!src.empty(), SIEB200_INVALID_ARG, "sweep instance needs at least one incident region");
    const int64_t ne = in.mesh.num_edges;
    const int64_t N = system_dimension(o->formulation, ne);
    cudaStream_t st = ctx->stream;
    const auto t_asm = Clock::now();
    SIEB_RETURN_IF(lb.Z.reserve(sizeof(cplx) * N * N));
    SIEB_RETURN_IF(assemble_device(ctx, in.mesh, *o, in.tensors, lb.Z.as<cplx>(), N));
    SIEB_RETURN_IF(lb.Src.reserve(sizeof(cplx) * N * src.size()));
    SIEB_RETURN_IF(assemble_rhs_device(ctx, in.mesh, *o, src.data(), (int)src.size(), lb.Src.as<cplx>(), N));
    std::vector<double> hs(2 * N * src.size()), hb(2 * N, 0.0);
    SIEB_TRY_CUDA(cudaMemcpyAsync(hs.data(), lb.Src.ptr, sizeof(cplx) * N * src.size(), cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    const double asm_s = seconds_since(t_asm);
    for (size_t k = 0; k < src.size(); ++k)
        for (int64_t i = 0; i < 2 * N; ++i) hb[i] += hs[2 * N * k + i];
    const double rhs_norm = host_norm(hb.data(), N);
    SIEB_CHECK(rhs_norm > 0.0 && std::isfinite(rhs_norm), SIEB200_INVALID_ARG,
               "incident RHS norm must be finite and nonzero");
    SIEB_RETURN_IF(lb.B.reserve(sizeof(cplx) * N));
    SIEB_TRY_CUDA(cudaMemcpyAsync(lb.B.ptr, hb.data(), sizeof(cplx) * N, cudaMemcpyHostToDevice, st));
    SIEB_CHECK(o->solver == SIEB200_SOLVER_MIXED_IR || o->solver == SIEB200_SOLVER_LU_CUSOLVER ||
                   o->solver == SIEB200_SOLVER_LU_FP64,
               SIEB200_INVALID_ARG, "sweep instances are solved by the mixed, the own FP64 or the cuSOLVER LU");
    const bool in_place = o->solver == SIEB200_SOLVER_LU_CUSOLVER;
    if (in_place && o->compute_residual) {
        SIEB_RETURN_IF(lb.R.reserve(sizeof(cplx) * N * N + sizeof(cplx) * N));
        SIEB_TRY_CUDA(cudaMemcpyAsync(lb.R.ptr, lb.Z.ptr, sizeof(cplx) * N * N, cudaMemcpyDeviceToDevice, st));
    }
    solver.ctx = ctx;
    solver.n = N;
    solver.method = o->solver;
    solver.sm_cap = sm_cap;
    const auto t_fac = Clock::now();
    SIEB_RETURN_IF(solver.factorize(lb.Z.as<double>(), N));
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    const double fac_s = seconds_since(t_fac);
    const auto t_sol = Clock::now();
    int iters = 0;
    const int stt = solver.solve(1, lb.B.as<double>(), N, false, o->tolerance, o->max_iterations, &iters);
    if (stt != SIEB200_OK && stt != SIEB200_NOT_CONVERGED) return stt;
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    const double sol_s = seconds_since(t_sol);
    double abs_res = 0.0, res_s = 0.0;
    if (o->compute_residual) {
        const auto t_res = Clock::now();
        const double* Zr = in_place ? lb.R.as<double>() : lb.Z.as<double>();
        cplx* r = in_place ? lb.R.as<cplx>() + N * N : nullptr;
        if (!in_place) {
            SIEB_RETURN_IF(lb.R.reserve(sizeof(cplx) * N));
            r = lb.R.as<cplx>();
        }
        SIEB_TRY_CUDA(cudaMemcpyAsync(r, hb.data(), sizeof(cplx) * N, cudaMemcpyHostToDevice, st));
        SIEB_RETURN_IF(gemv_device(ctx, N, Zr, N, 0, lb.B.as<cplx>(), -1.0, r, lb.scratch));
        std::vector<double> hr(2 * N);
        SIEB_TRY_CUDA(cudaMemcpyAsync(hr.data(), r, sizeof(cplx) * N, cudaMemcpyDeviceToHost, st));
        SIEB_TRY_CUDA(cudaStreamSynchronize(st));
        abs_res = host_norm(hr.data(), N);
        res_s = seconds_since(t_res);
    }
    SIEB_TRY_CUDA(cudaMemcpyAsync(in.currents_out, lb.B.ptr, sizeof(cplx) * N, cudaMemcpyDeviceToHost, st));
    SIEB_TRY_CUDA(cudaStreamSynchronize(st));
    sieb200_metrics* m = in.metrics;
    if (m) {
        std::memset(m, 0, sizeof(*m));
        m->matrix_dimension = N;
        m->dense_matrix_bytes = (int64_t)(sizeof(cplx) * N * N);
        m->assembly_seconds = asm_s;
        m->factorization_seconds = fac_s;
        m->solve_seconds = sol_s;
        m->residual_seconds = res_s;
        m->residual_computed = o->compute_residual ? 1 : 0;
        m->rhs_norm = rhs_norm;
        m->absolute_residual = abs_res;
        m->relative_residual = o->compute_residual ? abs_res / rhs_norm : 0.0;
        m->refinement_iterations = iters;
        m->solver = o->solver;
    }
    SIEB_RETURN_IF(finish_currents(*o, ne, in.currents_out, m));
    return stt;
}

}  // namespace
}  // namespace sieb200

using namespace sieb200;

extern "C" {

const char* sieb200_last_error(void) { return g_last_error.c_str(); }
int sieb200_version(void) { return SIEB200_ABI_VERSION; }

int sieb200_ctx_create(int device, sieb200_ctx** out) {
    SIEB_CHECK(out, SIEB200_INVALID_ARG, "output pointer must not be null");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        set_error("no CUDA-capable device is available");
        return SIEB200_NO_DEVICE;
    }
    SIEB_CHECK(device >= 0 && device < count, SIEB200_INVALID_ARG, "device index out of range");
    SIEB_TRY_CUDA(cudaSetDevice(device));
    sieb200_ctx* c = new sieb200_ctx();
    c->device = device;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        set_error(std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
        return SIEB200_CUDA_ERROR;
    }
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    *out = c;
    return SIEB200_OK;
}

int sieb200_ctx_destroy(sieb200_ctx* ctx) {
    if (!ctx) return SIEB200_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    destroy_cusolver(ctx);
    ctx->prof.collect();
    for (cudaEvent_t e : ctx->prof.pool) cudaEventDestroy(e);
    if (ctx->prof.base) cudaEventDestroy(ctx->prof.base);
    ctx->prof.pool.clear();
    ctx->faces.release(); ctx->geom.release(); ctx->qpts.release(); ctx->qw.release();
    ctx->pairs.release(); ctx->near_list.release(); ctx->counter.release(); ctx->inc.release();
    ctx->mass.release(); ctx->zbuf.release(); ctx->rhsbuf.release(); ctx->srcbuf.release();
    ctx->tens.release();
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SIEB200_OK;
}

int sieb200_ctx_synchronize(sieb200_ctx* ctx) {
    SIEB_CHECK(ctx, SIEB200_INVALID_ARG, "context must not be null");
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

void* sieb200_ctx_stream(sieb200_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int sieb200_quadrature_rule(int rule, float* pts, float* w) {
    float p[160], ww[80];
    const int n = expand_rule(rule, p, ww);
    if (n < 0) {
        set_error("Dunavant quadrature rule must be in [1, 20]");
        return -1;
    }
    if (pts) std::memcpy(pts, p, sizeof(float) * 2 * n);
    if (w) std::memcpy(w, ww, sizeof(float) * n);
    return n;
}

int sieb200_build_edges(const int32_t* faces, int64_t num_faces, int32_t* edges_out,
                        int32_t* faces_edges_out, int64_t* num_edges_out) {
    SIEB_CHECK(faces && faces_edges_out && num_edges_out && num_faces >= 0, SIEB200_INVALID_ARG,
               "build_edges: null argument");
    std::unordered_map<uint64_t, int32_t> map;
    map.reserve((size_t)num_faces * 2);
    int32_t next = 0;
    for (int64_t f = 0; f < num_faces; ++f)
        for (int le = 0; le < 3; ++le) {
            const int32_t a = faces[3 * f + le], b = faces[3 * f + (le + 1) % 3];
            SIEB_CHECK(a >= 0 && b >= 0, SIEB200_INVALID_ARG, "negative vertex index");
            const uint32_t lo = (uint32_t)std::min(a, b), hi = (uint32_t)std::max(a, b);
            const uint64_t key = ((uint64_t)lo << 32) | hi;
            auto it = map.find(key);
            int32_t id;
            if (it == map.end()) {
                id = next++;
                map.emplace(key, id);
                if (edges_out) { edges_out[2 * id] = (int32_t)lo; edges_out[2 * id + 1] = (int32_t)hi; }
            } else {
                id = it->second;
            }
            faces_edges_out[3 * f + le] = id;
        }
    *num_edges_out = next;
    return SIEB200_OK;
}

int sieb200_options_default(int formulation, sieb200_options* o) {
    SIEB_CHECK(o, SIEB200_INVALID_ARG, "options pointer must not be null");
    SIEB_CHECK(formulation >= 0 && formulation <= 2, SIEB200_INVALID_ARG, "unknown formulation");
    std::memset(o, 0, sizeof(*o));
    o->formulation = formulation;
    o->eps_r_interior = o->mu_r_interior = o->eps_r_exterior = o->mu_r_exterior = 1.0;
    o->singularity_threshold_lambda0 = 0.1;
    o->compute_residual = 1;
    o->tolerance = 1e-10;
    o->max_iterations = 50;
    o->restart = 30;
    o->line_quadrature_points = 20;
    o->solver = SIEB200_SOLVER_LU_CUSOLVER;
    if (formulation == SIEB200_GSTC) {
        o->quadrature_rule = 17;
        o->vacuum_permittivity = 8.8541878188e-12;
        o->vacuum_permeability = 1.25663706127e-6;
        o->basis = SIEB200_BASIS_FACE;
    } else {
        o->quadrature_rule = formulation == SIEB200_PEC_EFIE ? 7 : 17;
        o->vacuum_permittivity = 8.8541878128e-12;
        o->vacuum_permeability = 1.25663706212e-6;
    }
    return SIEB200_OK;
}

int sieb200_solve_pec_dense(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                            const sieb200_source* source, double* current_out, sieb200_metrics* m) {
    SIEB_CHECK(opt && opt->formulation == SIEB200_PEC_EFIE, SIEB200_INVALID_ARG,
               "solve_pec_dense needs formulation SIEB200_PEC_EFIE");
    SIEB_CHECK(source && current_out, SIEB200_INVALID_ARG, "source and output must not be null");
    const int col = 0;
    return solve_dense_common(ctx, mesh, opt, nullptr, source, 1, &col, 1, current_out, m);
}

int sieb200_solve_dielectric_dense(sieb200_ctx* ctx, const sieb200_mesh* mesh,
                                   const sieb200_options* opt, const sieb200_source* source,
                                   double* currents_out, sieb200_metrics* m) {
    SIEB_CHECK(opt && opt->formulation == SIEB200_PMCHWT, SIEB200_INVALID_ARG,
               "solve_dielectric_dense needs formulation SIEB200_PMCHWT");
    SIEB_CHECK(source && currents_out, SIEB200_INVALID_ARG, "source and output must not be null");
    const int col = 0;
    return solve_dense_common(ctx, mesh, opt, nullptr, source, 1, &col, 1, currents_out, m);
}

int sieb200_solve_gstc_dense_batch(sieb200_ctx* ctx, const sieb200_mesh* mesh,
                                   const double* tensors, const sieb200_options* opt,
                                   const sieb200_source* sources, int num_cases,
                                   double* currents_out, sieb200_metrics* m) {
    SIEB_CHECK(opt && opt->formulation == SIEB200_GSTC, SIEB200_INVALID_ARG,
               "solve_gstc_dense_batch needs formulation SIEB200_GSTC");
    SIEB_CHECK(sources && currents_out, SIEB200_INVALID_ARG, "sources and output must not be null");
    SIEB_CHECK(num_cases > 0, SIEB200_INVALID_ARG, "SIE batch must contain at least one excitation case");
    std::vector<sieb200_source> flat;
    std::vector<int> cols;
    for (int c = 0; c < num_cases; ++c) {
        bool any = false;
        for (int slot = 0; slot < 2; ++slot) {
            const sieb200_source& s = sources[2 * c + slot];
            if (s.kind < 0) continue;
            if (s.region != slot + 1) {
                set_error("SIE batch case " + std::to_string(c) + ": excitation does not match its regional slot");
                return SIEB200_INVALID_ARG;
            }
            flat.push_back(s);
            cols.push_back(c);
            any = true;
        }
        if (!any) {
            set_error("SIE batch case " + std::to_string(c) + ": at least one incident region is required");
            return SIEB200_INVALID_ARG;
        }
    }
    return solve_dense_common(ctx, mesh, opt, tensors, flat.data(), num_cases, cols.data(),
                              (int)flat.size(), currents_out, m);
}

int sieb200_solve_gstc_sweep(sieb200_ctx* ctx, const sieb200_sweep_instance* instances, int count,
                             int concurrency, double* seconds_out) {
    SIEB_CHECK(ctx && instances && count > 0, SIEB200_INVALID_ARG, "sweep needs a context and at least one instance");
    SIEB_CHECK(concurrency >= 1, SIEB200_INVALID_ARG, "sweep concurrency must be at least 1");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    // Largest systems first (their cost grows as N^3): each lane takes the
    // next one as it finishes, so the lanes end close together.
    std::vector<int> order(count);
    for (int i = 0; i < count; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return instances[a].mesh.num_edges > instances[b].mesh.num_edges;
    });
    const int lanes = std::min(concurrency, count);
    const int sm_cap = lanes > 1 ? std::max(16, ctx->sm_count / lanes) : 0;
    std::atomic<int> next{0};
    std::atomic<bool> failed{false};
    std::mutex mu;
    int status = SIEB200_OK;
    std::string message;
    const int device = ctx->device;
    auto lane = [&]() {
        sieb200_ctx* lctx = nullptr;
        int rc = sieb200_ctx_create(device, &lctx);
        if (rc == SIEB200_OK) {
            DenseSolver solver;
            LaneBuffers lb;
            for (int k = next.fetch_add(1); k < count && !failed.load(); k = next.fetch_add(1)) {
                rc = lane_solve(lctx, solver, lb, instances[order[k]], sm_cap);
                if (rc != SIEB200_OK && rc != SIEB200_NOT_CONVERGED) {
                    set_error("sweep instance " + std::to_string(order[k]) + ": " + g_last_error);
                    break;
                }
                if (rc == SIEB200_NOT_CONVERGED) {
                    std::lock_guard<std::mutex> lock(mu);
                    if (status == SIEB200_OK) {
                        status = rc;
                        message = "sweep instance " + std::to_string(order[k]) + ": " + g_last_error;
                    }
                    rc = SIEB200_OK;
                }
            }
            mixed_release(&solver);
            lb.Z.release(); lb.B.release(); lb.Src.release(); lb.R.release(); lb.scratch.release();
            sieb200_ctx_destroy(lctx);
        }
        if (rc != SIEB200_OK) {
            failed.store(true);
            std::lock_guard<std::mutex> lock(mu);
            if (status == SIEB200_OK || status == SIEB200_NOT_CONVERGED) {
                status = rc;
                message = g_last_error;
            }
        }
    };
    const auto t0 = Clock::now();
    if (lanes == 1) {
        lane();
    } else {
        std::vector<std::thread> pool;
        for (int l = 0; l < lanes; ++l) pool.emplace_back(lane);
        for (auto& t : pool) t.join();
    }
    if (seconds_out) *seconds_out = seconds_since(t0);
    if (status != SIEB200_OK) set_error(message);
    return status;
}

int sieb200_assemble_matrix(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                            const double* tensors, double* Z, int z_on_device) {
    SIEB_RETURN_IF(validate(mesh, opt, tensors));
    SIEB_CHECK(ctx && Z, SIEB200_INVALID_ARG, "context and output must not be null");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    const int64_t N = system_dimension(opt->formulation, mesh->num_edges);
    if (z_on_device) {
        SIEB_RETURN_IF(assemble_device(ctx, *mesh, *opt, tensors, reinterpret_cast<cplx*>(Z), N));
        SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
        return SIEB200_OK;
    }
    SIEB_RETURN_IF(ctx->zbuf.reserve(sizeof(cplx) * N * N));
    SIEB_RETURN_IF(assemble_device(ctx, *mesh, *opt, tensors, ctx->zbuf.as<cplx>(), N));
    SIEB_TRY_CUDA(cudaMemcpyAsync(Z, ctx->zbuf.ptr, sizeof(cplx) * N * N, cudaMemcpyDeviceToHost, ctx->stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int sieb200_matvec_matrix_free(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                               const double* tensors, const double* x, double* y, int on_device) {
    SIEB_RETURN_IF(validate(mesh, opt, tensors));
    SIEB_CHECK(ctx && x && y, SIEB200_INVALID_ARG, "invalid matrix-free product arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    const int64_t N = system_dimension(opt->formulation, mesh->num_edges);
    if (on_device) {
        SIEB_RETURN_IF(matvec_free_device(ctx, *mesh, *opt, tensors, reinterpret_cast<const cplx*>(x),
                                          reinterpret_cast<cplx*>(y)));
        SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
        return SIEB200_OK;
    }
    DeviceBuffer tmp;
    SIEB_RETURN_IF(tmp.reserve(sizeof(cplx) * 2 * N));
    cplx* dx = tmp.as<cplx>();
    cplx* dy = dx + N;
    SIEB_TRY_CUDA(cudaMemcpyAsync(dx, x, sizeof(cplx) * N, cudaMemcpyHostToDevice, ctx->stream));
    SIEB_RETURN_IF(matvec_free_device(ctx, *mesh, *opt, tensors, dx, dy));
    SIEB_TRY_CUDA(cudaMemcpyAsync(y, dy, sizeof(cplx) * N, cudaMemcpyDeviceToHost, ctx->stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int sieb200_gstc_tensor_gradient(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                                 const double* lambda, const double* x, int on_device, double* s_out) {
    SIEB_RETURN_IF(validate(mesh, opt, nullptr, false));
    SIEB_CHECK(ctx && lambda && x && s_out, SIEB200_INVALID_ARG, "invalid gradient arguments");
    SIEB_CHECK(opt->formulation == SIEB200_GSTC, SIEB200_INVALID_ARG,
               "the tensor gradient exists for the GSTC formulation only");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    const int64_t N = system_dimension(opt->formulation, mesh->num_edges);
    const int64_t ns = 32 * mesh->num_faces;
    if (on_device) {
        SIEB_RETURN_IF(tensor_gradient_device(ctx, *mesh, *opt, reinterpret_cast<const cplx*>(lambda),
                                              reinterpret_cast<const cplx*>(x), reinterpret_cast<cplx*>(s_out)));
        SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
        return SIEB200_OK;
    }
    DeviceBuffer tmp;
    SIEB_RETURN_IF(tmp.reserve(sizeof(cplx) * (2 * N + ns)));
    cplx* dl = tmp.as<cplx>();
    cplx* dx = dl + N;
    cplx* ds = dx + N;
    SIEB_TRY_CUDA(cudaMemcpyAsync(dl, lambda, sizeof(cplx) * N, cudaMemcpyHostToDevice, ctx->stream));
    SIEB_TRY_CUDA(cudaMemcpyAsync(dx, x, sizeof(cplx) * N, cudaMemcpyHostToDevice, ctx->stream));
    SIEB_RETURN_IF(tensor_gradient_device(ctx, *mesh, *opt, dl, dx, ds));
    SIEB_TRY_CUDA(cudaMemcpyAsync(s_out, ds, sizeof(cplx) * ns, cudaMemcpyDeviceToHost, ctx->stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int sieb200_assemble_rhs(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                         const sieb200_source* sources, int num_sources, double* B, int b_on_device) {
    SIEB_RETURN_IF(validate(mesh, opt, nullptr, false));
    SIEB_CHECK(ctx && B && sources && num_sources > 0, SIEB200_INVALID_ARG, "invalid RHS arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    const int64_t N = system_dimension(opt->formulation, mesh->num_edges);
    if (b_on_device) {
        SIEB_RETURN_IF(assemble_rhs_device(ctx, *mesh, *opt, sources, num_sources, reinterpret_cast<cplx*>(B), N));
        SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
        return SIEB200_OK;
    }
    DeviceBuffer tmp;
    SIEB_RETURN_IF(tmp.reserve(sizeof(cplx) * N * num_sources));
    SIEB_RETURN_IF(assemble_rhs_device(ctx, *mesh, *opt, sources, num_sources, tmp.as<cplx>(), N));
    SIEB_TRY_CUDA(cudaMemcpyAsync(B, tmp.ptr, sizeof(cplx) * N * num_sources, cudaMemcpyDeviceToHost, ctx->stream));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int sieb200_dense_solver_create(sieb200_ctx* ctx, int64_t n, int method, sieb200_dense_solver** out) {
    SIEB_CHECK(ctx && out && n > 0, SIEB200_INVALID_ARG, "invalid dense solver arguments");
    SIEB_CHECK(method >= 0 && method <= 3, SIEB200_INVALID_ARG, "unsupported dense solver method");
    SIEB_CHECK(n <= std::numeric_limits<int>::max(), SIEB200_OVERFLOW, "matrix dimension exceeds the int limit");
    sieb200_dense_solver* s = new sieb200_dense_solver();
    s->impl.ctx = ctx;
    s->impl.n = n;
    s->impl.method = method;
    *out = s;
    return SIEB200_OK;
}

int sieb200_dense_solver_destroy(sieb200_dense_solver* s) {
    if (!s) return SIEB200_OK;
    cudaStreamSynchronize(s->impl.ctx->stream);
    mixed_release(&s->impl);
    delete s;
    return SIEB200_OK;
}

int sieb200_dense_solver_factorize(sieb200_dense_solver* s, double* A, int64_t lda) {
    SIEB_CHECK(s && A && lda >= s->impl.n, SIEB200_INVALID_ARG, "invalid factorize arguments");
    SIEB_TRY_CUDA(cudaSetDevice(s->impl.ctx->device));
    return s->impl.factorize(A, lda);
}

int sieb200_dense_solver_solve(sieb200_dense_solver* s, int64_t nrhs, double* B, int64_t ldb,
                               double tolerance, int max_iterations, int* iterations_out) {
    SIEB_CHECK(s && B && nrhs > 0 && ldb >= s->impl.n, SIEB200_INVALID_ARG, "invalid solve arguments");
    SIEB_TRY_CUDA(cudaSetDevice(s->impl.ctx->device));
    return s->impl.solve(nrhs, B, ldb, false, tolerance, max_iterations, iterations_out);
}

int sieb200_dense_solver_solve_adjoint(sieb200_dense_solver* s, int64_t nrhs, double* B, int64_t ldb,
                                       double tolerance, int max_iterations, int* iterations_out) {
    SIEB_CHECK(s && B && nrhs > 0 && ldb >= s->impl.n, SIEB200_INVALID_ARG, "invalid solve arguments");
    SIEB_TRY_CUDA(cudaSetDevice(s->impl.ctx->device));
    return s->impl.solve(nrhs, B, ldb, true, tolerance, max_iterations, iterations_out);
}

int sieb200_matvec(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec,
                   const double* x, double beta, double* y) {
    SIEB_CHECK(ctx && A && x && y && n > 0 && lda >= n && (prec == 0 || prec == 1),
               SIEB200_INVALID_ARG, "invalid matvec arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    DeviceBuffer scratch;
    SIEB_RETURN_IF(gemv_device(ctx, n, A, lda, prec, reinterpret_cast<const cplx*>(x), beta,
                               reinterpret_cast<cplx*>(y), scratch));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int sieb200_matvec_noalloc(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec,
                           const double* x, double beta, double* y) {
    SIEB_CHECK(ctx && A && x && y && n > 0 && lda >= n && (prec == 0 || prec == 1),
               SIEB200_INVALID_ARG, "invalid matvec arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    SIEB_RETURN_IF(gemv_device_static_scratch(ctx, n, A, lda, prec, reinterpret_cast<const cplx*>(x), beta,
                                              reinterpret_cast<cplx*>(y)));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int sieb200_zgemm(sieb200_ctx* ctx, int64_t m, int64_t nc, int64_t k, const double* A, int64_t lda,
                  const double* X, int64_t ldx, double* C, int64_t ldc, const double* alpha, const double* beta) {
    SIEB_CHECK(ctx && alpha && beta && m >= 0 && nc >= 0 && k >= 0, SIEB200_INVALID_ARG, "invalid zgemm arguments");
    if (m == 0 || nc == 0) return SIEB200_OK;
    SIEB_CHECK(C && ldc >= m && (k == 0 || (A && X && lda >= m && ldx >= k)), SIEB200_INVALID_ARG,
               "invalid zgemm arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    cudaEvent_t ev;
    ctx->prof.begin(ctx->stream, 2, 8.0 * (double)m * (double)nc * (double)k,
                    16.0 * ((double)m * k + (double)k * nc + 2.0 * (double)m * nc), &ev);
    SIEB_RETURN_IF(zgemm_device(ctx->stream, m, nc, k, reinterpret_cast<const cplx*>(A), lda,
                                reinterpret_cast<const cplx*>(X), ldx, reinterpret_cast<cplx*>(C), ldc,
                                cx(alpha[0], alpha[1]), cx(beta[0], beta[1])));
    ctx->prof.end(ctx->stream, ev);
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int sieb200_prepare_records(sieb200_ctx* ctx, int64_t faces, const double* maps, double reference_impedance,
                            double* records_out, double* diag_out) {
    SIEB_CHECK(ctx && faces >= 0, SIEB200_INVALID_ARG, "invalid record preparation arguments");
    SIEB_CHECK(std::isfinite(reference_impedance) && reference_impedance > 0, SIEB200_INVALID_ARG,
               "reference_impedance must be finite and positive");
    if (faces == 0) return SIEB200_OK;
    SIEB_CHECK(maps && records_out && diag_out, SIEB200_INVALID_ARG, "record arrays must not be null");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    SIEB_RETURN_IF(prepare_records_device(ctx, faces, maps, reference_impedance, records_out, diag_out));
    SIEB_TRY_CUDA(cudaStreamSynchronize(ctx->stream));
    return SIEB200_OK;
}

int64_t sieb200_launch_count(void) { return (int64_t)g_launches.load(); }

int sieb200_fp64_fma_peak(sieb200_ctx* ctx, double* tflops) {
    SIEB_CHECK(ctx && tflops, SIEB200_INVALID_ARG, "invalid FP64 probe arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    return fp64_fma_rate(ctx, tflops);
}

int sieb200_fp64_mma_peak(sieb200_ctx* ctx, double* tflops) {
    SIEB_CHECK(ctx && tflops, SIEB200_INVALID_ARG, "invalid FP64 probe arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    return fp64_mma_rate(ctx, tflops);
}

int sieb200_profile_enable(sieb200_ctx* ctx, int enable) {
    SIEB_CHECK(ctx && enable >= 0 && enable <= 2, SIEB200_INVALID_ARG, "invalid profile mode");
    ctx->prof.collect();
    ctx->prof.enabled = enable != 0;
    for (auto& k : ctx->prof.k) k = KernelProfile();
    ctx->prof.spans.clear();
    ctx->prof.timeline = enable == 2;
    if (ctx->prof.timeline) {
        SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
        if (!ctx->prof.base) SIEB_TRY_CUDA(cudaEventCreate(&ctx->prof.base));
        SIEB_TRY_CUDA(cudaEventRecord(ctx->prof.base, ctx->stream));
    }
    return SIEB200_OK;
}

int sieb200_profile_timeline(sieb200_ctx* ctx, int64_t capacity, int* kernel, double* start_ms,
                             double* end_ms, int64_t* count) {
    SIEB_CHECK(ctx && count && capacity >= 0 && (capacity == 0 || (kernel && start_ms && end_ms)),
               SIEB200_INVALID_ARG, "invalid timeline query");
    ctx->prof.collect();
    const auto& sp = ctx->prof.spans;
    *count = (int64_t)sp.size();
    for (int64_t i = 0; i < std::min<int64_t>(capacity, (int64_t)sp.size()); ++i) {
        kernel[i] = sp[i].kernel;
        start_ms[i] = sp[i].start_ms;
        end_ms[i] = sp[i].end_ms;
    }
    return SIEB200_OK;
}

int sieb200_profile_read(sieb200_ctx* ctx, int kernel, int64_t* launches, double* total_ms,
                         double* flops, double* bytes) {
    SIEB_CHECK(ctx && kernel >= 0 && kernel < Profiler::kKinds, SIEB200_INVALID_ARG, "invalid profile query");
    ctx->prof.collect();
    const KernelProfile& k = ctx->prof.k[kernel];
    if (launches) *launches = k.launches;
    if (total_ms) *total_ms = k.ms;
    if (flops) *flops = k.flops;
    if (bytes) *bytes = k.bytes;
    return SIEB200_OK;
}

int sieb200_gemm_tf32_sub_shifted(sieb200_ctx* ctx, int64_t m2, int64_t n, int k, const float* A,
                                  const float* B, float* C, int64_t ldc, int mode, int64_t col_shift) {
    SIEB_CHECK(ctx && A && B && C && ldc >= m2 && mode >= 0 && mode <= 5, SIEB200_INVALID_ARG,
               "invalid GEMM arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    GemmTC* g = nullptr;
    SIEB_RETURN_IF(gemm_tc_create(&g));
    gemm_tc_set_mode(g, mode >= 4 ? mode - 2 : mode);
    int st = gemm_tc_sub(g, ctx->stream, C, ldc, A, B, m2, n, k, 0, mode >= 4 ? 1 : 0, col_shift);
    if (st == SIEB200_OK) st = gemm_tc_check(g, ctx->stream);
    gemm_tc_destroy(g);
    return st;
}

int sieb200_gemm_tf32_sub(sieb200_ctx* ctx, int64_t m2, int64_t n, int k, const float* A,
                          const float* B, float* C, int64_t ldc, int mode) {
    return sieb200_gemm_tf32_sub_shifted(ctx, m2, n, k, A, B, C, ldc, mode, 0);
}

int sieb200_far_field(sieb200_ctx* ctx, const sieb200_mesh* mesh, const double* j_cur,
                      const double* m_cur, double k0, double eta0, int64_t ndir,
                      const double* r_hat, const double* theta_hat, const double* phi_hat,
                      double* f_theta, double* f_phi, double* intensity) {
    SIEB_CHECK(ctx && mesh && j_cur && ndir >= 0, SIEB200_INVALID_ARG, "invalid far-field arguments");
    SIEB_CHECK(ndir == 0 || (r_hat && theta_hat && phi_hat && f_theta && f_phi && intensity),
               SIEB200_INVALID_ARG, "far-field direction and output arrays must not be null");
    SIEB_CHECK(k0 > 0 && eta0 > 0, SIEB200_INVALID_ARG, "k0 and eta0 must be positive");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    return far_field_device(ctx, *mesh, j_cur, m_cur, k0, eta0, ndir, r_hat, theta_hat, phi_hat,
                            f_theta, f_phi, intensity);
}

int sieb200_incident_fields(sieb200_ctx* ctx, const sieb200_options* opt, const sieb200_source* source,
                            int64_t num_points, const double* points, double* E, double* H) {
    SIEB_CHECK(ctx && opt && source && num_points >= 0 && (num_points == 0 || (points && E && H)),
               SIEB200_INVALID_ARG, "invalid incident-field arguments");
    SIEB_CHECK(opt->frequency_hz > 0 && std::isfinite(opt->frequency_hz), SIEB200_INVALID_ARG,
               "SIE frequency must be positive");
    SIEB_CHECK(opt->vacuum_permittivity > 0 && opt->vacuum_permeability > 0, SIEB200_INVALID_ARG,
               "vacuum permittivity and permeability must be positive");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    return sieb200::incident_fields_device(ctx, *opt, *source, num_points, points, E, H);
}

int sieb200_far_field_matrix(sieb200_ctx* ctx, const sieb200_mesh* mesh, double k0, double eta0, int64_t ndir,
                             const double* r_hat, const double* theta_hat, const double* phi_hat, int a_on_device,
                             double* A) {
    SIEB_CHECK(ctx && mesh && mesh->vertices && mesh->faces && mesh->faces_edges && A && r_hat && theta_hat &&
                   phi_hat && ndir > 0 && ndir < (1 << 24) && mesh->num_edges > 0,
               SIEB200_INVALID_ARG, "invalid far-field matrix arguments");
    SIEB_CHECK(k0 > 0 && eta0 > 0, SIEB200_INVALID_ARG, "k0 and eta0 must be positive");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    if (a_on_device)
        return sieb200::far_field_matrix_device(ctx, *mesh, k0, eta0, ndir, r_hat, theta_hat, phi_hat,
                                                reinterpret_cast<sieb200::cplx*>(A));
    const size_t bytes = sizeof(sieb200::cplx) * 2 * (size_t)ndir * 2 * (size_t)mesh->num_edges;
    sieb200::DeviceBuffer tmp;
    SIEB_RETURN_IF(tmp.reserve(bytes));
    SIEB_RETURN_IF(sieb200::far_field_matrix_device(ctx, *mesh, k0, eta0, ndir, r_hat, theta_hat, phi_hat,
                                                    tmp.as<sieb200::cplx>()));
    SIEB_TRY_CUDA(cudaMemcpy(A, tmp.ptr, bytes, cudaMemcpyDeviceToHost));
    return SIEB200_OK;
}

int sieb200_surface_fields(sieb200_ctx* ctx, const sieb200_mesh* mesh, const double* j_cur,
                           const double* m_cur, int64_t nobs, const double* points, double frequency_hz,
                           double eps_r, double mu_r, double eps0, double mu0, int rule, double* E,
                           double* H) {
    SIEB_CHECK(ctx && mesh && mesh->vertices && mesh->faces && mesh->faces_edges && j_cur &&
                   (nobs == 0 || (points && E && H)),
               SIEB200_INVALID_ARG, "invalid surface-field arguments");
    SIEB_TRY_CUDA(cudaSetDevice(ctx->device));
    return sieb200::surface_fields_device(ctx, *mesh, j_cur, m_cur, nobs, points, frequency_hz, eps_r, mu_r,
                                          eps0, mu0, rule, E, H);
}

}  // extern "C"
