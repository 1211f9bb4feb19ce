/*
 * sieb200.h — C ABI of the B200-native dense method-of-moments library.
 *
 * Each entry point replaces one piece of the SIE-GSTC solver's public C++
 * surface (paths relative to that project). All arguments are plain pointers
 * and sizes; complex numbers are interleaved (re, im) doubles or floats;
 * dense matrices are column-major. Functions never throw, abort or trap:
 * they return a status code and leave a message for sieb200_last_error().
 *
 * Pointers documented as "host" may be any host memory; pointers documented
 * as "device" must be CUDA device (or managed) memory on the context's GPU.
 */
#ifndef SIEB200_H
#define SIEB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status ---- */
/* Replaces the C++ exceptions of src/sie_mom/solvers/gstc_sie.cu:71-179
 * (std::invalid_argument), include/sie_mom/cuda/dense_lu_solver.cuh:97-111
 * (singular LU, std::runtime_error) and gstc_sie.cu:474-503 (non-finite). */
enum {
    SIEB200_OK = 0,
    SIEB200_INVALID_ARG = 1,
    SIEB200_OVERFLOW = 2,
    SIEB200_SINGULAR = 3,
    SIEB200_NONFINITE = 4,
    SIEB200_NOT_CONVERGED = 5,
    SIEB200_CUDA_ERROR = 6,
    SIEB200_TIMEOUT = 7,
    SIEB200_NO_DEVICE = 8,
    SIEB200_OUT_OF_MEMORY = 9,
    SIEB200_UNSUPPORTED = 10     /* reserved: a reference option this library does not build
                                    (every option of the declared entry points is built) */
};

/* Thread-local message of the last failing call on this host thread. */
const char* sieb200_last_error(void);
/* ABI version of the declarations below; a binding checks it on load.
 * 2: sieb200_options gained variant, ntl_form, line_quadrature_points.
 * 3: sieb200_zgemm, sieb200_solve_gstc_sweep, sieb200_prepare_records,
 *    the own FP64 LU (SIEB200_SOLVER_LU_FP64); the mixed solver solves
 *    several right-hand sides together (profile kind 5). */
#define SIEB200_ABI_VERSION 3
int sieb200_version(void);

/* ----------------------------------------------------------- context ---- */
/* Owns one CUDA stream, device workspaces, LU factors and library handles.
 * One context per host thread; contexts on the same device are independent.
 * Replaces the per-call RAII buffers of include/sie_mom/cuda/device_buffer.cuh:46-172. */
typedef struct sieb200_ctx sieb200_ctx;
int sieb200_ctx_create(int device, sieb200_ctx** out);
int sieb200_ctx_destroy(sieb200_ctx* ctx);
int sieb200_ctx_synchronize(sieb200_ctx* ctx);
/* cudaStream_t of the context (as void*), for callers that order their own
 * work against it. */
void* sieb200_ctx_stream(sieb200_ctx* ctx);

/* -------------------------------------------------------------- mesh ---- */
/* Unique edges in first-appearance order over (face, local edge
 * (le, le+1 mod 3)), key (min, max); faces_edges[3f+le] = edge index.
 * Replaces ObjMeshLoader::buildEdgesAndMapping (src/sie_mom/mesh/obj_mesh_loader.cpp:360-386)
 * and SphericalSurface::buildEdgesAndMapping (src/sie_mom/mesh/spherical_surface.cpp:100-136).
 * edges_out: host, 2*3*num_faces ints capacity; faces_edges_out: host, 3*num_faces. */
int sieb200_build_edges(const int32_t* faces, int64_t num_faces, int32_t* edges_out,
                        int32_t* faces_edges_out, int64_t* num_edges_out);

/* Dunavant rule `rule` (1..20) as the kernels use it: points (xi, eta) and
 * weights rounded to float, in the expansion order of
 * src/sie_mom/quadrature/triangle_dunavant_rule.cpp:135-256, as
 * make_quadrature (include/sie_mom/quadrature/triangle_dunavant_rule.hpp:82-101)
 * returns them. Returns the point count (pts: 2*count floats, w: count), or
 * -1 for an invalid rule; NULL outputs only query the count. */
int sieb200_quadrature_rule(int rule, float* pts, float* w);

/* MeshData (include/sie_mom/mesh/spherical_surface.hpp:10-15); host pointers,
 * vertices as nV x 3 doubles, faces and faces_edges as nF x 3 ints. */
typedef struct {
    const double* vertices;
    int64_t num_vertices;
    const int32_t* faces;
    int64_t num_faces;
    const int32_t* faces_edges;
    int64_t num_edges;
} sieb200_mesh;

/* --------------------------------------------------------- options ---- */
enum { SIEB200_PEC_EFIE = 0, SIEB200_PMCHWT = 1, SIEB200_GSTC = 2 };
enum {
    SIEB200_SOLVER_LU_FP64 = 0,     /* own FP64 LU: butterfly transform + blocked LU without pivoting in
                                       complex128 (own kernels, FP64 GEMM trailing update), FP64
                                       refinement against the intact matrix; no adjoint solves */
    SIEB200_SOLVER_LU_CUSOLVER = 1, /* cusolverDnZgetrf/Zgetrs, as dense_lu_solver.cuh */
    SIEB200_SOLVER_MIXED_IR = 2,    /* split-FP32 tensor-core LU + FP64 GMRES refinement */
    SIEB200_SOLVER_GMRES_C64 = 3    /* Jacobi-preconditioned GMRES, complex64 copy of Z for the
                                       Krylov products, FP64 residual (gmres_solver.cuh:258-520) */
};
enum { SIEB200_BASIS_FACE = 0, SIEB200_BASIS_SPHERICAL = 1 };

/* Mirrors GstcSieOptions (include/sie_mom/solvers/gstc_sie.hpp:32-57),
 * DielectricOptions (include/sie_mom/solvers/dielectric/dielectric_solver.hpp:30-44)
 * and PecOptions (include/sie_mom/solvers/pec_solver.hpp:16-29).
 * Fill with sieb200_options_default(formulation, &opt) first: it sets the
 * reference's per-solver defaults (rule 7 / 17 / 17, threshold 0.1 lambda0,
 * vacuum constants of pec_solver.hpp:26-27 or gstc_sie.hpp:55-56). */
typedef struct {
    int formulation;
    double frequency_hz;
    double eps_r_interior, mu_r_interior;
    double eps_r_exterior, mu_r_exterior;
    int quadrature_rule;
    double singularity_threshold_lambda0;
    double vacuum_permittivity, vacuum_permeability;
    int basis;               /* GSTC frame */
    int tensors_are_uniform; /* GSTC: 32 complex values instead of 32 per face */
    int compute_residual;
    int solver;              /* SIEB200_SOLVER_* */
    double tolerance;        /* refinement / GMRES target on the scaled system */
    int max_iterations;
    int restart;
    /* Testing variant within the formulation: PecFormulation
     * (include/sie_mom/solvers/pec_solver.hpp:12) or DielectricFormulation
     * (include/sie_mom/solvers/dielectric/dielectric_solver.hpp:15-19);
     * SIEB200_VARIANT_* below, 0 for GSTC. */
    int variant;
    /* nTL integral form of the rotated variants (NtlIntegralForm,
     * dielectric_solver.hpp:22-25; PecNtlForm, pec_solver.hpp:13):
     * SIEB200_NTL_SURFACE (form B, the reference default) or SIEB200_NTL_LINE
     * (form A: the scalar term as a Gauss-Legendre line integral along the
     * testing edges), with line_quadrature_points (1..20, default 20). */
    int ntl_form;
    int line_quadrature_points;
} sieb200_options;
enum {
    SIEB200_VARIANT_T = 0,       /* T-EFIE / T-PMCHWT: RWG testing */
    SIEB200_VARIANT_N = 1,       /* N-EFIE / N-PMCHWT: n x RWG testing, nTL / nTK */
    SIEB200_VARIANT_N_JUMP = 2   /* N-MFIE (1/2 Gram - nTK) / N-Muller (nTL, nTK, Gram) */
};
enum { SIEB200_NTL_SURFACE = 0, SIEB200_NTL_LINE = 1 };
int sieb200_options_default(int formulation, sieb200_options* out);

/* Excitation (include/sie_mom/excitation/excitation.hpp:19-30): kind 0 is a
 * plane wave (a = real E0, b = propagation direction), kind 1 a dipole
 * (a = effective moment, b = position, is_magnetic). region 1 interior,
 * 2 exterior. The wavenumber and impedance are bound from the region's
 * medium as prepare_source does (src/sie_mom/excitation/excitation.cu:110-137). */
typedef struct {
    int kind;
    int region;
    double a[3];
    double b[3];
    int is_magnetic;
} sieb200_source;

/* Metrics (gstc_sie.hpp:108-202, dielectric_solver.hpp:49-67, pec_solver.hpp:31-44)
 * plus the refinement counters of the mixed solver. Residuals refer to the
 * internally scaled system, as in the reference. */
typedef struct {
    int64_t matrix_dimension;
    int64_t dense_matrix_bytes;
    double assembly_seconds;
    double factorization_seconds;
    double solve_seconds;
    double residual_seconds;
    int residual_computed;
    double rhs_norm;
    double absolute_residual;
    double relative_residual;
    double maximum_coefficient[4]; /* per current block [J1, M1, J2, M2] / [J, M] / [J] */
    int refinement_iterations;
    int solver;
} sieb200_metrics;

/* ------------------------------------------------------------ solvers --- */
/* PEC T-EFIE: solve_pec_dense (include/sie_mom/solvers/pec_solver.hpp:57-61).
 * current_out: host, num_edges complex (exterior J2). */
int sieb200_solve_pec_dense(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                            const sieb200_source* source, double* current_out,
                            sieb200_metrics* metrics);

/* T-PMCHWT: solve_dielectric_dense (include/sie_mom/solvers/dielectric/dielectric_solver.hpp:92-96).
 * currents_out: host, 2*num_edges complex [J, M], physical (M x eta0). */
int sieb200_solve_dielectric_dense(sieb200_ctx* ctx, const sieb200_mesh* mesh,
                                   const sieb200_options* opt, const sieb200_source* source,
                                   double* currents_out, sieb200_metrics* metrics);

/* SIE-GSTC batch: solve_gstc_dense_batch (include/sie_mom/solvers/gstc_sie.hpp:226-239)
 * and, with num_cases = 1, solve_gstc_dense (gstc_sie.hpp:214-219).
 * tensors: host, 32 complex per face (Lambda row-major then its inverse) or
 * 32 if tensors_are_uniform. Each case has up to one interior and one
 * exterior source: sources[2*c] (interior, kind < 0 = absent) and
 * sources[2*c+1] (exterior). currents_out: host, num_cases x 4*num_edges
 * complex [J1, M1, J2, M2], physical. metrics: num_cases entries. */
int sieb200_solve_gstc_dense_batch(sieb200_ctx* ctx, const sieb200_mesh* mesh,
                                   const double* tensors, const sieb200_options* opt,
                                   const sieb200_source* sources, int num_cases,
                                   double* currents_out, sieb200_metrics* metrics);

/* Batched sweep of independent SIE-GSTC systems (frequencies, meshes of
 * uneven size, tensor records): what the reference's sweep workflows do by
 * running solve_gstc_dense_batch once per instance
 * (applications/anisotropic_gstc_sphere/sie_gstc_sphere.py:198-297 driving
 * src/sie_mom/solvers/gstc_sie.cu:622), here in one call. The instances run
 * largest first on `concurrency` lanes; each lane owns a context (stream,
 * assembly workspaces) and device buffers sized by its first (largest)
 * instance, and its trailing GEMMs use 1/concurrency of the SMs, so small
 * systems' latency-bound steps overlap each other. Per instance: mesh,
 * tensors (host, 32 per face or 32 if uniform), options (GSTC; solver
 * SIEB200_SOLVER_MIXED_IR or SIEB200_SOLVER_LU_CUSOLVER), up to one interior
 * and one exterior source (kind < 0 = absent), host output of 4*num_edges
 * complex physical currents, optional metrics. seconds_out (optional): wall
 * time of the sweep. The first failing instance's status and message are
 * returned (NOT_CONVERGED does not stop the others). */
typedef struct {
    sieb200_mesh mesh;
    const double* tensors;
    sieb200_options opt;
    sieb200_source source[2];
    double* currents_out;
    sieb200_metrics* metrics;
} sieb200_sweep_instance;
int sieb200_solve_gstc_sweep(sieb200_ctx* ctx, const sieb200_sweep_instance* instances, int count,
                             int concurrency, double* seconds_out);

/* ------------------------------------------------- assembly building blocks */
/* Dense system matrix exactly as the reference kernels place it
 * (PEC: sie_kernels_assembly.cuh:610-705; PMCHWT: dielectric_kernels.cu:23-149;
 * GSTC: sie_kernels_assembly.cuh:156-272 + 460-594), eta0-scaled.
 * Z: complex128, N x N column-major with leading dimension N; device memory
 * when z_on_device != 0, else host. tensors: GSTC only (host). */
int sieb200_assemble_matrix(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                            const double* tensors, double* Z, int z_on_device);

/* Right-hand sides of num_sources sources as num_sources columns of length N
 * (sie_kernels_utils.cuh:184-232, dielectric_solver.cu:399-530, pec_solver.cu:242-264).
 * For GSTC, each column receives one source in its region's rows. */
int sieb200_assemble_rhs(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                         const sieb200_source* sources, int num_sources, double* B,
                         int b_on_device);

/* Matrix-free product y = Z x (sie_kernels_matvec.cuh:9-141 Calderon and
 * 143-327 mass blocks, there for GSTC with unscaled blocks and complex64
 * vectors): Z is the eta0-scaled matrix sieb200_assemble_matrix builds, for
 * every formulation, recomputed by the same quadrature kernels and contracted
 * with x slab by slab instead of stored (a pair-block workspace bounded by
 * the free memory replaces the N x N matrix). x, y: N complex128, device when
 * on_device != 0, else host. */
int sieb200_matvec_matrix_free(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                               const double* tensors, const double* x, double* y, int on_device);

/* Adjoint contraction of the SIE-GSTC system with respect to its per-face
 * tensor records (no counterpart in the reference, which has no adjoint):
 * s[32 f + k] = lambda^H (dZ / d record[f][k]) x, with record[f] the 32
 * complex values of face f (Lambda row-major, then its inverse) and Z the
 * eta0-scaled matrix sieb200_assemble_matrix builds. Z is linear in the
 * records (only the jump-condition mass blocks of face f depend on
 * record[f]). With lambda solving Z^H lambda = dL/dx (torch convention,
 * x.grad), dL/d record = -conj(s). lambda, x: 4*num_edges complex; s_out:
 * 32*num_faces complex (for uniform tensors sum over faces); device memory
 * when on_device != 0, else host. */
int sieb200_gstc_tensor_gradient(sieb200_ctx* ctx, const sieb200_mesh* mesh, const sieb200_options* opt,
                                 const double* lambda, const double* x, int on_device, double* s_out);

/* ---------------------------------------------------------- dense LA ---- */
/* DenseLuSolver (include/sie_mom/cuda/dense_lu_solver.cuh:17-184) as an
 * object: factorize a device complex128 matrix with the selected method, then
 * solve any number of right-hand sides. For SIEB200_SOLVER_MIXED_IR the
 * solver keeps its own split-FP32 factors plus a pointer to the FP64 matrix
 * (which must stay alive and unchanged) for the refinement residual. */
typedef struct sieb200_dense_solver sieb200_dense_solver;
int sieb200_dense_solver_create(sieb200_ctx* ctx, int64_t n, int method,
                                sieb200_dense_solver** out);
int sieb200_dense_solver_destroy(sieb200_dense_solver* s);
/* A: device, n x n complex128, leading dimension lda. SIEB200_SOLVER_LU_CUSOLVER
 * factors in place (as cusolverDnZgetrf does); the own FP64 LU and the mixed
 * method keep their factors apart and leave A intact (it must stay alive and
 * unchanged: their solves refine against it). */
int sieb200_dense_solver_factorize(sieb200_dense_solver* s, double* A, int64_t lda);
/* B: device, n x nrhs complex128 (ldb), overwritten with the solution.
 * tolerance/max_iterations apply to the mixed method (relative residual of
 * each column); iterations_out (optional) receives the refinement count. */
int sieb200_dense_solver_solve(sieb200_dense_solver* s, int64_t nrhs, double* B, int64_t ldb,
                               double tolerance, int max_iterations, int* iterations_out);
/* Conjugate-transpose solve A^H X = B with the same factors (adjoint). */
int sieb200_dense_solver_solve_adjoint(sieb200_dense_solver* s, int64_t nrhs, double* B,
                                       int64_t ldb, double tolerance, int max_iterations,
                                       int* iterations_out);

/* Complex matvec y = A x (+ beta y) on device data: A complex128 (prec 0) or
 * complex64 (prec 1), n x n, lda; x, y complex128. Replaces the cublasZgemv
 * residual of src/sie_mom/solvers/gstc_sie.cu:398-457. */
int sieb200_matvec(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec,
                   const double* x, double beta, double* y);

/* The matvec above without any allocation (no counterpart in the reference):
 * its partial sums go to one fixed 2 MiB device array per device instead of
 * a per-call workspace, for callers that may not allocate device memory at
 * the point of the call. n <= 131072, else SIEB200_INVALID_ARG. The first
 * call on a device does the set-up: it resolves the array's address
 * (cudaGetSymbolAddress) and loads this path's kernels onto the device
 * (lazy module loading would otherwise load them, and may allocate, at their
 * first launch); make that first call before any stream capture. After a
 * device reset the next call does the set-up again. Calls whose kernels
 * overlap in time on one device (two host threads, two contexts) race on
 * the array.
 * Synchronizes the context stream like sieb200_matvec. */
int sieb200_matvec_noalloc(sieb200_ctx* ctx, int64_t n, const void* A, int64_t lda, int prec,
                           const double* x, double beta, double* y);

/* FP64 complex product C = alpha A X + beta C on device data, column-major,
 * complex interleaved: A m x k (lda), X k x nc (ldx), C m x nc (ldc); alpha
 * and beta 2 doubles each (re, im); beta = 0 does not read C. The residual
 * R = B - Z X and the Krylov products of the multi-right-hand-side mixed
 * solve (hand-written SIMT FP64 kernel). Replaces, for a batch of cases,
 * the one cublasZgemv per case of src/sie_mom/solvers/gstc_sie.cu:398-457.
 * Synchronizes the context stream. */
int sieb200_zgemm(sieb200_ctx* ctx, int64_t m, int64_t nc, int64_t k, const double* A, int64_t lda,
                  const double* X, int64_t ldx, double* C, int64_t ldc, const double* alpha,
                  const double* beta);

/* Surface-parameter record preparation on the device: the per-face checks
 * and inversion of prepare_tensor_records
 * (src/sie_mom/gstc/tensor_io.py:17-132), one thread per face in FP64.
 * maps: device, faces x 16 complex (row-major physical 4x4 map per face).
 * records_out: device, faces x 32 complex (the map, then its inverse: the
 * record layout of face_tensors.bin). diag_out: device, faces x 8 doubles:
 * reciprocity defect, skew-Hermitian defect and off-diagonal size of the
 * impedance-balanced map (each relative to its largest entry), its largest
 * and smallest singular values (one-sided Jacobi), the balanced two-sided
 * inverse residual, the physical inverse residual (Frobenius), and flags
 * (1 balanced map non-finite, 2 zero pivot, 4 inverse non-finite,
 * 8 balanced inverse non-finite). The caller applies the reference's
 * tolerances and messages (sieb200.records). Synchronizes the stream. */
int sieb200_prepare_records(sieb200_ctx* ctx, int64_t faces, const double* maps, double reference_impedance,
                            double* records_out, double* diag_out);

/* Split-TF32 tensor-core contraction used by the mixed LU's trailing update
 * (no counterpart in the reference, which calls cuSOLVER): on device data,
 *   C[m2 x n] (fp32, column-major, ldc) -= A[m2 x k] * B[n x k]^T,
 * A and B K-major fp32, k a multiple of 32. mode 3: persistent tcgen05
 * kernel whose epilogue adds -A B^T to C by TMA reduction (no C load in the
 * CTA), mode 2: persistent tcgen05 kernel that loads, subtracts and stores
 * the C tile by TMA (modes 2 and 3 need C and ldc*4 16-byte aligned, else
 * mode 1 runs), mode 1: one-CTA-per-tile tcgen05 kernel, mode 0: SIMT kernel
 * on the same operands (checking path). Modes 4 and 5 (the epilogues of
 * modes 2 and 3) take split operands instead: A = [A_hi | A_lo] and
 * B = [B_hi | B_lo] along k (k a multiple of 64, C and ldc*4 16-byte
 * aligned), C -= A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T, each operand read
 * once per tile. */
int sieb200_gemm_tf32_sub(sieb200_ctx* ctx, int64_t m2, int64_t n, int k, const float* A,
                          const float* B, float* C, int64_t ldc, int mode);
/* The same contraction with the first 128 rows of C (one 64-unknown block row
 * of a realified complex matrix) restricted to columns [col_shift, n): those
 * rows' first col_shift columns are left untouched. This is the shape of the
 * mixed LU's trailing update, which leaves the next diagonal block to a
 * kernel running at the same time. 0 <= col_shift < n. */
int sieb200_gemm_tf32_sub_shifted(sieb200_ctx* ctx, int64_t m2, int64_t n, int k, const float* A,
                                  const float* B, float* C, int64_t ldc, int mode, int64_t col_shift);

/* Per-context kernel timing (no counterpart in the reference, which times
 * phases with std::chrono): when enabled, the library brackets each launch
 * of the listed kernels with CUDA events on the context stream and
 * accumulates launch count, device milliseconds and algorithmic work.
 * kernel 0: split-TF32 trailing GEMM (work = 2*m2*n*k TF32 flops and
 * 4*(2*m2*n + (m2 + n)*k) bytes per launch); 1: triangular solves
 * (work = bytes of factors read); 2: FP64 matvec (bytes of Z read);
 * 3: diagonal-block LU + inverses (with the previous block step's update
 * of the block; on the solver's lookahead stream); 4: block-step panels
 * (L21 with the previous step's update of its rows, and U12: one launch per
 * step); 5: the two blocked triangular solves of a multi-right-hand-side
 * preconditioner application (work = 24 np^2 nrhs TF32 flops and 48 np^2
 * bytes of packed factors); 6: whole mixed factorizations; 7: whole refined
 * solves (spans on the context stream unless stated). Kind 2 also counts the
 * FP64 complex GEMMs (8 m nc k flops). */
int sieb200_profile_enable(sieb200_ctx* ctx, int enable);
/* enable = 2 also keeps a timeline: per span its kernel kind and its start
 * and end in ms after the enable call (device timestamps, all streams).
 * Copies up to `capacity` spans in recording order; *count = spans kept. */
int sieb200_profile_timeline(sieb200_ctx* ctx, int64_t capacity, int* kernel, double* start_ms,
                             double* end_ms, int64_t* count);
/* Number of CUDA kernels the library has launched in this process. */
int64_t sieb200_launch_count(void);
/* Measured FP64 FMA throughput of the context's device in TFLOP/s (FMA = 2
 * flops; dependent-FMA chains on every SM, best of 5 timed launches): the
 * denominator of the assembly's FP64-pipe roofline (no reference counterpart). */
int sieb200_fp64_fma_peak(sieb200_ctx* ctx, double* tflops);
/* The same for the FP64 tensor cores (mma.sync m8n8k4 .f64, independent
 * accumulators on every SM): the denominator of the FP64 complex GEMM's
 * roofline (sieb200_zgemm; no reference counterpart). */
int sieb200_fp64_mma_peak(sieb200_ctx* ctx, double* tflops);
int sieb200_profile_read(sieb200_ctx* ctx, int kernel, int64_t* launches, double* total_ms,
                         double* flops, double* bytes);

/* --------------------------------------------------------- far field ---- */
/* Schelkunoff radiation vectors of the exterior RWG currents at the 7-point
 * rule, as MetasurfaceFarFieldEvaluator does
 * (applications/anisotropic_gstc_sphere/plot_far_field.py:118-220).
 * j_cur, m_cur: host, num_edges complex each (m_cur may be NULL).
 * Directions: host, ndir x 3 unit vectors each. Outputs: host, ndir complex
 * F_theta and F_phi, ndir real radiation intensities U. */
/* Incident E and H of one source (plane wave or dipole, bound to its
 * region's medium from opt) at num_points host points (x, y, z); E and H:
 * host, 3 complex per point. Replaces evaluate_incident_fields
 * (src/sie_mom/excitation/excitation.cu:158-210, declared in
 * include/sie_mom/excitation/excitation.hpp), which the apps subtract the
 * surface integrals from for their field cuts. */
int sieb200_incident_fields(sieb200_ctx* ctx, const sieb200_options* opt, const sieb200_source* source,
                            int64_t num_points, const double* points, double* E, double* H);

int sieb200_far_field(sieb200_ctx* ctx, const sieb200_mesh* mesh, const double* j_cur,
                      const double* m_cur, double k0, double eta0, int64_t ndir,
                      const double* r_hat, const double* theta_hat, const double* phi_hat,
                      double* f_theta, double* f_phi, double* intensity);

/* The same far field as an explicit operator, for differentiable objectives
 * (no counterpart in the reference): A is (2*ndir) x (2*num_edges) complex,
 * row-major, rows F_theta(d) then F_phi(d), columns J(e) then M(e) of the
 * exterior currents, so that [F_theta; F_phi] = A [J; M]. Directions: host;
 * A: device memory when a_on_device != 0, else host. */
int sieb200_far_field_matrix(sieb200_ctx* ctx, const sieb200_mesh* mesh, double k0, double eta0, int64_t ndir,
                             const double* r_hat, const double* theta_hat, const double* phi_hat, int a_on_device,
                             double* A);

/* Surface-integral field values at observation points
 * (evaluate_surface_integral_fields, include/sie_mom/solvers/
 * surface_current_fields.hpp:12-44; kernel sie_kernels_utils.cuh:21-140):
 *   E = +j w mu L[J] + K[M],   H = -K[J] + j w eps L[M]
 * with w = 2 pi f, eps = eps_r eps0, mu = mu_r mu0, k = w sqrt(mu eps); each
 * face by ordinary quadrature of the given Dunavant rule, or by quadrature of
 * the extracted kernel plus the analytic (Wilton) part when its centroid is
 * within 0.1 wavelength of the point. These are not the scattered or total
 * fields by themselves (F_total = F_incident - Q in the region of the
 * currents). j_cur, m_cur: host, num_edges physical coefficients each
 * (complex interleaved; m_cur NULL = 0). points: host, nobs x 3. E, H: host,
 * nobs x 3 complex interleaved. Same validation as the reference
 * (positive finite frequency, media and vacuum constants, rule 1..20,
 * finite points); nobs = 0 returns at once. */
int sieb200_surface_fields(sieb200_ctx* ctx, const sieb200_mesh* mesh, const double* j_cur,
                           const double* m_cur, int64_t nobs, const double* points, double frequency_hz,
                           double eps_r, double mu_r, double eps0, double mu0, int rule, double* E,
                           double* H);

#ifdef __cplusplus
}
#endif
#endif /* SIEB200_H */
