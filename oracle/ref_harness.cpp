// Test infrastructure only: a thin extern "C" harness around the reference's
// own host-compiled quadrature (sie_mom headers, USE_DOUBLE_PRECISION build).
// It is compiled by oracle/Makefile into oracle/_ref/libsieref.so and is used
//   * to pin the C restatement in oracle/sieoracle.c,
//   * to generate the golden fixtures under tests/golden/,
//   * as the timed CPU baseline ("reference" arm of bench.py).
// Nothing in the product links this file.
//
// The per-pair loops below mirror the reference CUDA kernels one-to-one,
// including their float demotions, so that the harness reproduces the
// reference GPU path ("ref-compat"), not the reference's host tests:
//   PEC T-EFIE     include/sie_mom/cuda/sie_kernels_assembly.cuh:610-705
//   T-PMCHWT       src/sie_mom/solvers/dielectric/dielectric_kernels.cu:23-149
//   GSTC Calderon  include/sie_mom/cuda/sie_kernels_assembly.cuh:156-272
//   GSTC mass      include/sie_mom/cuda/sie_kernels_assembly.cuh:460-594
//   RHS            include/sie_mom/cuda/sie_kernels_utils.cuh:184-232,
//                  src/sie_mom/solvers/dielectric/dielectric_solver.cu:399-530,
//                  src/sie_mom/solvers/pec_solver.cu:242-264

#include "sie_mom/cuda/platform.cuh"
#include "sie_mom/cuda/math_utils.cuh"
#include "sie_mom/cuda/mesh_geometry.cuh"
#include "sie_mom/cuda/dunavant_quadrature.cuh"
#include "sie_mom/cuda/semi_analytic_integrals.cuh"
#include "sie_mom/cuda/sie_scaling.cuh"
#include "sie_mom/cuda/gstc_tensor_utils.cuh"
#include "sie_mom/excitation/source_functors.cuh"
#include "sie_mom/quadrature/triangle_dunavant_rule.hpp"
#include "sie_mom/quadrature/gauss_legendre_rule.hpp"
#include "sie_mom/mesh/spherical_surface.hpp"

#include <Eigen/Dense>

#include <omp.h>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

namespace {

inline size_t cm_index(size_t row, size_t col, size_t ld) { return col * ld + row; }

inline void atomic_add(double* Z, size_t idx, const complex_t& v) {
#pragma omp atomic
    Z[2 * idx] += v.x;
#pragma omp atomic
    Z[2 * idx + 1] += v.y;
}

struct Quad {
    std::vector<float> pts, w;
    int n = 0;
    // Gauss-Legendre line rule of the nTL form A, float as the solvers upload it
    // (dielectric_solver.cu:179-197); empty for the surface form B.
    std::vector<float> lt, lw;
    int nl = 0;
};

void add_line_rule(Quad& q, int points) {
    if (points <= 0) return;
    std::vector<double> t(points), w(points);
    gauss_legendre_rule(points, t.data(), w.data());
    q.lt.assign(t.begin(), t.end());
    q.lw.assign(w.begin(), w.end());
    q.nl = points;
}

Quad make_rule(int rule) {
    Quad q;
    q.n = dunavant_order_num(rule);
    std::vector<double> p(2 * q.n), w(q.n);
    dunavant_rule(rule, q.n, p.data(), w.data());
    q.pts.resize(2 * q.n);
    q.w.resize(q.n);
    for (int i = 0; i < q.n; ++i) {
        q.pts[2 * i] = static_cast<float>(p[2 * i]);
        q.pts[2 * i + 1] = static_cast<float>(p[2 * i + 1]);
        q.w[i] = static_cast<float>(w[i]);
    }
    return q;
}

// Per face pair: TL/TK for k1 and k2, exactly as the assembly kernels call them.
void pair_blocks(const double* V, const int* F, int m, int n, const Quad& q, float k1, float k2,
                 float thr, complex_t tl1[3][3], complex_t tl2[3][3], complex_t tk1[3][3],
                 complex_t tk2[3][3]) {
    const int ti[3] = {F[3 * m], F[3 * m + 1], F[3 * m + 2]};
    const int si[3] = {F[3 * n], F[3 * n + 1], F[3 * n + 2]};
    vec3_t tv[3], sv[3];
    for (int a = 0; a < 3; ++a) {
        tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
        sv[a] = make_vec3(V[3 * si[a]], V[3 * si[a] + 1], V[3 * si[a] + 2]);
    }
    const vec3_t tc = (tv[0] + tv[1] + tv[2]) / 3.f;
    const vec3_t sc = (sv[0] + sv[1] + sv[2]) / 3.f;
    const float dist = length(tc - sc);
    if (dist < thr) {
        calculateDoubleQuadrature(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k1, k2, true,
                                  tl1, tl2, tk1, tk2);
        complex_t s1[3][3], s2[3][3], s3[3][3], s4[3][3];
        calculateSingularPartQuadrature(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k1, k2,
                                        s1, s2, s3, s4);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                complexAddInPlace(tl1[j][i], s1[j][i]);
                complexAddInPlace(tl2[j][i], s2[j][i]);
                complexAddInPlace(tk1[j][i], s3[j][i]);
                complexAddInPlace(tk2[j][i], s4[j][i]);
            }
    } else {
        calculateDoubleQuadrature(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k1, k2, false,
                                  tl1, tl2, tk1, tk2);
    }
}

// Per face pair: nTL/nTK (surface form B) for k1 and k2 as n_pmchwt_kernel
// calls them (dielectric_kernels.cu:155-270), float centroid distance.
void pair_blocks_n(const double* V, const int* F, int m, int n, const Quad& q, float k1, float k2,
                   float thr, complex_t l1[3][3], complex_t l2[3][3], complex_t n1[3][3],
                   complex_t n2[3][3]) {
    const int ti[3] = {F[3 * m], F[3 * m + 1], F[3 * m + 2]};
    const int si[3] = {F[3 * n], F[3 * n + 1], F[3 * n + 2]};
    vec3_t tv[3], sv[3];
    for (int a = 0; a < 3; ++a) {
        tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
        sv[a] = make_vec3(V[3 * si[a]], V[3 * si[a] + 1], V[3 * si[a] + 2]);
    }
    const vec3_t tc = (tv[0] + tv[1] + tv[2]) / 3.f;
    const vec3_t sc = (sv[0] + sv[1] + sv[2]) / 3.f;
    const float dist = length(tc - sc);
    if (dist < thr) {
        complex_t s1[3][3], s2[3][3], s3[3][3], s4[3][3];
        if (q.nl > 0) {
            calculateFormAQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, q.lt.data(),
                                             q.lw.data(), q.nl, k1, k2, true, l1, l2, n1, n2);
            calculateFormASingularPartQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n,
                                                         q.lt.data(), q.lw.data(), q.nl, k1, k2, s1, s2,
                                                         s3, s4);
        } else {
            calculateDoubleQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k1, k2,
                                              true, l1, l2, n1, n2);
            calculateSingularPartQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k1,
                                                    k2, s1, s2, s3, s4);
        }
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                complexAddInPlace(l1[j][i], s1[j][i]);
                complexAddInPlace(l2[j][i], s2[j][i]);
                complexAddInPlace(n1[j][i], s3[j][i]);
                complexAddInPlace(n2[j][i], s4[j][i]);
            }
    } else if (q.nl > 0) {
        calculateFormAQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, q.lt.data(),
                                         q.lw.data(), q.nl, k1, k2, false, l1, l2, n1, n2);
    } else {
        calculateDoubleQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k1, k2, false,
                                          l1, l2, n1, n2);
    }
}

// N-EFIE pair (pec_solver.cu:113-168): nTL2 at k2, extraction decided on the
// double centroid distance, only the singular nTL2 added.
void pair_n_efie(const double* V, const int* F, int m, int n, const Quad& q, float k2, float thr,
                 complex_t l2[3][3]) {
    const int ti[3] = {F[3 * m], F[3 * m + 1], F[3 * m + 2]};
    const int si[3] = {F[3 * n], F[3 * n + 1], F[3 * n + 2]};
    vec3_t tv[3], sv[3];
    for (int a = 0; a < 3; ++a) {
        tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
        sv[a] = make_vec3(V[3 * si[a]], V[3 * si[a] + 1], V[3 * si[a] + 2]);
    }
    const vec3_t cm = (tv[0] + tv[1] + tv[2]) / real_t(3);
    const vec3_t cn = (sv[0] + sv[1] + sv[2]) / real_t(3);
    const bool extract = length(cm - cn) < thr;
    complex_t l1[3][3], n1[3][3], n2[3][3];
    if (q.nl > 0)
        calculateFormAQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, q.lt.data(),
                                         q.lw.data(), q.nl, k2, k2, extract, l1, l2, n1, n2);
    else
        calculateDoubleQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k2, k2, extract,
                                          l1, l2, n1, n2);
    if (extract) {
        complex_t s1[3][3], s2[3][3], s3[3][3], s4[3][3];
        if (q.nl > 0)
            calculateFormASingularPartQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n,
                                                         q.lt.data(), q.lw.data(), q.nl, k2, k2, s1, s2,
                                                         s3, s4);
        else
            calculateSingularPartQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, k2, k2,
                                                    s1, s2, s3, s4);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) complexAddInPlace(l2[j][i], s2[j][i]);
    }
}

// Right-hand side of one source functor as the reference RHS kernels place it
// (see ref_rhs_plane_wave).
template <class Source>
int rhs_source(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
               const Source& pw, int region, double mu0_d, double eps0_d, double* b, int variant,
               double eps_r_src, double mu_r_src) {
    const bool rotated = variant != 0;
    const Quad q = make_rule(rule);
    const size_t N = (kind == 0) ? ne : (kind == 1 ? 2 * (size_t)ne : 4 * (size_t)ne);
    std::memset(b, 0, sizeof(double) * 2 * N);
    for (int m = 0; m < nf; ++m) {
        const int ti[3] = {F[3 * m], F[3 * m + 1], F[3 * m + 2]};
        vec3_t tv[3];
        for (int a = 0; a < 3; ++a)
            tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
        complex_t ve[3], vh[3];
        if (rotated)
            calculateExcitationQuadrature<TestingFunction::NxRWG>(tv, ti, q.pts.data(), q.w.data(),
                                                                  q.n, pw, ve, vh);
        else
            calculateExcitationQuadrature<TestingFunction::RWG>(tv, ti, q.pts.data(), q.w.data(),
                                                                q.n, pw, ve, vh);
        for (int i = 0; i < 3; ++i) {
            const size_t e = FE[3 * m + i];
            if (kind == 0 && variant == 2) {
                atomic_add(b, e, vh[i]);
            } else if (kind == 0) {
                atomic_add(b, e, ve[i]);
            } else if (kind == 1 && variant == 2) {
                const real_t eta0 = std::sqrt(mu0_d / eps0_d);
                const real_t scale_e = static_cast<real_t>(eps_r_src * eps0_d);
                const real_t scale_h = -static_cast<real_t>(mu_r_src * mu0_d) * eta0;
                atomic_add(b, e, complexScale(ve[i], scale_e));
                atomic_add(b, e + ne, complexScale(vh[i], scale_h));
            } else if (kind == 1) {
                const real_t eta0 = std::sqrt(mu0_d / eps0_d);
                const real_t sign = region == 2 ? real_t(1) : real_t(-1);
                atomic_add(b, e, complexScale(ve[i], sign));
                atomic_add(b, e + ne, complexScale(vh[i], sign * eta0));
            } else {
                const float mu0 = (float)mu0_d, eps0 = (float)eps0_d;
                const real_t eta0 = sqrt(static_cast<real_t>(mu0) / static_cast<real_t>(eps0));
                const size_t off = region == 1 ? 0 : 2 * (size_t)ne;
                atomic_add(b, e + off, ve[i]);
                atomic_add(b, e + off + ne, complexScale(vh[i], eta0));
            }
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int ref_dunavant(int rule, float* pts, float* w) {
    const Quad q = make_rule(rule);
    if (pts) std::memcpy(pts, q.pts.data(), sizeof(float) * 2 * q.n);
    if (w) std::memcpy(w, q.w.data(), sizeof(float) * q.n);
    return q.n;
}

// Double-precision Dunavant orbit data (suborder multiplicity, barycentric
// triple, weight) for one rule; returns the number of orbits.
int ref_dunavant_orbits(int rule, int* mult, double* xyz, double* w) {
    const int ns = dunavant_suborder_num(rule);
    int* so = dunavant_suborder(rule, ns);
    std::vector<double> sx(3 * ns), sw(ns);
    dunavant_subrule(rule, ns, sx.data(), sw.data());
    for (int s = 0; s < ns; ++s) {
        if (mult) mult[s] = so[s];
        if (xyz) for (int a = 0; a < 3; ++a) xyz[3 * s + a] = sx[3 * s + a];
        if (w) w[s] = sw[s];
    }
    delete[] so;
    return ns;
}

// Icosphere from the reference's SphericalSurface (vertices, faces, edges,
// faces_edges). Call once with null outputs to size.
int ref_icosphere(float radius, int level, int* nv, int* nf, int* ne, double* V, int* F, int* E,
                  int* FE) {
    sie_mom::mesh::SphericalSurface s(radius, level);
    const auto& d = s.getMeshData();
    *nv = (int)d.vertices.size();
    *nf = (int)d.faces.size();
    *ne = (int)d.edges.size();
    if (V)
        for (size_t i = 0; i < d.vertices.size(); ++i) {
            V[3 * i] = d.vertices[i].x;
            V[3 * i + 1] = d.vertices[i].y;
            V[3 * i + 2] = d.vertices[i].z;
        }
    if (F)
        for (size_t i = 0; i < d.faces.size(); ++i) {
            F[3 * i] = d.faces[i].x;
            F[3 * i + 1] = d.faces[i].y;
            F[3 * i + 2] = d.faces[i].z;
        }
    if (E)
        for (size_t i = 0; i < d.edges.size(); ++i) {
            E[2 * i] = d.edges[i].x;
            E[2 * i + 1] = d.edges[i].y;
        }
    if (FE)
        for (size_t i = 0; i < d.faces_edges.size(); ++i) {
            FE[3 * i] = d.faces_edges[i].x;
            FE[3 * i + 1] = d.faces_edges[i].y;
            FE[3 * i + 2] = d.faces_edges[i].z;
        }
    return 0;
}

// Wilton potentials of one observation point against one triangle
// (semi_analytic_integrals.cuh:563-667). out: phi0, phi1_base[3], phi2,
// phi3_base[3], r_pi[3], d  (12 doubles).
void ref_wilton(const double* r, const double* tri, double* out) {
    vec3_t t[3];
    for (int a = 0; a < 3; ++a) t[a] = make_vec3(tri[3 * a], tri[3 * a + 1], tri[3 * a + 2]);
    const WiltonPotentials p = calculateAllWiltonPotentials(make_vec3(r[0], r[1], r[2]), t);
    out[0] = p.phi_0;
    out[1] = p.phi_1_base.x; out[2] = p.phi_1_base.y; out[3] = p.phi_1_base.z;
    out[4] = p.phi_2;
    out[5] = p.phi_3_base.x; out[6] = p.phi_3_base.y; out[7] = p.phi_3_base.z;
    out[8] = p.r_pi.x; out[9] = p.r_pi.y; out[10] = p.r_pi.z;
    out[11] = p.d;
}

// phi_0 as the reference's standalone routine (semi_analytic_integrals.cuh:108-173).
double ref_phi0(const double* r, const double* tri) {
    vec3_t t[3];
    for (int a = 0; a < 3; ++a) t[a] = make_vec3(tri[3 * a], tri[3 * a + 1], tri[3 * a + 2]);
    return calculate_phi_0(make_vec3(r[0], r[1], r[2]), t);
}

// Local 3x3 blocks of one face pair: out = [tl1, tl2, tk1, tk2] each 3x3
// complex row-major (j test, i source), interleaved re/im (72 doubles).
// nTL1, nTL2, nTK1, nTK2 of face pair (m, n): surface form B (line_points 0)
// or line form A with that many Gauss-Legendre points.
void ref_pair_blocks_n(const double* V, const int* F, int m, int n, int rule, float k1, float k2,
                       float thr, int line_points, double* out) {
    Quad q = make_rule(rule);
    add_line_rule(q, line_points);
    complex_t a[3][3], b[3][3], c[3][3], d[3][3];
    pair_blocks_n(V, F, m, n, q, k1, k2, thr, a, b, c, d);
    complex_t(*blk[4])[3] = {a, b, c, d};
    for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                out[2 * (k * 9 + j * 3 + i)] = blk[k][j][i].x;
                out[2 * (k * 9 + j * 3 + i) + 1] = blk[k][j][i].y;
            }
}

void ref_pair_blocks(const double* V, const int* F, int m, int n, int rule, float k1, float k2,
                     float thr, double* out) {
    const Quad q = make_rule(rule);
    complex_t a[3][3], b[3][3], c[3][3], d[3][3];
    pair_blocks(V, F, m, n, q, k1, k2, thr, a, b, c, d);
    complex_t(*blk[4])[3] = {a, b, c, d};
    for (int k = 0; k < 4; ++k)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                out[2 * (k * 9 + j * 3 + i)] = blk[k][j][i].x;
                out[2 * (k * 9 + j * 3 + i) + 1] = blk[k][j][i].y;
            }
}

// Dense system matrix as the reference kernels assemble it.
// kind 0: PEC T-EFIE (N = ne), 1: T-PMCHWT (N = 2 ne), 2: GSTC (N = 4 ne,
// Calderon + mass, eta0-scaled); variant 1: N-EFIE / N-PMCHWT surface form
// (pec_solver.cu:113-168, dielectric_kernels.cu:155-318); variant 2: N-MFIE /
// N-Muller (pec_solver.cu:171-240, dielectric_kernels.cu:323-489). Z is complex
// interleaved, column-major,
// and is overwritten. Physical scalars are the float-demoted kernel arguments.
int ref_assemble(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
                 float k1, float k2, float mu_r1, float mu_r2, float eps_r1, float eps_r2,
                 float mu0, float eps0, float omega, float thr, const double* tensors,
                 int tensors_uniform, int basis, double* Z, int threads, int variant, int line_points) {
    Quad q = make_rule(rule);
    if (variant == 1 || (variant == 2 && kind == 1)) add_line_rule(q, line_points);
    const size_t N = (kind == 0) ? ne : (kind == 1 ? 2 * (size_t)ne : 4 * (size_t)ne);
    std::memset(Z, 0, sizeof(double) * 2 * N * N);
    if (threads > 0) omp_set_num_threads(threads);

#pragma omp parallel for schedule(dynamic, 1)
    for (int m = 0; m < nf; ++m) {
        for (int n = 0; n < nf; ++n) {
            complex_t tl1[3][3], tl2[3][3], tk1[3][3], tk2[3][3];
            const int te[3] = {FE[3 * m], FE[3 * m + 1], FE[3 * m + 2]};
            const int se[3] = {FE[3 * n], FE[3 * n + 1], FE[3 * n + 2]};
            if (kind == 0 && variant == 2) {
                // N-MFIE (pec_solver.cu:171-240).
                const int ti[3] = {F[3 * m], F[3 * m + 1], F[3 * m + 2]};
                const int si[3] = {F[3 * n], F[3 * n + 1], F[3 * n + 2]};
                vec3_t tv[3], sv[3];
                for (int a = 0; a < 3; ++a) {
                    tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
                    sv[a] = make_vec3(V[3 * si[a]], V[3 * si[a] + 1], V[3 * si[a] + 2]);
                }
                if (m == n) {
                    complex_t mass[3][3];
                    calculateMassMatrixQuadrature(tv, ti, q.pts.data(), q.w.data(), q.n, mass);
                    for (int j = 0; j < 3; ++j)
                        for (int i = 0; i < 3; ++i)
                            atomic_add(Z, cm_index(te[j], se[i], N), complexScale(mass[j][i], real_t(0.5)));
                    continue;
                }
                const vec3_t cm = (tv[0] + tv[1] + tv[2]) / real_t(3);
                const vec3_t cn = (sv[0] + sv[1] + sv[2]) / real_t(3);
                const bool extract = length(cm - cn) < thr;
                complex_t l1[3][3], l2[3][3], n1[3][3], n2[3][3];
                calculateFormAQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(), q.n, nullptr,
                                                 nullptr, 0, k2, k2, extract, l1, l2, n1, n2);
                if (extract) {
                    complex_t s1[3][3], s2[3][3], s3[3][3], s4[3][3];
                    calculateFormASingularPartQuadrature_nTL_nTK(tv, ti, sv, si, q.pts.data(), q.w.data(),
                                                                 q.n, nullptr, nullptr, 0, k2, k2, s1, s2,
                                                                 s3, s4);
                    for (int j = 0; j < 3; ++j)
                        for (int i = 0; i < 3; ++i) complexAddInPlace(n2[j][i], s4[j][i]);
                }
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i)
                        atomic_add(Z, cm_index(te[j], se[i], N), complexScale(n2[j][i], real_t(-1)));
                continue;
            }
            if (kind == 0 && variant == 1) {
                pair_n_efie(V, F, m, n, q, k2, thr, tl2);
                const float mu2 = (float)((double)mu_r2 * (double)mu0);
                const complex_t factor = make_complex(real_t(0), omega * mu2);
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i)
                        atomic_add(Z, cm_index(te[j], se[i], N), factor * tl2[j][i]);
                continue;
            }
            if (variant != 0)
                pair_blocks_n(V, F, m, n, q, k1, k2, thr, tl1, tl2, tk1, tk2);
            else
                pair_blocks(V, F, m, n, q, k1, k2, thr, tl1, tl2, tk1, tk2);
            if (kind == 1 && variant == 2) {
                // N-Muller (dielectric_kernels.cu:433-488).
                complex_t mass[3][3];
                if (m == n) {
                    const int ti[3] = {F[3 * m], F[3 * m + 1], F[3 * m + 2]};
                    vec3_t tv[3];
                    for (int a = 0; a < 3; ++a)
                        tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
                    calculateMassMatrixQuadrature(tv, ti, q.pts.data(), q.w.data(), q.n, mass);
                }
                const complex_t j_omega = make_complex(0.f, omega);
                const float mu1 = mu_r1 * mu0, mu2 = mu_r2 * mu0;
                const float eps1 = eps_r1 * eps0, eps2 = eps_r2 * eps0;
                const float eta0 = sqrtf(mu0 / eps0);
                const complex_t c_eps1 = j_omega * eps1, c_eps2 = j_omega * eps2;
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i) {
                        const complex_t z_jj = (c_eps2 * mu2) * tl2[j][i] - (c_eps1 * mu1) * tl1[j][i];
                        const complex_t z_mm = complexScale(-1.0f, z_jj);
                        complex_t z_jm = eps2 * tk2[j][i] - eps1 * tk1[j][i];
                        complex_t z_mj = mu2 * tk2[j][i] - mu1 * tk1[j][i];
                        if (m == n) {
                            const complex_t g = mass[j][i];
                            const float eps_factor = (eps1 + eps2) / 2.0f;
                            const float mu_factor = (mu1 + mu2) / 2.0f;
                            z_jm = z_jm - complexScale(eps_factor, g);
                            z_mj = z_mj - complexScale(mu_factor, g);
                        }
                        atomic_add(Z, cm_index(te[j], se[i], N), z_jj);
                        atomic_add(Z, cm_index(te[j], se[i] + ne, N), complexScale(z_jm, eta0));
                        atomic_add(Z, cm_index(te[j] + ne, se[i], N), complexScale(z_mj, eta0));
                        atomic_add(Z, cm_index(te[j] + ne, se[i] + ne, N), complexScale(z_mm, eta0 * eta0));
                    }
                continue;
            }
            if (kind == 0) {
                const complex_t c_efie = make_complex(0.f, omega * mu_r2 * mu0);
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i)
                        atomic_add(Z, cm_index(te[j], se[i], N), c_efie * tl2[j][i]);
            } else if (kind == 1) {
                const complex_t j_omega = make_complex(0.f, omega);
                const float mu1 = mu_r1 * mu0, mu2 = mu_r2 * mu0;
                const float e1 = eps_r1 * eps0, e2 = eps_r2 * eps0;
                const float eta0 = sqrtf(mu0 / eps0);
                const complex_t c_mu1 = j_omega * mu1, c_mu2 = j_omega * mu2;
                const complex_t c_eps1 = j_omega * e1, c_eps2 = j_omega * e2;
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i) {
                        const complex_t tk = tk1[j][i] + tk2[j][i];
                        const complex_t z_jj = c_mu1 * tl1[j][i] + c_mu2 * tl2[j][i];
                        const complex_t z_mm = c_eps1 * tl1[j][i] + c_eps2 * tl2[j][i];
                        const complex_t z_mj = -1.f * tk;
                        const complex_t z_jm = 1.f * tk;
                        atomic_add(Z, cm_index(te[j], se[i], N), z_jj);
                        atomic_add(Z, cm_index(te[j], se[i] + ne, N), complexScale(z_jm, eta0));
                        atomic_add(Z, cm_index(te[j] + ne, se[i], N), complexScale(z_mj, eta0));
                        atomic_add(Z, cm_index(te[j] + ne, se[i] + ne, N),
                                   complexScale(z_mm, eta0 * eta0));
                    }
            } else {
                // nvcc resolves this unqualified sqrt on a float argument to the
                // float overload (CUDA's math_functions.h: using std::sqrt), so the
                // reference GPU kernel forms eta0 in float; mirror that here.
                const real_t eta0 = sqrtf(mu0 / eps0);
                const auto f1 = sie_mom::cuda::make_eta0_scaled_calderon_factors(
                    omega, mu_r1 * mu0, eps_r1 * eps0, eta0);
                const auto f2 = sie_mom::cuda::make_eta0_scaled_calderon_factors(
                    omega, mu_r2 * mu0, eps_r2 * eps0, eta0);
                for (int j = 0; j < 3; ++j)
                    for (int i = 0; i < 3; ++i) {
                        const auto b1 =
                            sie_mom::cuda::make_eta0_scaled_calderon_block(tl1[j][i], tk1[j][i], f1);
                        const auto b2 =
                            sie_mom::cuda::make_eta0_scaled_calderon_block(tl2[j][i], tk2[j][i], f2);
                        const size_t r = te[j], c = se[i], E = ne;
                        atomic_add(Z, cm_index(r, c, N), b1.jj);
                        atomic_add(Z, cm_index(r, c + E, N), b1.jm);
                        atomic_add(Z, cm_index(r + E, c, N), b1.mj);
                        atomic_add(Z, cm_index(r + E, c + E, N), b1.mm);
                        atomic_add(Z, cm_index(r + 2 * E, c + 2 * E, N), b2.jj);
                        atomic_add(Z, cm_index(r + 2 * E, c + 3 * E, N), b2.jm);
                        atomic_add(Z, cm_index(r + 3 * E, c + 2 * E, N), b2.mj);
                        atomic_add(Z, cm_index(r + 3 * E, c + 3 * E, N), b2.mm);
                    }
            }
        }
    }

    if (kind == 2) {
        // GSTC jump-condition block A_M'' with eta0 scaling.
        const float eta0 = sqrtf(mu0 / eps0);
        const float eta0_sq = eta0 * eta0;
        const auto btype = basis == 0 ? GstcBasisType::face : GstcBasisType::spherical;
        for (int m = 0; m < nf; ++m) {
            const int ti[3] = {F[3 * m], F[3 * m + 1], F[3 * m + 2]};
            vec3_t tv[3];
            for (int a = 0; a < 3; ++a)
                tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
            vec3_t u, v;
            get_local_basis_vectors(tv[0], tv[1], tv[2], btype, u, v);
            const double* tp = tensors_uniform ? tensors : tensors + (size_t)m * 64;
            auto lift = [&](const double* M4, int rb, int cb, complex_t T[3][3]) {
                const int r0 = rb * 2, c0 = cb * 2;
                auto at = [&](int r, int c) { return make_complex(M4[2 * (r * 4 + c)], M4[2 * (r * 4 + c) + 1]); };
                rotate_tensor_2x2_to_3x3(at(r0, c0), at(r0, c0 + 1), at(r0 + 1, c0),
                                         at(r0 + 1, c0 + 1), u, v, T);
            };
            complex_t Y[4][3][3], Zt[4][3][3];
            lift(tp, 0, 0, Y[0]); lift(tp, 0, 1, Y[1]); lift(tp, 1, 0, Y[2]); lift(tp, 1, 1, Y[3]);
            lift(tp + 32, 0, 0, Zt[0]); lift(tp + 32, 0, 1, Zt[1]);
            lift(tp + 32, 1, 0, Zt[2]); lift(tp + 32, 1, 1, Zt[3]);
            complex_t T[8][3][3], R[8][3][3];
            const vec3_t nvec = normalize(cross(tv[1] - tv[0], tv[2] - tv[0]));
            for (int k = 0; k < 4; ++k) apply_perp_transform(Y[k], nvec, T[k]);
            for (int k = 0; k < 4; ++k) copy_tensor_3x3(Zt[k], T[4 + k]);
            calculateMassMatrixQuadrature(tv, ti, q.pts.data(), q.w.data(), q.n, T, R);
            const int le[3] = {FE[3 * m], FE[3 * m + 1], FE[3 * m + 2]};
            const size_t E = ne;
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    auto add = [&](size_t ro, size_t co, complex_t val, float s) {
                        atomic_add(Z, cm_index(le[j] + ro, le[i] + co, N), complexScale(val, s));
                    };
                    const float f = 0.5f, fq = 0.5f * 0.25f;
                    const complex_t Zee = R[4][j][i], Zem = R[5][j][i], Zme = R[6][j][i], Zmm = R[7][j][i];
                    const complex_t Yee = R[0][j][i], Yem = R[1][j][i], Yme = R[2][j][i], Ymm = R[3][j][i];
                    add(0, 0, complexAdd(complexScale(Zee, f), complexScale(Ymm, fq)), 1.f);
                    add(0, E, complexSub(complexScale(Zem, f), complexScale(Yme, fq)), eta0);
                    add(0, 2 * E, complexSub(complexScale(Zee, f), complexScale(Ymm, fq)), 1.f);
                    add(0, 3 * E, complexAdd(complexScale(Zem, f), complexScale(Yme, fq)), eta0);
                    add(E, 0, complexSub(complexScale(Zme, f), complexScale(Yem, fq)), eta0);
                    add(E, E, complexAdd(complexScale(Zmm, f), complexScale(Yee, fq)), eta0_sq);
                    add(E, 2 * E, complexAdd(complexScale(Zme, f), complexScale(Yem, fq)), eta0);
                    add(E, 3 * E, complexSub(complexScale(Zmm, f), complexScale(Yee, fq)), eta0_sq);
                    add(2 * E, 0, complexSub(complexScale(Zee, f), complexScale(Ymm, fq)), 1.f);
                    add(2 * E, E, complexAdd(complexScale(Zem, f), complexScale(Yme, fq)), eta0);
                    add(2 * E, 2 * E, complexAdd(complexScale(Zee, f), complexScale(Ymm, fq)), 1.f);
                    add(2 * E, 3 * E, complexSub(complexScale(Zem, f), complexScale(Yme, fq)), eta0);
                    add(3 * E, 0, complexAdd(complexScale(Zme, f), complexScale(Yem, fq)), eta0);
                    add(3 * E, E, complexSub(complexScale(Zmm, f), complexScale(Yee, fq)), eta0_sq);
                    add(3 * E, 2 * E, complexSub(complexScale(Zme, f), complexScale(Yem, fq)), eta0);
                    add(3 * E, 3 * E, complexAdd(complexScale(Zmm, f), complexScale(Yee, fq)), eta0_sq);
                }
        }
    }
    return 0;
}

// Right-hand side for one plane wave, as the reference RHS kernels place it.
// kind 0: PEC (E only, N = ne); 1: T-PMCHWT (N = 2 ne, sign by region,
// H rows x sign*eta0); 2: GSTC (N = 4 ne, region 1 -> [J1,M1] rows,
// region 2 -> [J2,M2] rows, H rows x eta0 from float mu0/eps0).
// k, eta: the source medium's wavenumber and impedance (double, unrounded).
// variant != 0: n x RWG testing (pec_solver.cu:372-386, dielectric_solver.cu:461-510);
// variant 2: N-MFIE places V_H, N-Muller scales by the source region's
// eps_r_src, mu_r_src.
int ref_rhs_plane_wave(int kind, const double* V, const int* F, const int* FE, int nf, int ne,
                       int rule, const double* E0, const double* khat, double k, double eta,
                       int region, double mu0_d, double eps0_d, double* b, int variant,
                       double eps_r_src, double mu_r_src) {
    sie_mom::cuda::PlaneWave pw;
    pw.E0 = make_vec3(E0[0], E0[1], E0[2]);
    pw.propagation_k = make_vec3(khat[0], khat[1], khat[2]);
    pw.k = k;
    pw.eta = eta;
    return rhs_source(kind, V, F, FE, nf, ne, rule, pw, region, mu0_d, eps0_d, b, variant, eps_r_src, mu_r_src);
}

// The same for a dipole (source_functors.cuh:51-130): moment, position, type.
int ref_rhs_dipole(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
                   const double* moment, const double* position, int is_magnetic, double k, double eta,
                   int region, double mu0_d, double eps0_d, double* b, int variant, double eps_r_src,
                   double mu_r_src) {
    sie_mom::cuda::DipoleSource d;
    d.p_vec = make_vec3(moment[0], moment[1], moment[2]);
    d.r_0 = make_vec3(position[0], position[1], position[2]);
    d.k = k;
    d.eta = eta;
    d.is_magnetic = is_magnetic != 0;
    return rhs_source(kind, V, F, FE, nf, ne, rule, d, region, mu0_d, eps0_d, b, variant, eps_r_src, mu_r_src);
}

// Surface-integral field values Q_E = j w mu L[J] + K[M], Q_H = -K[J] + j w eps L[M]
// at observation points, with the reference's own per-face quadrature helpers
// (calculateScatterFieldQuadrature / calculateScatterFieldSingular,
// dunavant_quadrature.cuh:1634-1770) in the loop of compute_scattered_fields_kernel
// (sie_kernels_utils.cuh:21-140) and the constants of
// surface_current_fields.cu:96-112 and :255-275. J, M, E, H complex interleaved.
int ref_surface_fields(const double* V, const int* F, const int* FE, int nf, int ne, const double* J,
                       const double* M, int nobs, const double* obs, double freq, double eps_r,
                       double mu_r, double eps0, double mu0, int rule, double* E, double* H) {
    (void)ne;
    const Quad q = make_rule(rule);
    const real_t pi = std::acos(real_t(-1));
    const real_t omega = real_t(2) * pi * freq;
    const real_t epsilon = eps_r * eps0, mu = mu_r * mu0;
    const real_t k = omega * std::sqrt(mu * epsilon);
    const complex__float coeff_J = make_complex(real_t(0), omega * mu);
    const complex__float coeff_M = make_complex(real_t(1), real_t(0));
    const complex__float coeff_J_h = make_complex(real_t(-1), real_t(0));
    const complex__float coeff_M_h = make_complex(real_t(0), omega * epsilon);
    for (int p = 0; p < nobs; ++p) {
        const vec3_t obs_point = make_vec3(obs[3 * p], obs[3 * p + 1], obs[3 * p + 2]);
        const complex__float zero = make_complex(real_t(0), real_t(0));
        cvec3_t acc_E = make_cvec3(zero, zero, zero), acc_H = make_cvec3(zero, zero, zero);
        for (int f = 0; f < nf; ++f) {
            const int ti[3] = {F[3 * f], F[3 * f + 1], F[3 * f + 2]};
            vec3_t tv[3];
            for (int a = 0; a < 3; ++a) tv[a] = make_vec3(V[3 * ti[a]], V[3 * ti[a] + 1], V[3 * ti[a] + 2]);
            const vec3_t centroid = (tv[0] + tv[1] + tv[2]) / 3.f;
            const float dist = length(obs_point - centroid);
            const float lambda = 2.0f * static_cast<float>(M_PI) / k;
            const float threshold = 0.1f * lambda;
            cvec3_t Lr[3], Kr[3];
            if (dist < threshold) {
                calculateScatterFieldQuadrature(obs_point, tv, ti, q.pts.data(), q.w.data(), q.n, k, true, Lr, Kr);
                cvec3_t Ls[3], Ks[3];
                calculateScatterFieldSingular(obs_point, tv, ti, k, Ls, Ks);
                for (int i = 0; i < 3; ++i) {
                    Lr[i] += Ls[i];
                    Kr[i] += Ks[i];
                }
            } else {
                calculateScatterFieldQuadrature(obs_point, tv, ti, q.pts.data(), q.w.data(), q.n, k, false, Lr, Kr);
            }
            for (int i = 0; i < 3; ++i) {
                const int e = FE[3 * f + i];
                const complex__float je = make_complex(J[2 * e], J[2 * e + 1]);
                const complex__float me = M ? make_complex(M[2 * e], M[2 * e + 1]) : zero;
                acc_E += complexMul(coeff_J, je) * Lr[i];
                acc_E += complexMul(coeff_M, me) * Kr[i];
                acc_H += complexMul(coeff_J_h, je) * Kr[i];
                acc_H += complexMul(coeff_M_h, me) * Lr[i];
            }
        }
        const cvec3_t* outs[2] = {&acc_E, &acc_H};
        double* dst[2] = {E + 6 * (size_t)p, H + 6 * (size_t)p};
        for (int o = 0; o < 2; ++o) {
            dst[o][0] = outs[o]->x.x; dst[o][1] = outs[o]->x.y;
            dst[o][2] = outs[o]->y.x; dst[o][3] = outs[o]->y.y;
            dst[o][4] = outs[o]->z.x; dst[o][5] = outs[o]->z.y;
        }
    }
    return 0;
}

// Eigen partial-pivot LU solve in complex128 (the reference host tests'
// solver, tests/cpp/sie_dielectric_sphere_test.cpp:290). A column-major.
// Returns seconds spent in factor+solve.
double ref_lu_solve(int n, const double* A, const double* b, double* x, int nrhs, int threads) {
    using Mat = Eigen::Matrix<std::complex<double>, Eigen::Dynamic, Eigen::Dynamic, Eigen::ColMajor>;
    if (threads > 0) {
        omp_set_num_threads(threads);
        Eigen::setNbThreads(threads);
    }
    Eigen::Map<const Mat> Am(reinterpret_cast<const std::complex<double>*>(A), n, n);
    Eigen::Map<const Mat> bm(reinterpret_cast<const std::complex<double>*>(b), n, nrhs);
    Mat Acopy = Am;
    const double t0 = omp_get_wtime();
    Eigen::PartialPivLU<Mat> lu(Acopy);
    Mat xs = lu.solve(bm);
    const double t1 = omp_get_wtime();
    std::memcpy(x, xs.data(), sizeof(double) * 2 * (size_t)n * nrhs);
    return t1 - t0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// The reference's source functors (include/sie_mom/excitation/source_functors.cuh:14-130)
// at n points: kind 0 plane wave (a = E0, b = unit direction), 1 dipole
// (a = moment, b = position). E, H complex interleaved, 3 per point.
int ref_incident_fields(int kind, const double* a, const double* b, int is_magnetic, double k, double eta,
                        int n, const double* pts, double* E, double* H) {
    for (int i = 0; i < n; ++i) {
        const vec3_t r = make_vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]);
        cvec3_t e, h;
        if (kind == 0) {
            sie_mom::cuda::PlaneWave pw;
            pw.E0 = make_vec3(a[0], a[1], a[2]);
            pw.propagation_k = make_vec3(b[0], b[1], b[2]);
            pw.k = k;
            pw.eta = eta;
            pw(r, e, h);
        } else {
            sie_mom::cuda::DipoleSource d;
            d.p_vec = make_vec3(a[0], a[1], a[2]);
            d.r_0 = make_vec3(b[0], b[1], b[2]);
            d.k = k;
            d.eta = eta;
            d.is_magnetic = is_magnetic != 0;
            d(r, e, h);
        }
        const complex_t ec[3] = {e.x, e.y, e.z}, hc[3] = {h.x, h.y, h.z};
        for (int c = 0; c < 3; ++c) {
            E[2 * (3 * i + c)] = ec[c].x; E[2 * (3 * i + c) + 1] = ec[c].y;
            H[2 * (3 * i + c)] = hc[c].x; H[2 * (3 * i + c) + 1] = hc[c].y;
        }
    }
    return 0;
}

// The reference's Gauss-Legendre rule on [0, 1] (gauss_legendre_rule.cpp), doubles.
int ref_gauss_legendre(int n, double* t, double* w) {
    if (n < 1 || n > gauss_legendre_max_points()) return -1;
    gauss_legendre_rule(n, t, w);
    return n;
}

}  // extern "C"
