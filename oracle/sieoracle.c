/* Test infrastructure only (the checker, never the product).
 *
 * A plain-C, single-pass restatement of the reference solver's dense MoM hot
 * path, written per face pair exactly as the reference CUDA kernels evaluate
 * it, float demotions included ("ref-compat"). It is pinned against the
 * reference's own host-compiled quadrature (oracle/_ref, tests under tests/)
 * and the golden fixtures in tests/golden/. Citations are relative to the
 * reference checkout.
 *
 * Compiled with -ffp-contract=off so that every product is rounded on its
 * own, as in the straightforward reading of the reference's source.
 */
#include "sieoracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double x, y, z; } v3;
typedef struct { double re, im; } cx;

static inline v3 V3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vscale(v3 a, double s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double vlen(v3 a) { return sqrt(vdot(a, a)); }
/* math_utils.cuh:139-142: normalize multiplies by the reciprocal length. */
static inline v3 vnorm(v3 a) { double inv = 1.0 / vlen(a); return vscale(a, inv); }

static inline cx CX(double re, double im) { cx r = {re, im}; return r; }
static inline cx cadd(cx a, cx b) { return CX(a.re + b.re, a.im + b.im); }
static inline cx csub(cx a, cx b) { return CX(a.re - b.re, a.im - b.im); }
static inline cx cmul(cx a, cx b) { return CX(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline cx cscale(cx a, double s) { return CX(a.re * s, a.im * s); }

/* ---------------------------------------------------------------- rules -- */
typedef struct { int mult; double a, b, c, w; } orbit_t;
typedef struct { int n; orbit_t o[19]; } rule_t;
static const rule_t RULES[20] = {
#include "../sie-gstc-2026_b200/csrc/dunavant_table.inc"
};

/* Expansion order of src/sie_mom/quadrature/triangle_dunavant_rule.cpp:135-256,
 * then the float rounding of triangle_dunavant_rule.hpp:95-100. */
int so_rule(int rule, float* pts, float* w) {
    if (rule < 1 || rule > 20) return -1;
    const rule_t* r = &RULES[rule - 1];
    int o = 0;
    for (int s = 0; s < r->n; ++s) {
        const double t[3] = {r->o[s].a, r->o[s].b, r->o[s].c};
        const int m = r->o[s].mult;
        const int reps = (m == 1) ? 1 : 3;
        for (int k = 0; k < reps; ++k) {
            if (pts) { pts[2 * o] = (float)t[k % 3]; pts[2 * o + 1] = (float)t[(k + 1) % 3]; }
            if (w) w[o] = (float)r->o[s].w;
            ++o;
        }
        if (m == 6)
            for (int k = 0; k < 3; ++k) {
                if (pts) { pts[2 * o] = (float)t[(k + 1) % 3]; pts[2 * o + 1] = (float)t[k]; }
                if (w) w[o] = (float)r->o[s].w;
                ++o;
            }
    }
    return o;
}

/* Gauss-Legendre rules on [0, 1] (src/sie_mom/quadrature/gauss_legendre_rule.cpp),
 * rounded to float as the solvers upload them (pec_solver.cu:67-75). */
#include "../sie-gstc-2026_b200/csrc/gauss_legendre_table.inc"

int so_gauss_legendre(int n, float* t, float* w) {
    if (n < 1 || n > 20) return -1;
    const int off = n * (n - 1) / 2;
    for (int q = 0; q < n; ++q) {
        if (t) t[q] = (float)kGaussLegendreNodes[off + q];
        if (w) w[q] = (float)kGaussLegendreWeights[off + q];
    }
    return n;
}

/* ---------------------------------------------------------------- mesh --- */
/* src/sie_mom/mesh/obj_mesh_loader.cpp:360-386: edges numbered by first
 * appearance over (face, local edge (le, le+1 mod 3)), key (min, max).
 * Quadratic search: the oracle only sees small meshes. */
int so_build_edges(const int* faces, int nf, int* edges, int* faces_edges) {
    int ne = 0;
    int* tmp = (int*)malloc(sizeof(int) * 2 * 3 * (size_t)nf);
    for (int f = 0; f < nf; ++f)
        for (int le = 0; le < 3; ++le) {
            int a = faces[3 * f + le], b = faces[3 * f + (le + 1) % 3];
            int lo = a < b ? a : b, hi = a < b ? b : a, found = -1;
            for (int e = 0; e < ne; ++e)
                if (tmp[2 * e] == lo && tmp[2 * e + 1] == hi) { found = e; break; }
            if (found < 0) { tmp[2 * ne] = lo; tmp[2 * ne + 1] = hi; found = ne++; }
            faces_edges[3 * f + le] = found;
        }
    if (edges) memcpy(edges, tmp, sizeof(int) * 2 * (size_t)ne);
    free(tmp);
    return ne;
}

/* ------------------------------------------------------------ geometry --- */
typedef struct {
    int idx[3];
    v3 v[3];
    v3 free_v[3];
    double len[3]; /* signed edge length */
} tri_t;

/* mesh_geometry.cuh:51-80 (getEdgeInfo). */
static void load_tri(const double* V, const int* F, int f, tri_t* t) {
    for (int a = 0; a < 3; ++a) {
        t->idx[a] = F[3 * f + a];
        t->v[a] = V3(V[3 * t->idx[a]], V[3 * t->idx[a] + 1], V[3 * t->idx[a] + 2]);
    }
    static const int A[3] = {0, 1, 2}, B[3] = {1, 2, 0}, FR[3] = {2, 0, 1};
    for (int e = 0; e < 3; ++e) {
        v3 ev = vsub(t->v[B[e]], t->v[A[e]]);
        double l = sqrt(ev.x * ev.x + ev.y * ev.y + ev.z * ev.z);
        t->free_v[e] = t->v[FR[e]];
        t->len[e] = (t->idx[A[e]] > t->idx[B[e]] ? 1.0 : -1.0) * l;
    }
}

/* mesh_geometry.cuh:211-222. */
static inline v3 map_point(const tri_t* t, double xi, double eta) {
    double zeta = 1.0 - xi - eta;
    return V3(t->v[0].x * zeta + t->v[1].x * xi + t->v[2].x * eta,
              t->v[0].y * zeta + t->v[1].y * xi + t->v[2].y * eta,
              t->v[0].z * zeta + t->v[1].z * xi + t->v[2].z * eta);
}

static inline int same_face(const tri_t* a, const tri_t* b) {
    return a->idx[0] == b->idx[0] && a->idx[1] == b->idx[1] && a->idx[2] == b->idx[2];
}

/* --------------------------------------------------------------- Wilton -- */
typedef struct { double phi0; v3 phi1b; double phi2; v3 phi3b; v3 r_pi; double d; } pots_t;

/* semi_analytic_integrals.cuh:35-92 (geometric terms) and 563-667 (all
 * potentials in one pass). */
static pots_t wilton(v3 r, const v3 tri[3]) {
    pots_t P;
    v3 n = vnorm(vcross(vsub(tri[1], tri[0]), vsub(tri[2], tri[0])));
    P.d = vdot(vsub(r, tri[0]), n);
    P.r_pi = vsub(r, vscale(n, P.d));
    const double ad = fabs(P.d);
    const double eps9f = (double)1e-9f;
    P.phi0 = 0.0; P.phi2 = 0.0;
    P.phi1b = V3(0, 0, 0); P.phi3b = V3(0, 0, 0);
    for (int e = 0; e < 3; ++e) {
        v3 vs = tri[e], ve = tri[(e + 1) % 3];
        v3 th = vnorm(vsub(ve, vs));
        v3 u = vcross(th, n);
        v3 rs = vsub(vs, vscale(n, vdot(n, vs)));
        v3 re = vsub(ve, vscale(n, vdot(n, ve)));
        v3 to_s = vsub(rs, P.r_pi);
        double p0 = fabs(vdot(to_s, u));
        double orient = vdot(to_s, u) >= 0.0 ? 1.0 : -1.0;
        double lp = vdot(vsub(re, P.r_pi), th);
        double lm = vdot(vsub(rs, P.r_pi), th);
        double Pp = hypot(p0, lp), Pm = hypot(p0, lm);
        double R0 = hypot(p0, ad);
        double Rp = hypot(Pp, ad), Rm = hypot(Pm, ad);
        double logt = (log(Rp) + log1p(lp / Rp)) - (log(Rm) + log1p(lm / Rm));
        if (p0 > eps9f) {
            double at = 0.0;
            if (ad > eps9f)
                at = atan2(p0 * lp, R0 * R0 + ad * Rp) - atan2(p0 * lm, R0 * R0 + ad * Rm);
            P.phi0 += orient * (p0 * logt - ad * at);
        }
        double st = (R0 * R0) * logt + (lp * Rp) - (lm * Rm);
        P.phi1b = vadd(P.phi1b, vscale(u, st));
        double term = 0.0;
        if (ad > 1e-6)
            term = (1.0 / ad) * (atan2(p0 * lp, R0 * R0 + ad * Rp) - atan2(p0 * lm, R0 * R0 + ad * Rm));
        else if (p0 > 1e-9)
            term = -((lp / (p0 * Pp)) - (lm / (p0 * Pm)));
        P.phi2 += orient * term;
        P.phi3b = vsub(P.phi3b, vscale(u, logt));
    }
    P.phi1b = vscale(P.phi1b, 0.5);
    return P;
}

void so_wilton(const double* r, const double* tri, double* out) {
    v3 t[3];
    for (int a = 0; a < 3; ++a) t[a] = V3(tri[3 * a], tri[3 * a + 1], tri[3 * a + 2]);
    pots_t P = wilton(V3(r[0], r[1], r[2]), t);
    out[0] = P.phi0; out[1] = P.phi1b.x; out[2] = P.phi1b.y; out[3] = P.phi1b.z;
    out[4] = P.phi2; out[5] = P.phi3b.x; out[6] = P.phi3b.y; out[7] = P.phi3b.z;
    out[8] = P.r_pi.x; out[9] = P.r_pi.y; out[10] = P.r_pi.z; out[11] = P.d;
}

/* semi_analytic_integrals.cuh:108-171 (calculate_phi_0, used on the testing
 * edges of the line form): an edge whose end is within 1e-9 of the point is
 * skipped, and on an edge's line (R0 < 1e-8) the end distances are
 * regularised by 1e-8. */
static double phi0_line(v3 r, const v3 tri[3]) {
    v3 n = vnorm(vcross(vsub(tri[1], tri[0]), vsub(tri[2], tri[0])));
    const double d = vdot(vsub(r, tri[0]), n);
    const v3 r_pi = vsub(r, vscale(n, d));
    const double ad = fabs(d);
    double phi0 = 0.0;
    for (int e = 0; e < 3; ++e) {
        v3 vs = tri[e], ve = tri[(e + 1) % 3];
        v3 th = vnorm(vsub(ve, vs));
        v3 u = vcross(th, n);
        v3 rs = vsub(vs, vscale(n, vdot(n, vs)));
        v3 re = vsub(ve, vscale(n, vdot(n, ve)));
        v3 to_s = vsub(rs, r_pi);
        double p0 = fabs(vdot(to_s, u));
        double orient = vdot(to_s, u) >= 0.0 ? 1.0 : -1.0;
        double lp = vdot(vsub(re, r_pi), th);
        double lm = vdot(vsub(rs, r_pi), th);
        double Pp = hypot(p0, lp), Pm = hypot(p0, lm);
        double R0 = hypot(p0, ad);
        double Rp = hypot(Pp, ad), Rm = hypot(Pm, ad);
        if (Rp < 1e-9 || Rm < 1e-9) continue;
        if (R0 < 1e-8) {
            Rp = sqrt(Rp * Rp + 1e-8 * 1e-8);
            Rm = sqrt(Rm * Rm + 1e-8 * 1e-8);
        }
        double logt = (log(Rp) + log1p(lp / Rp)) - (log(Rm) + log1p(lm / Rm));
        double at = 0.0;
        if (ad > 1e-9)
            at = atan2(p0 * lp, R0 * R0 + ad * Rp) - atan2(p0 * lm, R0 * R0 + ad * Rm);
        phi0 += orient * (p0 * logt - ad * at);
    }
    return phi0;
}

/* semi_analytic_integrals.cuh:422-427. */
static inline v3 psi1(const pots_t* P, v3 fv) {
    v3 irp = vadd(P->phi1b, vscale(P->r_pi, P->phi0));
    return vsub(irp, vscale(fv, P->phi0));
}

/* semi_analytic_integrals.cuh:481-498: k arrives as float, k^2/2 is formed in
 * float. */
static inline v3 upsilon(const pots_t* P, v3 fv, v3 r, float k) {
    v3 phi3 = vadd(P->phi3b, vscale(vsub(P->r_pi, fv), P->phi2));
    v3 ps = psi1(P, fv);
    const float k2o2 = k * k * 0.5f;
    v3 comb = vadd(phi3, vscale(ps, (double)k2o2));
    v3 Ri = vsub(r, fv);
    return vscale(vcross(Ri, comb), -1.0);
}

/* ------------------------------------------------------- Green kernels --- */
typedef struct { cx tl[2]; cx tk[2][3]; } kern_t;

/* green_functions_utils.cuh:236-288 (standard) and 295-361 (extracted). */
static void kernels(v3 r1, v3 r2, const double k[2], int regular, kern_t* K) {
    v3 Rv = vsub(r1, r2);
    double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
    if (!regular) {
        if (R < 1e-12) { memset(K, 0, sizeof(*K)); return; }
        double inv_R = 1.0 / R;
        v3 Rh = V3(Rv.x * inv_R, Rv.y * inv_R, Rv.z * inv_R);
        double i4pR = 1.0 / (4.0 * M_PI * R);
        for (int a = 0; a < 2; ++a) {
            double s = sin(k[a] * R), c = cos(k[a] * R);
            K->tl[a] = CX(c * i4pR, -s * i4pR);
            cx wg = cmul(CX(inv_R, k[a]), K->tl[a]);
            K->tk[a][0] = cscale(wg, Rh.x);
            K->tk[a][1] = cscale(wg, Rh.y);
            K->tk[a][2] = cscale(wg, Rh.z);
        }
    } else {
        if (R < 1e-9) {
            memset(K, 0, sizeof(*K));
            for (int a = 0; a < 2; ++a) K->tl[a] = CX(0.0, -k[a] / (4.0 * M_PI));
            return;
        }
        double i4p = 1.0 / (4.0 * M_PI);
        double inv_R = 1.0 / R, inv_R2 = inv_R * inv_R, inv_R3 = inv_R2 * inv_R;
        double i4pR = i4p * inv_R;
        for (int a = 0; a < 2; ++a) {
            double s = sin(k[a] * R), c = cos(k[a] * R);
            K->tl[a] = CX((c - 1.0) * i4pR, -s * i4pR);
            cx Kr = cmul(CX(inv_R3, k[a] * inv_R2), CX(c, -s));
            Kr.re += -(inv_R3 + k[a] * k[a] * 0.5 * inv_R);
            cx sc = cscale(Kr, i4p);
            K->tk[a][0] = cscale(sc, Rv.x);
            K->tk[a][1] = cscale(sc, Rv.y);
            K->tk[a][2] = cscale(sc, Rv.z);
        }
    }
}

/* ------------------------------------------------------ pair quadrature -- */
typedef struct { cx tl1[3][3], tl2[3][3], tk1[3][3], tk2[3][3]; } blocks_t;

/* dunavant_quadrature.cuh:207-324 (double quadrature with the standard or
 * extracted kernels). */
static void double_quad(const tri_t* T, const tri_t* S, const float* pts, const float* wts, int Q,
                        double k1, double k2, int regular, blocks_t* B) {
    memset(B, 0, sizeof(*B));
    const double k[2] = {k1, k2};
    const int coinc = same_face(T, S);
    for (int p = 0; p < Q; ++p) {
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        double wp = (double)wts[p];
        for (int q = 0; q < Q; ++q) {
            v3 rq = map_point(S, (double)pts[2 * q], (double)pts[2 * q + 1]);
            double wq = (double)wts[q];
            kern_t K;
            kernels(rp, rq, k, regular, &K);
            double cw = wp * wq;
            for (int j = 0; j < 3; ++j) {
                v3 rm = vsub(rp, T->free_v[j]);
                for (int i = 0; i < 3; ++i) {
                    v3 rn = vsub(rq, S->free_v[i]);
                    double db = 0.25 * vdot(rm, rn);
                    double m1 = db - 1.0 / (k1 * k1), m2 = db - 1.0 / (k2 * k2);
                    v3 tkm = vscale(vcross(rm, rn), 0.25);
                    B->tl1[j][i] = cadd(B->tl1[j][i], cscale(cscale(K.tl[0], m1), cw));
                    B->tl2[j][i] = cadd(B->tl2[j][i], cscale(cscale(K.tl[1], m2), cw));
                    if (!coinc) {
                        for (int a = 0; a < 2; ++a) {
                            cx d = CX(tkm.x * K.tk[a][0].re + tkm.y * K.tk[a][1].re + tkm.z * K.tk[a][2].re,
                                      tkm.x * K.tk[a][0].im + tkm.y * K.tk[a][1].im + tkm.z * K.tk[a][2].im);
                            cx* dst = a == 0 ? &B->tk1[j][i] : &B->tk2[j][i];
                            *dst = cadd(*dst, cscale(d, cw));
                        }
                    }
                }
            }
        }
    }
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = T->len[j] * S->len[i];
            B->tl1[j][i] = cscale(B->tl1[j][i], s);
            B->tl2[j][i] = cscale(B->tl2[j][i], s);
            B->tk1[j][i] = cscale(B->tk1[j][i], s);
            B->tk2[j][i] = cscale(B->tk2[j][i], s);
        }
}

/* dunavant_quadrature.cuh:769-875 (singular part: analytic inner integral,
 * Dunavant outer integral). k arrives as float-valued doubles. */
static void singular_quad(const tri_t* T, const tri_t* S, const float* pts, const float* wts,
                          int Q, double k1, double k2, blocks_t* B) {
    memset(B, 0, sizeof(*B));
    const int coinc = same_face(T, S);
    for (int p = 0; p < Q; ++p) {
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        double wp = (double)wts[p];
        pots_t P = wilton(rp, S->v);
        for (int j = 0; j < 3; ++j) {
            v3 rm = vsub(rp, T->free_v[j]);
            for (int i = 0; i < 3; ++i) {
                v3 ps = psi1(&P, S->free_v[i]);
                double db = 0.25 * vdot(rm, ps);
                v3 u1 = upsilon(&P, S->free_v[i], rp, (float)k1);
                v3 u2 = upsilon(&P, S->free_v[i], rp, (float)k2);
                double t1 = db - 1.0 / (k1 * k1) * P.phi0;
                double t2 = db - 1.0 / (k2 * k2) * P.phi0;
                B->tl1[j][i].re += t1 * wp;
                B->tl2[j][i].re += t2 * wp;
                if (!coinc) {
                    B->tk1[j][i].re += 0.25 * vdot(rm, u1) * wp;
                    B->tk2[j][i].re += 0.25 * vdot(rm, u2) * wp;
                }
            }
        }
    }
    v3 c = vcross(vsub(S->v[1], S->v[0]), vsub(S->v[2], S->v[0]));
    double area = 0.5 * vlen(c);
    double as = 1.0 / (4.0 * M_PI * area);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = as * T->len[j] * S->len[i];
            B->tl1[j][i] = cscale(B->tl1[j][i], s);
            B->tl2[j][i] = cscale(B->tl2[j][i], s);
            B->tk1[j][i] = cscale(B->tk1[j][i], s);
            B->tk2[j][i] = cscale(B->tk2[j][i], s);
        }
}

/* sie_kernels_assembly.cuh:195-229: float centroid distance against the float
 * threshold selects extraction. */
static void pair(const tri_t* T, const tri_t* S, const float* pts, const float* wts, int Q,
                 float k1, float k2, float thr, blocks_t* B) {
    v3 tc = vscale(vadd(vadd(T->v[0], T->v[1]), T->v[2]), 1.0);
    v3 sc = vscale(vadd(vadd(S->v[0], S->v[1]), S->v[2]), 1.0);
    tc = V3(tc.x / 3.0, tc.y / 3.0, tc.z / 3.0);
    sc = V3(sc.x / 3.0, sc.y / 3.0, sc.z / 3.0);
    float dist = (float)vlen(vsub(tc, sc));
    if (dist < thr) {
        blocks_t Sg;
        double_quad(T, S, pts, wts, Q, (double)k1, (double)k2, 1, B);
        singular_quad(T, S, pts, wts, Q, (double)k1, (double)k2, &Sg);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                B->tl1[j][i] = cadd(B->tl1[j][i], Sg.tl1[j][i]);
                B->tl2[j][i] = cadd(B->tl2[j][i], Sg.tl2[j][i]);
                B->tk1[j][i] = cadd(B->tk1[j][i], Sg.tk1[j][i]);
                B->tk2[j][i] = cadd(B->tk2[j][i], Sg.tk2[j][i]);
            }
    } else {
        double_quad(T, S, pts, wts, Q, (double)k1, (double)k2, 0, B);
    }
}

/* ------------------------------------------- rotated (n x RWG) testing -- */
static inline v3 face_normal(const tri_t* t) {
    return vnorm(vcross(vsub(t->v[1], t->v[0]), vsub(t->v[2], t->v[0])));
}

static inline cx vdot_c(v3 a, const cx c[3]) {
    return CX(a.x * c[0].re + a.y * c[1].re + a.z * c[2].re, a.x * c[0].im + a.y * c[1].im + a.z * c[2].im);
}

/* dunavant_quadrature.cuh:342-480 (surface form B): tau_mj = rho_mj x n_m,
 * nTL = 1/4 (tau . rho_ni) G - 1/(2 k^2) tau . tk, nTK = 1/4 (tau x rho_ni) . tk
 * with tk the TK kernel vector; nTK is left out on the coincident face, the
 * gradient term of nTL is not. Blocks: tl1/tl2 = nTL, tk1/tk2 = nTK. */
static void double_quad_n(const tri_t* T, const tri_t* S, const float* pts, const float* wts, int Q,
                          double k1, double k2, int regular, blocks_t* B) {
    memset(B, 0, sizeof(*B));
    const double k[2] = {k1, k2};
    const int coinc = same_face(T, S);
    const v3 nm = face_normal(T);
    for (int p = 0; p < Q; ++p) {
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        double wp = (double)wts[p];
        for (int q = 0; q < Q; ++q) {
            v3 rq = map_point(S, (double)pts[2 * q], (double)pts[2 * q + 1]);
            double wq = (double)wts[q];
            kern_t K;
            kernels(rp, rq, k, regular, &K);
            double cw = wp * wq;
            for (int j = 0; j < 3; ++j) {
                v3 tau = vcross(vsub(rp, T->free_v[j]), nm);
                for (int i = 0; i < 3; ++i) {
                    v3 rn = vsub(rq, S->free_v[i]);
                    double dtr = vdot(tau, rn);
                    v3 km = vscale(vcross(tau, rn), 0.25);
                    for (int a = 0; a < 2; ++a) {
                        cx ntl = cscale(K.tl[a], 0.25 * dtr);
                        ntl = cadd(ntl, cscale(vdot_c(tau, K.tk[a]), -0.5 / (k[a] * k[a])));
                        cx* dl = a == 0 ? &B->tl1[j][i] : &B->tl2[j][i];
                        *dl = cadd(*dl, cscale(ntl, cw));
                        if (!coinc) {
                            cx* dk = a == 0 ? &B->tk1[j][i] : &B->tk2[j][i];
                            *dk = cadd(*dk, cscale(vdot_c(km, K.tk[a]), cw));
                        }
                    }
                }
            }
        }
    }
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = T->len[j] * S->len[i];
            B->tl1[j][i] = cscale(B->tl1[j][i], s);
            B->tl2[j][i] = cscale(B->tl2[j][i], s);
            B->tk1[j][i] = cscale(B->tk1[j][i], s);
            B->tk2[j][i] = cscale(B->tk2[j][i], s);
        }
}

/* dunavant_quadrature.cuh:889-1040 (singular part of form B): with
 * phi_1 = phi_1b - d phi_0 n_n and the extracted gradient phi_3b - d phi_2 n_n,
 * nTL += 1/2 tau . (phi_1 + 1/2 R_i phi_0 + grad / k^2) (the gradient left out
 * on the coincident face), nTK += 1/4 tau . Upsilon_coul (not on the
 * coincident face); e_mj e_ni / (4 pi A_n) afterwards. */
static void singular_quad_n(const tri_t* T, const tri_t* S, const float* pts, const float* wts,
                            int Q, double k1, double k2, blocks_t* B) {
    memset(B, 0, sizeof(*B));
    const int coinc = same_face(T, S);
    const v3 nm = face_normal(T), nn = face_normal(S);
    for (int p = 0; p < Q; ++p) {
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        double wp = (double)wts[p];
        pots_t P = wilton(rp, S->v);
        v3 phi1 = vsub(P.phi1b, vscale(nn, P.d * P.phi0));
        v3 grad = vsub(P.phi3b, vscale(nn, P.d * P.phi2));
        for (int j = 0; j < 3; ++j) {
            v3 tau = vcross(vsub(rp, T->free_v[j]), nm);
            for (int i = 0; i < 3; ++i) {
                v3 Ri = vsub(rp, S->free_v[i]);
                v3 br = vadd(phi1, vscale(vscale(Ri, 0.5), P.phi0));
                v3 b1 = coinc ? br : vadd(br, vscale(grad, 1.0 / (k1 * k1)));
                v3 b2 = coinc ? br : vadd(br, vscale(grad, 1.0 / (k2 * k2)));
                B->tl1[j][i].re += 0.5 * vdot(tau, b1) * wp;
                B->tl2[j][i].re += 0.5 * vdot(tau, b2) * wp;
                if (!coinc) {
                    v3 u1 = upsilon(&P, S->free_v[i], rp, (float)k1);
                    v3 u2 = upsilon(&P, S->free_v[i], rp, (float)k2);
                    B->tk1[j][i].re += 0.25 * vdot(tau, u1) * wp;
                    B->tk2[j][i].re += 0.25 * vdot(tau, u2) * wp;
                }
            }
        }
    }
    v3 c = vcross(vsub(S->v[1], S->v[0]), vsub(S->v[2], S->v[0]));
    double as = 1.0 / (4.0 * M_PI * (0.5 * vlen(c)));
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = as * T->len[j] * S->len[i];
            B->tl1[j][i] = cscale(B->tl1[j][i], s);
            B->tl2[j][i] = cscale(B->tl2[j][i], s);
            B->tk1[j][i] = cscale(B->tk1[j][i], s);
            B->tk2[j][i] = cscale(B->tk2[j][i], s);
        }
}

/* Line rule of the nTL form A (Gauss-Legendre on [0, 1], float-rounded); n = 0
 * selects the surface form B. */
typedef struct { const float* t; const float* w; int n; } line_t;

/* dunavant_quadrature.cuh:492-692 (form A): nTL = 1/4 (tau . rho) G on both
 * areas plus, for every source basis, the testing-edge line integral
 * (L_e / 2A_m) (tau . nu_e) G / k^2 against the source area; nTK as in form B.
 * n_m is the cross product divided by its length. */
static void double_quad_a(const tri_t* T, const tri_t* S, const float* pts, const float* wts, int Q,
                          const line_t* L, double k1, double k2, int regular, blocks_t* B) {
    memset(B, 0, sizeof(*B));
    const double k[2] = {k1, k2};
    const int coinc = same_face(T, S);
    const v3 cr = vcross(vsub(T->v[1], T->v[0]), vsub(T->v[2], T->v[0]));
    const double twoA = vlen(cr);
    const v3 nm = V3(cr.x / twoA, cr.y / twoA, cr.z / twoA);
    for (int p = 0; p < Q; ++p) {
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        double wp = (double)wts[p];
        for (int q = 0; q < Q; ++q) {
            v3 rq = map_point(S, (double)pts[2 * q], (double)pts[2 * q + 1]);
            double wq = (double)wts[q];
            kern_t K;
            kernels(rp, rq, k, regular, &K);
            const double aw = wp * wq, vw = 0.25 * aw;
            for (int j = 0; j < 3; ++j) {
                v3 tau = vcross(vsub(rp, T->free_v[j]), nm);
                for (int i = 0; i < 3; ++i) {
                    v3 rn = vsub(rq, S->free_v[i]);
                    const double f = vw * vdot(tau, rn);
                    B->tl1[j][i] = cadd(B->tl1[j][i], cscale(K.tl[0], f));
                    B->tl2[j][i] = cadd(B->tl2[j][i], cscale(K.tl[1], f));
                    if (!coinc) {
                        v3 km = vscale(vcross(tau, rn), 0.25);
                        B->tk1[j][i] = cadd(B->tk1[j][i], cscale(vdot_c(km, K.tk[0]), aw));
                        B->tk2[j][i] = cadd(B->tk2[j][i], cscale(vdot_c(km, K.tk[1]), aw));
                    }
                }
            }
        }
    }
    for (int e = 0; e < 3; ++e) {
        const v3 vA = T->v[e], vB = T->v[(e + 1) % 3];
        const v3 E = vsub(vB, vA);
        const double Le = vlen(E);
        const v3 c = vcross(E, nm);
        const v3 nu = V3(c.x / Le, c.y / Le, c.z / Le);
        const double geom = Le / twoA;
        for (int q = 0; q < L->n; ++q) {
            const double t = (double)L->t[q], wl = (double)L->w[q];
            const v3 req = V3(vA.x + t * (vB.x - vA.x), vA.y + t * (vB.y - vA.y), vA.z + t * (vB.z - vA.z));
            for (int p = 0; p < Q; ++p) {
                v3 rnp = map_point(S, (double)pts[2 * p], (double)pts[2 * p + 1]);
                kern_t K;
                kernels(req, rnp, k, regular, &K);
                const double cw = wl * (double)wts[p];
                for (int j = 0; j < 3; ++j) {
                    v3 tau = vcross(vsub(req, T->free_v[j]), nm);
                    const double ff = geom * vdot(tau, nu);
                    const cx n1 = cscale(cscale(K.tl[0], ff / (k1 * k1)), cw);
                    const cx n2 = cscale(cscale(K.tl[1], ff / (k2 * k2)), cw);
                    for (int i = 0; i < 3; ++i) {
                        B->tl1[j][i] = cadd(B->tl1[j][i], n1);
                        B->tl2[j][i] = cadd(B->tl2[j][i], n2);
                    }
                }
            }
        }
    }
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            double s = T->len[j] * S->len[i];
            B->tl1[j][i] = cscale(B->tl1[j][i], s);
            B->tl2[j][i] = cscale(B->tl2[j][i], s);
            B->tk1[j][i] = cscale(B->tk1[j][i], s);
            B->tk2[j][i] = cscale(B->tk2[j][i], s);
        }
}

/* dunavant_quadrature.cuh:1040-1179 (singular part of form A): area nTL
 * 1/4 w tau . Psi_1 (no gradient), nTK 1/4 w tau . Upsilon_coul (not on the
 * coincident face), both scaled by e_mj e_ni / (4 pi A_n); the line part
 * sum_e sum_q L_e w_q (tau . nu_e) phi_0(r_eq) scaled by
 * e_mj e_ni / (8 pi A_m A_n k^2). */
static void singular_quad_a(const tri_t* T, const tri_t* S, const float* pts, const float* wts, int Q,
                            const line_t* L, double k1, double k2, blocks_t* B) {
    memset(B, 0, sizeof(*B));
    const v3 cr = vcross(vsub(T->v[1], T->v[0]), vsub(T->v[2], T->v[0]));
    const double twoA = vlen(cr);
    const double Am = 0.5 * twoA;
    const v3 nm = V3(cr.x / twoA, cr.y / twoA, cr.z / twoA);
    const double An = 0.5 * vlen(vcross(vsub(S->v[1], S->v[0]), vsub(S->v[2], S->v[0])));
    const int coinc = same_face(T, S);
    for (int p = 0; p < Q; ++p) {
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        const double wp = (double)wts[p];
        pots_t P = wilton(rp, S->v);
        for (int j = 0; j < 3; ++j) {
            v3 tau = vcross(vsub(rp, T->free_v[j]), nm);
            for (int i = 0; i < 3; ++i) {
                const double an = 0.25 * wp * vdot(tau, psi1(&P, S->free_v[i]));
                B->tl1[j][i].re += an;
                B->tl2[j][i].re += an;
                if (!coinc) {
                    v3 u1 = upsilon(&P, S->free_v[i], rp, (float)k1);
                    v3 u2 = upsilon(&P, S->free_v[i], rp, (float)k2);
                    B->tk1[j][i].re += 0.25 * wp * vdot(tau, u1);
                    B->tk2[j][i].re += 0.25 * wp * vdot(tau, u2);
                }
            }
        }
    }
    double line[3] = {0.0, 0.0, 0.0};
    for (int e = 0; e < 3; ++e) {
        const v3 vA = T->v[e], vB = T->v[(e + 1) % 3];
        const v3 E = vsub(vB, vA);
        const double Le = vlen(E);
        const v3 c = vcross(E, nm);
        const v3 nu = V3(c.x / Le, c.y / Le, c.z / Le);
        for (int q = 0; q < L->n; ++q) {
            const double t = (double)L->t[q], wl = (double)L->w[q];
            const v3 req = V3(vA.x + t * (vB.x - vA.x), vA.y + t * (vB.y - vA.y), vA.z + t * (vB.z - vA.z));
            const double ph0 = phi0_line(req, S->v);
            for (int j = 0; j < 3; ++j) {
                v3 tau = vcross(vsub(req, T->free_v[j]), nm);
                line[j] += Le * wl * vdot(tau, nu) * ph0;
            }
        }
    }
    const double as = 1.0 / (4.0 * M_PI * An);
    const double ls = 1.0 / (8.0 * M_PI * Am * An);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            const double edges = T->len[j] * S->len[i];
            const double l1 = edges * ls * line[j] / (k1 * k1);
            const double l2 = edges * ls * line[j] / (k2 * k2);
            B->tl1[j][i] = cadd(cscale(B->tl1[j][i], edges * as), CX(l1, 0.0));
            B->tl2[j][i] = cadd(cscale(B->tl2[j][i], edges * as), CX(l2, 0.0));
            B->tk1[j][i] = cscale(B->tk1[j][i], edges * as);
            B->tk2[j][i] = cscale(B->tk2[j][i], edges * as);
        }
}

/* dielectric_kernels.cu:155-270 and pec_solver.cu:113-168: rotated-testing
 * pair, form B (L->n == 0) or form A. Extraction below the threshold: the
 * dielectric kernels compare the float-rounded centroid distance, the PEC
 * kernels (exact != 0) the double one. */
static void pair_n(const tri_t* T, const tri_t* S, const float* pts, const float* wts, int Q,
                   const line_t* L, float k1, float k2, float thr, int exact, blocks_t* B) {
    v3 tc = vadd(vadd(T->v[0], T->v[1]), T->v[2]);
    v3 sc = vadd(vadd(S->v[0], S->v[1]), S->v[2]);
    tc = V3(tc.x / 3.0, tc.y / 3.0, tc.z / 3.0);
    sc = V3(sc.x / 3.0, sc.y / 3.0, sc.z / 3.0);
    const double dd = vlen(vsub(tc, sc));
    const int near = exact ? (dd < (double)thr) : ((float)dd < thr);
    blocks_t Sg;
    if (L->n > 0) {
        double_quad_a(T, S, pts, wts, Q, L, (double)k1, (double)k2, near, B);
        if (near) singular_quad_a(T, S, pts, wts, Q, L, (double)k1, (double)k2, &Sg);
    } else {
        double_quad_n(T, S, pts, wts, Q, (double)k1, (double)k2, near, B);
        if (near) singular_quad_n(T, S, pts, wts, Q, (double)k1, (double)k2, &Sg);
    }
    if (near)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                B->tl1[j][i] = cadd(B->tl1[j][i], Sg.tl1[j][i]);
                B->tl2[j][i] = cadd(B->tl2[j][i], Sg.tl2[j][i]);
                B->tk1[j][i] = cadd(B->tk1[j][i], Sg.tk1[j][i]);
                B->tk2[j][i] = cadd(B->tk2[j][i], Sg.tk2[j][i]);
            }
}

static void pair_blocks_out(const double* V, const int* F, int m, int n, int rule, float k1, float k2,
                            float thr, int rotated, int line_points, double* out) {
    float pts[2 * 80], wts[80], lt[20], lw[20];
    int Q = so_rule(rule, pts, wts);
    line_t L = {lt, lw, line_points > 0 ? so_gauss_legendre(line_points, lt, lw) : 0};
    tri_t T, S;
    load_tri(V, F, m, &T);
    load_tri(V, F, n, &S);
    blocks_t B;
    if (rotated)
        pair_n(&T, &S, pts, wts, Q, &L, k1, k2, thr, 0, &B);
    else
        pair(&T, &S, pts, wts, Q, k1, k2, thr, &B);
    cx(*blk[4])[3] = {B.tl1, B.tl2, B.tk1, B.tk2};
    for (int b = 0; b < 4; ++b)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                out[2 * (b * 9 + j * 3 + i)] = blk[b][j][i].re;
                out[2 * (b * 9 + j * 3 + i) + 1] = blk[b][j][i].im;
            }
}

void so_pair_blocks(const double* V, const int* F, int m, int n, int rule, float k1, float k2,
                    float thr, double* out) {
    pair_blocks_out(V, F, m, n, rule, k1, k2, thr, 0, 0, out);
}

/* nTL1, nTL2, nTK1, nTK2 of face pair (m, n): surface form B (line_points 0)
 * or line form A with that many Gauss-Legendre points. */
void so_pair_blocks_n(const double* V, const int* F, int m, int n, int rule, float k1, float k2,
                      float thr, int line_points, double* out) {
    pair_blocks_out(V, F, m, n, rule, k1, k2, thr, 1, line_points, out);
}

/* ------------------------------------------------------- GSTC frames ---- */
/* gstc_tensor_utils.cuh:72-91 (face frame) and 106-147 (spherical frame). */
static void frame(const v3 v[3], int basis, v3* u, v3* w) {
    if (basis == 0) {
        v3 e1 = vsub(v[1], v[0]), e2 = vsub(v[2], v[0]);
        v3 nn = vcross(e1, e2);
        double l1 = vlen(e1), ln = vlen(nn);
        if (l1 < 1e-20 || ln < 1e-20) { *u = V3(1, 0, 0); *w = V3(0, 1, 0); return; }
        v3 nh = vscale(nn, 1.0 / ln);
        *u = vscale(e1, 1.0 / l1);
        *w = vcross(nh, *u);
    } else {
        v3 c = V3((v[0].x + v[1].x + v[2].x) / 3.0, (v[0].y + v[1].y + v[2].y) / 3.0,
                  (v[0].z + v[1].z + v[2].z) / 3.0);
        double r = vlen(c);
        if (r < 1e-12) { *u = V3(1, 0, 0); *w = V3(0, 1, 0); return; }
        double ct = c.z / r;
        if (ct > 1.0) ct = 1.0;
        if (ct < -1.0) ct = -1.0;
        double th = acos(ct), ph = atan2(c.y, c.x);
        double cth = cos(th), sth = sin(th), cph = cos(ph), sph = sin(ph);
        *u = V3(cth * cph, cth * sph, -sth);
        *w = V3(-sph, cph, 0.0);
    }
}

/* gstc_tensor_utils.cuh:184-238: T = R t R^T with R = [u, w]. */
static void lift(cx t00, cx t01, cx t10, cx t11, v3 u, v3 w, cx T[3][3]) {
    const double uc[3] = {u.x, u.y, u.z}, wc[3] = {w.x, w.y, w.z};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            cx s = CX(0, 0);
            s = cadd(s, cscale(t00, uc[i] * uc[j]));
            s = cadd(s, cscale(t01, uc[i] * wc[j]));
            s = cadd(s, cscale(t10, wc[i] * uc[j]));
            s = cadd(s, cscale(t11, wc[i] * wc[j]));
            T[i][j] = s;
        }
}

/* gstc_tensor_utils.cuh:269-309: -[n]x T [n]x with float-cast entries. */
static void perp(cx Tin[3][3], v3 n, cx Tout[3][3]) {
    const double N[3][3] = {{0.0, -n.z, n.y}, {n.z, 0.0, -n.x}, {-n.y, n.x, 0.0}};
    cx tmp[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            cx s = CX(0, 0);
            for (int k = 0; k < 3; ++k) s = cadd(s, cscale(Tin[r][k], (double)(float)N[k][c]));
            tmp[r][c] = s;
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            cx s = CX(0, 0);
            for (int k = 0; k < 3; ++k) s = cadd(s, cscale(tmp[k][c], (double)(float)N[r][k]));
            Tout[r][c] = CX(-s.re, -s.im);
        }
}

/* dunavant_quadrature.cuh:1422-1508: 8 tensors in one pass, float geometry. */
static void mass8(const tri_t* T, const float* pts, const float* wts, int Q, cx Tt[8][3][3],
                  cx R[8][3][3]) {
    memset(R, 0, sizeof(cx) * 72);
    v3 c = vcross(vsub(T->v[1], T->v[0]), vsub(T->v[2], T->v[0]));
    const float area = (float)(0.5 * vlen(c));
    float el[3];
    for (int i = 0; i < 3; ++i) el[i] = (float)T->len[i];
    for (int p = 0; p < Q; ++p) {
        const float wp = wts[p];
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        v3 rho[3];
        for (int i = 0; i < 3; ++i) rho[i] = vsub(rp, T->free_v[i]);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i)
                for (int k = 0; k < 8; ++k) {
                    cx (*t)[3] = Tt[k];
                    cx tx = cadd(cscale(t[0][0], rho[i].x), cadd(cscale(t[0][1], rho[i].y), cscale(t[0][2], rho[i].z)));
                    cx ty = cadd(cscale(t[1][0], rho[i].x), cadd(cscale(t[1][1], rho[i].y), cscale(t[1][2], rho[i].z)));
                    cx tz = cadd(cscale(t[2][0], rho[i].x), cadd(cscale(t[2][1], rho[i].y), cscale(t[2][2], rho[i].z)));
                    cx ig = cadd(cscale(tx, rho[j].x), cadd(cscale(ty, rho[j].y), cscale(tz, rho[j].z)));
                    R[k][j][i] = cadd(R[k][j][i], cscale(ig, (double)wp));
                }
    }
    const float sc = 1.f / (4.f * area);
    for (int k = 0; k < 8; ++k)
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                const float fs = sc * el[j] * el[i];
                R[k][j][i] = cscale(R[k][j][i], (double)fs);
            }
}

/* dunavant_quadrature.cuh:1261-1326: RWG Gram block <f_j, f_i> of one face;
 * the dot product is rounded to float and multiplied by the float weight in
 * float, the scale 1/(4A) e_j e_i is formed in float. */
static void gram(const tri_t* T, const float* pts, const float* wts, int Q, double G[3][3]) {
    memset(G, 0, sizeof(double) * 9);
    v3 c = vcross(vsub(T->v[1], T->v[0]), vsub(T->v[2], T->v[0]));
    const float area = (float)(0.5 * vlen(c));
    float el[3];
    for (int i = 0; i < 3; ++i) el[i] = (float)T->len[i];
    for (int p = 0; p < Q; ++p) {
        const float wp = wts[p];
        v3 rp = map_point(T, (double)pts[2 * p], (double)pts[2 * p + 1]);
        v3 rho[3];
        for (int i = 0; i < 3; ++i) rho[i] = vsub(rp, T->free_v[i]);
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                const float d = (float)vdot(rho[j], rho[i]);
                G[j][i] += (double)(wp * d);
            }
    }
    const float sc = 1.f / (4.f * area);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) G[j][i] *= (double)(sc * el[j] * el[i]);
}

/* ------------------------------------------------------------ assembly -- */
/* Destination of an assembly: the whole matrix (rowmap NULL, ld = N) or
 * selected rows of it (rowmap[r] = output row or -1, ld = output rows). */
typedef struct { double* Z; size_t ld; const int* rowmap; } ztarget_t;

static inline void zadd(const ztarget_t* T, size_t N, size_t r, size_t c, cx v) {
    (void)N;
    if (T->rowmap) {
        const int rr = T->rowmap[r];
        if (rr < 0) return;
        r = (size_t)rr;
    }
    size_t idx = c * T->ld + r;
    T->Z[2 * idx] += v.re;
    T->Z[2 * idx + 1] += v.im;
}

/* kind 0: PEC T-EFIE (sie_kernels_assembly.cuh:610-705), with variant 1
 *         N-EFIE surface form (pec_solver.cu:113-168), variant 2 N-MFIE
 *         (pec_solver.cu:171-240),
 * kind 1: T-PMCHWT (dielectric_kernels.cu:23-149), with variant 1 N-PMCHWT
 *         surface form (dielectric_kernels.cu:155-318: nTL/nTK in the places
 *         of TL/TK), variant 2 N-Muller surface form (dielectric_kernels.cu:323-489),
 * kind 2: GSTC Calderon + mass, eta0-scaled (sie_kernels_assembly.cuh:156-272,
 *         460-594). Z: complex interleaved, column-major, overwritten.
 * Serial over faces so that the summation order is fixed. */
static int assemble_impl(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
                         float k1, float k2, float mu_r1, float mu_r2, float eps_r1, float eps_r2,
                         float mu0, float eps0, float omega, float thr, const double* tensors,
                         int tensors_uniform, int basis, const ztarget_t* Zt, const int* test_faces, int ntest,
                         int threads, int variant, int line_points) {
    float pts[2 * 80], wts[80];
    const int Q = so_rule(rule, pts, wts);
    if (Q < 0) return -1;
    float lt[20], lw[20];
    /* N-MFIE evaluates no line integral (pec_solver.cu:215-218). */
    const int NG = (variant == 1 || (variant == 2 && kind == 1)) && line_points > 0
                       ? so_gauss_legendre(line_points, lt, lw) : 0;
    if (NG < 0) return -1;
    const line_t L = {lt, lw, NG};
    const size_t E = (size_t)ne;
    const size_t N = kind == 0 ? E : (kind == 1 ? 2 * E : 4 * E);
    ztarget_t Zv = *Zt;
    ztarget_t* Z = &Zv;
    tri_t* tris = (tri_t*)malloc(sizeof(tri_t) * (size_t)nf);
    for (int f = 0; f < nf; ++f) load_tri(V, F, f, &tris[f]);
    if (threads <= 0) threads = omp_get_max_threads();

    /* Face-pair blocks of a chunk of test faces in parallel, then placed
     * serially in (test face, source face) order: the sums are the same,
     * bit for bit, for any thread count. */
    const int CH = 32;
    blocks_t* buf = (blocks_t*)malloc(sizeof(blocks_t) * (size_t)CH * (size_t)nf);
    for (int c0 = 0; c0 < ntest; c0 += CH) {
        const int cn = ntest - c0 < CH ? ntest - c0 : CH;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
        for (long idx = 0; idx < (long)cn * nf; ++idx) {
            const int mm = test_faces ? test_faces[c0 + idx / nf] : c0 + (int)(idx / nf);
            const int nn = (int)(idx % nf);
            if (variant != 0)
                pair_n(&tris[mm], &tris[nn], pts, wts, Q, &L, k1, k2, thr, kind == 0, &buf[idx]);
            else
                pair(&tris[mm], &tris[nn], pts, wts, Q, k1, k2, thr, &buf[idx]);
        }
      for (int ci = 0; ci < cn; ++ci) {
        const int m = test_faces ? test_faces[c0 + ci] : c0 + ci;
        for (int n = 0; n < nf; ++n) {
            const blocks_t B = buf[(size_t)ci * nf + n];
            const int* te = &FE[3 * m];
            const int* se = &FE[3 * n];
            double G[3][3];
            if (variant == 2 && m == n) gram(&tris[m], pts, wts, Q, G);
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    const size_t r = te[j], c = se[i];
                    if (kind == 0 && variant == 2) {
                        /* pec_solver.cu:171-240: 1/2 Gram on the same face,
                         * -nTK2 on the others (its self nTK is zero). */
                        if (m == n)
                            zadd(Z, N, r, c, CX(G[j][i] * 0.5, 0.0));
                        else
                            zadd(Z, N, r, c, cscale(B.tk2[j][i], -1.0));
                    } else if (kind == 1 && variant == 2) {
                        /* dielectric_kernels.cu:433-488 (N-Muller). */
                        const float m1 = mu_r1 * mu0, m2 = mu_r2 * mu0;
                        const float e1 = eps_r1 * eps0, e2 = eps_r2 * eps0;
                        const float eta0 = sqrtf(mu0 / eps0);
                        const cx w1 = CX(0.0, ((double)omega * e1) * m1);
                        const cx w2 = CX(0.0, ((double)omega * e2) * m2);
                        cx zjj = csub(cmul(w2, B.tl2[j][i]), cmul(w1, B.tl1[j][i]));
                        cx zmm = cscale(zjj, -1.0);
                        cx zjm = csub(cscale(B.tk2[j][i], (double)e2), cscale(B.tk1[j][i], (double)e1));
                        cx zmj = csub(cscale(B.tk2[j][i], (double)m2), cscale(B.tk1[j][i], (double)m1));
                        if (m == n) {
                            const float ef = (e1 + e2) / 2.0f, mf = (m1 + m2) / 2.0f;
                            zjm = csub(zjm, CX((double)ef * G[j][i], 0.0));
                            zmj = csub(zmj, CX((double)mf * G[j][i], 0.0));
                        }
                        const float eta0sq = eta0 * eta0;
                        zadd(Z, N, r, c, zjj);
                        zadd(Z, N, r, c + E, cscale(zjm, (double)eta0));
                        zadd(Z, N, r + E, c, cscale(zmj, (double)eta0));
                        zadd(Z, N, r + E, c + E, cscale(zmm, (double)eta0sq));
                    } else if (kind == 0 && variant == 1) {
                        /* pec_solver.cu:163-167: j (omega * mu2) nTL2, mu2 rounded
                         * to float from its double product. */
                        const float ce = omega * (float)((double)mu_r2 * (double)mu0);
                        zadd(Z, N, r, c, cmul(CX(0.0, (double)ce), B.tl2[j][i]));
                    } else if (kind == 0) {
                        const float ce = omega * mu_r2 * mu0;
                        zadd(Z, N, r, c, cmul(CX(0.0, (double)ce), B.tl2[j][i]));
                    } else if (kind == 1) {
                        const float m1 = mu_r1 * mu0, m2 = mu_r2 * mu0;
                        const float e1 = eps_r1 * eps0, e2 = eps_r2 * eps0;
                        const float eta0 = sqrtf(mu0 / eps0);
                        const cx cm1 = CX(0.0 * m1, (double)omega * m1);
                        const cx cm2 = CX(0.0 * m2, (double)omega * m2);
                        const cx ce1 = CX(0.0 * e1, (double)omega * e1);
                        const cx ce2 = CX(0.0 * e2, (double)omega * e2);
                        const cx tk = cadd(B.tk1[j][i], B.tk2[j][i]);
                        const cx zjj = cadd(cmul(cm1, B.tl1[j][i]), cmul(cm2, B.tl2[j][i]));
                        const cx zmm = cadd(cmul(ce1, B.tl1[j][i]), cmul(ce2, B.tl2[j][i]));
                        const float eta0sq = eta0 * eta0;
                        zadd(Z, N, r, c, zjj);
                        zadd(Z, N, r, c + E, cscale(tk, (double)eta0));
                        zadd(Z, N, r + E, c, cscale(cscale(tk, -1.0), (double)eta0));
                        zadd(Z, N, r + E, c + E, cscale(zmm, (double)eta0sq));
                    } else {
                        /* sie_scaling.cuh:48-77; sie_kernels_assembly.cuh:225 forms
                         * eta0 = sqrt(mu0 / eps0) from float arguments, which nvcc
                         * evaluates with the float overload of sqrt. */
                        const double eta0 = (double)sqrtf(mu0 / eps0);
                        for (int reg = 0; reg < 2; ++reg) {
                            const double mu = (double)(reg == 0 ? mu_r1 * mu0 : mu_r2 * mu0);
                            const double ep = (double)(reg == 0 ? eps_r1 * eps0 : eps_r2 * eps0);
                            const cx jw = CX(0.0, (double)omega);
                            const cx fjj = cscale(jw, mu);
                            const cx fmm = cscale(jw, eta0 * eta0 * ep);
                            const cx tl = reg == 0 ? B.tl1[j][i] : B.tl2[j][i];
                            const cx tk = reg == 0 ? B.tk1[j][i] : B.tk2[j][i];
                            const cx jm = cscale(tk, eta0);
                            const size_t o = reg == 0 ? 0 : 2 * E;
                            zadd(Z, N, r + o, c + o, cmul(fjj, tl));
                            zadd(Z, N, r + o, c + o + E, jm);
                            zadd(Z, N, r + o + E, c + o, CX(-jm.re, -jm.im));
                            zadd(Z, N, r + o + E, c + o + E, cmul(fmm, tl));
                        }
                    }
                }
        }
      }
    }
    free(buf);

    if (kind == 2) {
        const float eta0 = sqrtf(mu0 / eps0);
        const float eta0sq = eta0 * eta0;
        for (int ti = 0; ti < ntest; ++ti) {
            const int m = test_faces ? test_faces[ti] : ti;
            const tri_t* T = &tris[m];
            v3 u, w;
            frame(T->v, basis, &u, &w);
            const double* tp = tensors_uniform ? tensors : tensors + (size_t)m * 64;
#define AT(M4, r, c) CX((M4)[2 * ((r) * 4 + (c))], (M4)[2 * ((r) * 4 + (c)) + 1])
            cx Y[4][3][3], Zt[4][3][3], Tt[8][3][3], R[8][3][3];
            for (int blk = 0; blk < 4; ++blk) {
                int r0 = (blk / 2) * 2, c0 = (blk % 2) * 2;
                lift(AT(tp, r0, c0), AT(tp, r0, c0 + 1), AT(tp, r0 + 1, c0), AT(tp, r0 + 1, c0 + 1), u, w, Y[blk]);
                lift(AT(tp + 32, r0, c0), AT(tp + 32, r0, c0 + 1), AT(tp + 32, r0 + 1, c0),
                     AT(tp + 32, r0 + 1, c0 + 1), u, w, Zt[blk]);
            }
#undef AT
            v3 nv = vnorm(vcross(vsub(T->v[1], T->v[0]), vsub(T->v[2], T->v[0])));
            for (int k = 0; k < 4; ++k) perp(Y[k], nv, Tt[k]);
            for (int k = 0; k < 4; ++k) memcpy(Tt[4 + k], Zt[k], sizeof(cx) * 9);
            mass8(T, pts, wts, Q, Tt, R);
            const int* le = &FE[3 * m];
            const double f = 0.5, fq = 0.125;
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    const size_t r = le[j], c = le[i];
                    const cx Zee = R[4][j][i], Zem = R[5][j][i], Zme = R[6][j][i], Zmm = R[7][j][i];
                    const cx Yee = R[0][j][i], Yem = R[1][j][i], Yme = R[2][j][i], Ymm = R[3][j][i];
                    const cx a_p = cadd(cscale(Zee, f), cscale(Ymm, fq)), a_m = csub(cscale(Zee, f), cscale(Ymm, fq));
                    const cx b_p = cadd(cscale(Zem, f), cscale(Yme, fq)), b_m = csub(cscale(Zem, f), cscale(Yme, fq));
                    const cx c_p = cadd(cscale(Zme, f), cscale(Yem, fq)), c_m = csub(cscale(Zme, f), cscale(Yem, fq));
                    const cx d_p = cadd(cscale(Zmm, f), cscale(Yee, fq)), d_m = csub(cscale(Zmm, f), cscale(Yee, fq));
                    const double s1 = 1.0, se = (double)eta0, s2 = (double)eta0sq;
                    zadd(Z, N, r, c, cscale(a_p, s1));
                    zadd(Z, N, r, c + E, cscale(b_m, se));
                    zadd(Z, N, r, c + 2 * E, cscale(a_m, s1));
                    zadd(Z, N, r, c + 3 * E, cscale(b_p, se));
                    zadd(Z, N, r + E, c, cscale(c_m, se));
                    zadd(Z, N, r + E, c + E, cscale(d_p, s2));
                    zadd(Z, N, r + E, c + 2 * E, cscale(c_p, se));
                    zadd(Z, N, r + E, c + 3 * E, cscale(d_m, s2));
                    zadd(Z, N, r + 2 * E, c, cscale(a_m, s1));
                    zadd(Z, N, r + 2 * E, c + E, cscale(b_p, se));
                    zadd(Z, N, r + 2 * E, c + 2 * E, cscale(a_p, s1));
                    zadd(Z, N, r + 2 * E, c + 3 * E, cscale(b_m, se));
                    zadd(Z, N, r + 3 * E, c, cscale(c_p, se));
                    zadd(Z, N, r + 3 * E, c + E, cscale(d_m, s2));
                    zadd(Z, N, r + 3 * E, c + 2 * E, cscale(c_m, se));
                    zadd(Z, N, r + 3 * E, c + 3 * E, cscale(d_p, s2));
                }
        }
    }
    free(tris);
    return 0;
}

int so_assemble(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
                float k1, float k2, float mu_r1, float mu_r2, float eps_r1, float eps_r2,
                float mu0, float eps0, float omega, float thr, const double* tensors,
                int tensors_uniform, int basis, double* Z, int threads, int variant, int line_points) {
    const size_t E = (size_t)ne;
    const size_t N = kind == 0 ? E : (kind == 1 ? 2 * E : 4 * E);
    memset(Z, 0, sizeof(double) * 2 * N * N);
    const ztarget_t T = {Z, N, NULL};
    return assemble_impl(kind, V, F, FE, nf, ne, rule, k1, k2, mu_r1, mu_r2, eps_r1, eps_r2, mu0, eps0, omega,
                         thr, tensors, tensors_uniform, basis, &T, NULL, nf, threads, variant, line_points);
}

/* The contributions of the listed test faces only, into the rows that
 * rowmap selects (rowmap[r] = output row or -1; Zrows: nrows x N,
 * column-major, overwritten). A row of Z is complete when every face that
 * holds its edge is listed. */
int so_assemble_rows(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
                     float k1, float k2, float mu_r1, float mu_r2, float eps_r1, float eps_r2,
                     float mu0, float eps0, float omega, float thr, const double* tensors,
                     int tensors_uniform, int basis, const int* test_faces, int ntest, const int* rowmap,
                     int nrows, double* Zrows, int threads, int variant, int line_points) {
    const size_t E = (size_t)ne;
    const size_t N = kind == 0 ? E : (kind == 1 ? 2 * E : 4 * E);
    memset(Zrows, 0, sizeof(double) * 2 * (size_t)nrows * N);
    const ztarget_t T = {Zrows, (size_t)nrows, rowmap};
    return assemble_impl(kind, V, F, FE, nf, ne, rule, k1, k2, mu_r1, mu_r2, eps_r1, eps_r2, mu0, eps0, omega,
                         thr, tensors, tensors_uniform, basis, &T, test_faces, ntest, threads, variant,
                         line_points);
}

/* ----------------------------------------------------------------- RHS -- */
/* source_functors.cuh:14-42 (plane wave) and 51-130 (dipole). */
static void source_fields(int kind, v3 r, const double* a, const double* b, int is_mag, double k,
                          double eta, cx E[3], cx H[3]) {
    if (kind == 0) {
        v3 E0 = V3(a[0], a[1], a[2]), kh = V3(b[0], b[1], b[2]);
        double kdr = vdot(kh, r) * k;
        cx ph = CX(cos(-kdr), sin(-kdr));
        E[0] = cscale(ph, E0.x); E[1] = cscale(ph, E0.y); E[2] = cscale(ph, E0.z);
        /* H = (k_hat x E) / eta */
        cx kx = csub(cscale(E[2], kh.y), cscale(E[1], kh.z));
        cx ky = csub(cscale(E[0], kh.z), cscale(E[2], kh.x));
        cx kz = csub(cscale(E[1], kh.x), cscale(E[0], kh.y));
        double ie = 1.0 / eta;
        H[0] = cscale(kx, ie); H[1] = cscale(ky, ie); H[2] = cscale(kz, ie);
        return;
    }
    v3 p = V3(a[0], a[1], a[2]), r0 = V3(b[0], b[1], b[2]);
    v3 Rv = vsub(r, r0);
    double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
    if (R < 1e-6) { memset(E, 0, sizeof(cx) * 3); memset(H, 0, sizeof(cx) * 3); return; }
    v3 Rh = V3(Rv.x / R, Rv.y / R, Rv.z / R);
    double Rdp = Rh.x * p.x + Rh.y * p.y + Rh.z * p.z;
    v3 Rxp = V3(Rh.y * p.z - Rh.z * p.y, Rh.z * p.x - Rh.x * p.z, Rh.x * p.y - Rh.y * p.x);
    v3 tri = V3(Rxp.y * Rh.z - Rxp.z * Rh.y, Rxp.z * Rh.x - Rxp.x * Rh.z, Rxp.x * Rh.y - Rxp.y * Rh.x);
    cx ph = CX(cos(-k * R), sin(-k * R));
    double t1 = (k * k) / R, t2r = 1.0 / (R * R * R), t2i = k / (R * R);
    double tv[3] = {3.0 * Rh.x * Rdp - p.x, 3.0 * Rh.y * Rdp - p.y, 3.0 * Rh.z * Rdp - p.z};
    double trc[3] = {tri.x, tri.y, tri.z};
    cx Ec[3], Hc[3];
    for (int c = 0; c < 3; ++c) Ec[c] = cmul(CX(t1 * trc[c] + tv[c] * t2r, tv[c] * t2i), ph);
    cx hc = cmul(CX(-(k * k) / (eta * R), k / (eta * R * R)), ph);
    double rxp[3] = {Rxp.x, Rxp.y, Rxp.z};
    for (int c = 0; c < 3; ++c) Hc[c] = CX(hc.re * -rxp[c], hc.im * -rxp[c]);
    if (is_mag) {
        for (int c = 0; c < 3; ++c) {
            E[c] = CX(Hc[c].re * -eta, Hc[c].im * -eta);
            H[c] = CX(Ec[c].re / eta, Ec[c].im / eta);
        }
    } else {
        for (int c = 0; c < 3; ++c) { E[c] = Ec[c]; H[c] = Hc[c]; }
    }
}

/* compute_incident_field_kernel (src/sie_mom/excitation/excitation.cu:140-156):
 * the source functors at n points; E, H complex interleaved, 3 per point.
 * b is the unit propagation direction of a plane wave. */
int so_incident_fields(int source_kind, const double* a, const double* b, int is_magnetic, double k, double eta,
                       int n, const double* pts, double* E, double* H) {
    for (int i = 0; i < n; ++i) {
        cx Ei[3], Hi[3];
        source_fields(source_kind, V3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), a, b, is_magnetic, k, eta, Ei, Hi);
        for (int c = 0; c < 3; ++c) {
            E[2 * (3 * i + c)] = Ei[c].re; E[2 * (3 * i + c) + 1] = Ei[c].im;
            H[2 * (3 * i + c)] = Hi[c].re; H[2 * (3 * i + c) + 1] = Hi[c].im;
        }
    }
    return 0;
}

/* dunavant_quadrature.cuh:1543-1611 (RWG testing; variant != 0: n x RWG
 * testing, rho x n_m; variant 2: N-MFIE tests H, N-Muller scales by the
 * source region's eps_r_src, mu_r_src) with the placements of
 * pec_solver.cu:242-264 (kind 0), dielectric_solver.cu:399-530 (kind 1) and
 * sie_kernels_utils.cuh:184-232 (kind 2). source_kind 0: plane wave (a = E0,
 * b = k_hat), 1: dipole (a = moment, b = position). */
int so_rhs(int kind, int source_kind, const double* V, const int* F, const int* FE, int nf, int ne,
           int rule, const double* a, const double* b, int is_magnetic, double k, double eta,
           int region, double mu0, double eps0, double* rhs, int variant, double eps_r_src,
           double mu_r_src) {
    const int rotated = variant != 0;
    float pts[2 * 80], wts[80];
    const int Q = so_rule(rule, pts, wts);
    if (Q < 0) return -1;
    const size_t E = (size_t)ne;
    const size_t N = kind == 0 ? E : (kind == 1 ? 2 * E : 4 * E);
    memset(rhs, 0, sizeof(double) * 2 * N);
    for (int m = 0; m < nf; ++m) {
        tri_t T;
        load_tri(V, F, m, &T);
        float el[3];
        for (int i = 0; i < 3; ++i) el[i] = (float)T.len[i];
        cx ve[3] = {{0, 0}, {0, 0}, {0, 0}}, vh[3] = {{0, 0}, {0, 0}, {0, 0}};
        const v3 nm = face_normal(&T);
        for (int p = 0; p < Q; ++p) {
            const float wp = wts[p];
            v3 rp = map_point(&T, (double)pts[2 * p], (double)pts[2 * p + 1]);
            cx Ei[3], Hi[3];
            source_fields(source_kind, rp, a, b, is_magnetic, k, eta, Ei, Hi);
            for (int i = 0; i < 3; ++i) {
                v3 t = vsub(rp, T.free_v[i]);
                if (rotated) t = vcross(t, nm);
                cx de = CX(t.x * Ei[0].re + t.y * Ei[1].re + t.z * Ei[2].re,
                           t.x * Ei[0].im + t.y * Ei[1].im + t.z * Ei[2].im);
                cx dh = CX(t.x * Hi[0].re + t.y * Hi[1].re + t.z * Hi[2].re,
                           t.x * Hi[0].im + t.y * Hi[1].im + t.z * Hi[2].im);
                ve[i] = cadd(ve[i], cscale(de, (double)wp));
                vh[i] = cadd(vh[i], cscale(dh, (double)wp));
            }
        }
        for (int i = 0; i < 3; ++i) {
            const float s = 0.5f * el[i];
            ve[i] = cscale(ve[i], (double)s);
            vh[i] = cscale(vh[i], (double)s);
            const size_t e = (size_t)FE[3 * m + i];
            if (kind == 0 && variant == 2) {
                rhs[2 * e] += vh[i].re; rhs[2 * e + 1] += vh[i].im;
            } else if (kind == 0) {
                rhs[2 * e] += ve[i].re; rhs[2 * e + 1] += ve[i].im;
            } else if (kind == 1 && variant == 2) {
                /* dielectric_solver.cu:461-489: eps V_E, -mu eta0 V_H of the
                 * source region. */
                const double eta0 = sqrt(mu0 / eps0);
                const double sE = eps_r_src * eps0, sH = -(mu_r_src * mu0) * eta0;
                cx a1 = cscale(ve[i], sE), a2 = cscale(vh[i], sH);
                rhs[2 * e] += a1.re; rhs[2 * e + 1] += a1.im;
                rhs[2 * (e + E)] += a2.re; rhs[2 * (e + E) + 1] += a2.im;
            } else if (kind == 1) {
                const double eta0 = sqrt(mu0 / eps0);
                const double sg = region == 2 ? 1.0 : -1.0;
                cx a1 = cscale(ve[i], sg), a2 = cscale(vh[i], sg * eta0);
                rhs[2 * e] += a1.re; rhs[2 * e + 1] += a1.im;
                rhs[2 * (e + E)] += a2.re; rhs[2 * (e + E) + 1] += a2.im;
            } else {
                const double eta0 = sqrt((double)(float)mu0 / (double)(float)eps0);
                const size_t off = region == 1 ? 0 : 2 * E;
                cx a2 = cscale(vh[i], eta0);
                rhs[2 * (e + off)] += ve[i].re; rhs[2 * (e + off) + 1] += ve[i].im;
                rhs[2 * (e + off + E)] += a2.re; rhs[2 * (e + off + E) + 1] += a2.im;
            }
        }
    }
    return 0;
}

/* ----------------------------------------------------------- far field -- */
/* applications/anisotropic_gstc_sphere/plot_far_field.py:88-220: Schelkunoff
 * radiation vectors from RWG currents at the script's 7-point rule, evaluated
 * in double, directions given as unit-vector triples. j_cur/m_cur are the
 * exterior-oriented coefficient vectors (complex interleaved, length ne);
 * m_cur may be NULL (PEC). */
int so_far_field(const double* V, const int* F, int nf, int ne, const double* j_cur,
                 const double* m_cur, double k0, double eta0, int ndir, const double* r_hat,
                 const double* theta_hat, const double* phi_hat, double* f_theta, double* f_phi,
                 double* intensity) {
    int* FE = (int*)malloc(sizeof(int) * 3 * (size_t)nf);
    int ne_chk = so_build_edges(F, nf, NULL, FE);
    if (ne_chk != ne) { free(FE); return -1; }
    const double s15 = sqrt(15.0);
    const double a1 = (6.0 - s15) / 21.0, w1 = (155.0 - s15) / 1200.0;
    const double a2 = (6.0 + s15) / 21.0, w2 = (155.0 + s15) / 1200.0;
    const double nodes[7][2] = {{1.0 / 3.0, 1.0 / 3.0}, {a1, a1}, {1.0 - 2.0 * a1, a1}, {a1, 1.0 - 2.0 * a1},
                                {a2, a2}, {1.0 - 2.0 * a2, a2}, {a2, 1.0 - 2.0 * a2}};
    const double wq[7] = {0.225, w1, w1, w1, w2, w2, w2};
    const size_t M = (size_t)nf * 7;
    v3* rq = (v3*)malloc(sizeof(v3) * M);
    cx* cj = (cx*)calloc(M * 3, sizeof(cx));
    cx* cm = (cx*)calloc(M * 3, sizeof(cx));
    for (int f = 0; f < nf; ++f) {
        tri_t T;
        load_tri(V, F, f, &T);
        for (int q = 0; q < 7; ++q) {
            double xi = nodes[q][0], eta = nodes[q][1], zeta = 1.0 - xi - eta;
            rq[f * 7 + q] = vadd(vadd(vscale(T.v[0], zeta), vscale(T.v[1], xi)), vscale(T.v[2], eta));
        }
        for (int le = 0; le < 3; ++le) {
            int e = FE[3 * f + le];
            cx je = CX(j_cur[2 * e], j_cur[2 * e + 1]);
            cx me = m_cur ? CX(m_cur[2 * e], m_cur[2 * e + 1]) : CX(0, 0);
            cx coj = cscale(je, 0.5 * T.len[le]);
            cx com = cscale(me, 0.5 * T.len[le]);
            for (int q = 0; q < 7; ++q) {
                v3 rho = vsub(rq[f * 7 + q], T.free_v[le]);
                double rr[3] = {rho.x, rho.y, rho.z};
                for (int c = 0; c < 3; ++c) {
                    cj[(f * 7 + q) * 3 + c] = cadd(cj[(f * 7 + q) * 3 + c], cscale(coj, wq[q] * rr[c]));
                    cm[(f * 7 + q) * 3 + c] = cadd(cm[(f * 7 + q) * 3 + c], cscale(com, wq[q] * rr[c]));
                }
            }
        }
    }
    for (int d = 0; d < ndir; ++d) {
        v3 rh = V3(r_hat[3 * d], r_hat[3 * d + 1], r_hat[3 * d + 2]);
        cx Nv[3] = {{0, 0}, {0, 0}, {0, 0}}, Lv[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (size_t i = 0; i < M; ++i) {
            double ph = k0 * vdot(rh, rq[i]);
            cx e = CX(cos(ph), sin(ph));
            for (int c = 0; c < 3; ++c) {
                Nv[c] = cadd(Nv[c], cmul(e, cj[i * 3 + c]));
                Lv[c] = cadd(Lv[c], cmul(e, cm[i * 3 + c]));
            }
        }
        const double* th = &theta_hat[3 * d];
        const double* pp = &phi_hat[3 * d];
        cx nt = CX(0, 0), np_ = CX(0, 0), lt = CX(0, 0), lp = CX(0, 0);
        for (int c = 0; c < 3; ++c) {
            nt = cadd(nt, cscale(Nv[c], th[c]));
            np_ = cadd(np_, cscale(Nv[c], pp[c]));
            lt = cadd(lt, cscale(Lv[c], th[c]));
            lp = cadd(lp, cscale(Lv[c], pp[c]));
        }
        cx coeff = CX(0.0, -k0 / (4.0 * M_PI));
        cx ft = cmul(coeff, cadd(cscale(nt, eta0), lp));
        cx fp = cmul(coeff, csub(cscale(np_, eta0), lt));
        f_theta[2 * d] = ft.re; f_theta[2 * d + 1] = ft.im;
        f_phi[2 * d] = fp.re; f_phi[2 * d + 1] = fp.im;
        intensity[d] = (ft.re * ft.re + ft.im * ft.im + fp.re * fp.re + fp.im * fp.im) / (2.0 * eta0);
    }
    free(FE); free(rq); free(cj); free(cm);
    return 0;
}

/* ---------------------------------------- surface-integral field values -- */
/* green_functions_utils.cuh:142-221: G and grad G of the field evaluation,
 * standard (R < 1e-12 -> 0) or with the static and k^2 terms extracted
 * (R < 1e-6 -> G = -jk/(4 pi), grad G = 0). */
static void green_grad(v3 r1, v3 r2, double k, int regular, cx* G, cx g[3]) {
    v3 Rv = vsub(r1, r2);
    double R = sqrt(Rv.x * Rv.x + Rv.y * Rv.y + Rv.z * Rv.z);
    if (!regular) {
        if (R < 1e-12) {
            *G = CX(0.0, 0.0);
            g[0] = g[1] = g[2] = CX(0.0, 0.0);
            return;
        }
        double inv_R = 1.0 / R;
        v3 Rh = V3(Rv.x * inv_R, Rv.y * inv_R, Rv.z * inv_R);
        double i4pR = 1.0 / (4.0 * M_PI * R);
        double s = sin(k * R), c = cos(k * R);
        *G = CX(c * i4pR, -s * i4pR);
        cx wg = cmul(CX(inv_R, k), *G);
        g[0] = cscale(wg, Rh.x);
        g[1] = cscale(wg, Rh.y);
        g[2] = cscale(wg, Rh.z);
    } else {
        if (R < 1e-6) {
            *G = CX(0.0, -k / (4.0 * M_PI));
            g[0] = g[1] = g[2] = CX(0.0, 0.0);
            return;
        }
        double i4p = 1.0 / (4.0 * M_PI);
        double inv_R = 1.0 / R, inv_R2 = inv_R * inv_R, inv_R3 = inv_R2 * inv_R;
        double i4pR = i4p * inv_R;
        double s = sin(k * R), c = cos(k * R);
        *G = CX((c - 1.0) * i4pR, -s * i4pR);
        cx Kr = cmul(CX(inv_R3, k * inv_R2), CX(c, -s));
        Kr.re += -(inv_R3 + k * k * 0.5 * inv_R);
        cx sc = cscale(Kr, i4p);
        g[0] = cscale(sc, Rv.x);
        g[1] = cscale(sc, Rv.y);
        g[2] = cscale(sc, Rv.z);
    }
}

/* dunavant_quadrature.cuh:1634-1705: L and K integrals of the three half-RWG
 * functions of source triangle S at obs (k arrives as float; 1/k^2 and the
 * edge lengths are float). */
static void field_quad(v3 obs, const tri_t* S, const float* pts, const float* wts, int Q, float k,
                       int regular, cx L[3][3], cx K[3][3]) {
    memset(L, 0, sizeof(cx) * 9);
    memset(K, 0, sizeof(cx) * 9);
    const float k_sq_inv = 1.f / (k * k);
    for (int q = 0; q < Q; ++q) {
        v3 rq = map_point(S, (double)pts[2 * q], (double)pts[2 * q + 1]);
        const double w = (double)wts[q];
        cx G, g[3];
        green_grad(obs, rq, (double)k, regular, &G, g);
        for (int i = 0; i < 3; ++i) {
            v3 rho = vsub(rq, S->free_v[i]);
            const double rc[3] = {rho.x, rho.y, rho.z};
            for (int c = 0; c < 3; ++c) {
                cx l1 = cscale(cscale(G, rc[c]), 0.5);
                cx l2 = cscale(g[c], (double)(-k_sq_inv));
                L[i][c] = cadd(L[i][c], cscale(cadd(l1, l2), w));
            }
            cx cr[3];
            cr[0] = csub(cscale(g[2], rho.y), cscale(g[1], rho.z));
            cr[1] = csub(cscale(g[0], rho.z), cscale(g[2], rho.x));
            cr[2] = csub(cscale(g[1], rho.x), cscale(g[0], rho.y));
            for (int c = 0; c < 3; ++c) K[i][c] = cadd(K[i][c], cscale(cscale(cr[c], 0.5), w));
        }
    }
    for (int i = 0; i < 3; ++i) {
        const double el = (double)(float)S->len[i];
        for (int c = 0; c < 3; ++c) {
            L[i][c] = cscale(L[i][c], el);
            K[i][c] = cscale(K[i][c], el);
        }
    }
}

/* dunavant_quadrature.cuh:1719-1770: the analytic (Wilton) parts that the
 * extracted quadrature leaves out; real-valued, scaled by l_i / (8 pi A) in
 * float. */
static void field_singular(v3 obs, const tri_t* S, float k, cx L[3][3], cx K[3][3]) {
    const float A = (float)(0.5f * vlen(vcross(vsub(S->v[1], S->v[0]), vsub(S->v[2], S->v[0]))));
    const float base_scale = 1.0f / (8.0f * (float)M_PI * A);
    pots_t P = wilton(obs, S->v);
    const float k_sq_inv = 1.f / (k * k);
    for (int i = 0; i < 3; ++i) {
        v3 fv = S->free_v[i];
        v3 Rf = vsub(obs, fv);
        v3 ps = psi1(&P, fv);
        v3 phi3 = vadd(P.phi3b, vscale(vsub(P.r_pi, fv), P.phi2));
        v3 Lin = vadd(vsub(ps, vscale(vscale(Rf, 0.5), P.phi0)),
                      vscale(vsub(phi3, vscale(Rf, P.phi2)), (double)k_sq_inv));
        v3 Kv = upsilon(&P, fv, obs, k);
        const float l_scale = (float)S->len[i] * base_scale;
        v3 Lv = vscale(Lin, 2.0);
        L[i][0] = CX(Lv.x * l_scale, 0.0); L[i][1] = CX(Lv.y * l_scale, 0.0); L[i][2] = CX(Lv.z * l_scale, 0.0);
        K[i][0] = CX(Kv.x * l_scale, 0.0); K[i][1] = CX(Kv.y * l_scale, 0.0); K[i][2] = CX(Kv.z * l_scale, 0.0);
    }
}

/* surface_current_fields.cu:96-112 and sie_kernels_utils.cuh:21-140: the
 * positive surface-integral terms Q_E = j w mu L[J] + K[M] and
 * Q_H = -K[J] + j w eps L[M] at each observation point, every face by
 * ordinary quadrature, or by extracted quadrature plus the Wilton part when
 * its centroid is within 0.1 lambda (float distance and threshold). J, M:
 * physical coefficients per edge (complex interleaved). E, H out: nobs x 3
 * complex interleaved. */
int so_surface_fields(const double* V, const int* F, const int* FE, int nf, int ne, const double* J,
                      const double* M, int nobs, const double* obs, double freq, double eps_r, double mu_r,
                      double eps0, double mu0, int rule, double* E, double* H) {
    float pts[2 * 100], wts[100];
    const int Q = so_rule(rule, pts, wts);
    if (Q <= 0) return -1;
    (void)ne;
    const double omega = 2.0 * M_PI * freq;
    const double eps = eps_r * eps0, mu = mu_r * mu0;
    const double k = omega * sqrt(mu * eps);
    const cx cJ = CX(0.0, omega * mu), cM = CX(1.0, 0.0), cJh = CX(-1.0, 0.0), cMh = CX(0.0, omega * eps);
    const float lambda = (float)((double)(2.0f * (float)M_PI) / k);
    const float thr = 0.1f * lambda;
    const float kf = (float)k;
    for (int p = 0; p < nobs; ++p) {
        v3 r = V3(obs[3 * p], obs[3 * p + 1], obs[3 * p + 2]);
        cx e[3] = {{0, 0}, {0, 0}, {0, 0}}, h[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (int f = 0; f < nf; ++f) {
            tri_t S;
            load_tri(V, F, f, &S);
            const v3 c = V3((S.v[0].x + S.v[1].x + S.v[2].x) / 3.0, (S.v[0].y + S.v[1].y + S.v[2].y) / 3.0,
                            (S.v[0].z + S.v[1].z + S.v[2].z) / 3.0);
            const float dist = (float)vlen(vsub(r, c));
            cx L[3][3], K[3][3];
            if (dist < thr) {
                cx Ls[3][3], Ks[3][3];
                field_quad(r, &S, pts, wts, Q, kf, 1, L, K);
                field_singular(r, &S, kf, Ls, Ks);
                for (int i = 0; i < 3; ++i)
                    for (int d = 0; d < 3; ++d) {
                        L[i][d] = cadd(L[i][d], Ls[i][d]);
                        K[i][d] = cadd(K[i][d], Ks[i][d]);
                    }
            } else {
                field_quad(r, &S, pts, wts, Q, kf, 0, L, K);
            }
            for (int i = 0; i < 3; ++i) {
                const int ed = FE[3 * f + i];
                const cx je = CX(J[2 * ed], J[2 * ed + 1]);
                const cx me = M ? CX(M[2 * ed], M[2 * ed + 1]) : CX(0.0, 0.0);
                const cx wEJ = cmul(cJ, je), wEM = cmul(cM, me), wHJ = cmul(cJh, je), wHM = cmul(cMh, me);
                for (int d = 0; d < 3; ++d) {
                    e[d] = cadd(e[d], cmul(wEJ, L[i][d]));
                    e[d] = cadd(e[d], cmul(wEM, K[i][d]));
                    h[d] = cadd(h[d], cmul(wHJ, K[i][d]));
                    h[d] = cadd(h[d], cmul(wHM, L[i][d]));
                }
            }
        }
        for (int d = 0; d < 3; ++d) {
            E[6 * p + 2 * d] = e[d].re; E[6 * p + 2 * d + 1] = e[d].im;
            H[6 * p + 2 * d] = h[d].re; H[6 * p + 2 * d + 1] = h[d].im;
        }
    }
    return 0;
}
