/* Test infrastructure only: CPU restatement of the dense MoM hot path of the
 * SIE-GSTC solver (see sieoracle.c). Only tests/, the smoke check and the
 * CPU-baseline leg of bench.py may load it; the product never does. */
#ifndef SIEORACLE_H
#define SIEORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

int so_rule(int rule, float* pts, float* w);
int so_build_edges(const int* faces, int nf, int* edges, int* faces_edges);
void so_wilton(const double* r, const double* tri, double* out);
void so_pair_blocks(const double* V, const int* F, int m, int n, int rule, float k1, float k2,
                    float thr, double* out);
void so_pair_blocks_n(const double* V, const int* F, int m, int n, int rule, float k1, float k2,
                      float thr, int line_points, double* out);
int so_gauss_legendre(int n, float* t, float* w);
int so_assemble(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
                float k1, float k2, float mu_r1, float mu_r2, float eps_r1, float eps_r2,
                float mu0, float eps0, float omega, float thr, const double* tensors,
                int tensors_uniform, int basis, double* Z, int threads, int variant, int line_points);
int so_assemble_rows(int kind, const double* V, const int* F, const int* FE, int nf, int ne, int rule,
                float k1, float k2, float mu_r1, float mu_r2, float eps_r1, float eps_r2,
                float mu0, float eps0, float omega, float thr, const double* tensors,
                int tensors_uniform, int basis, const int* test_faces, int ntest, const int* rowmap,
                     int nrows, double* Zrows, int threads, int variant, int line_points);
int so_rhs(int kind, int source_kind, const double* V, const int* F, const int* FE, int nf, int ne,
           int rule, const double* a, const double* b, int is_magnetic, double k, double eta,
           int region, double mu0, double eps0, double* rhs, int variant, double eps_r_src,
           double mu_r_src);
int so_incident_fields(int source_kind, const double* a, const double* b, int is_magnetic, double k, double eta,
                       int n, const double* pts, double* E, double* H);
int so_far_field(const double* V, const int* F, int nf, int ne, const double* j_cur,
                 const double* m_cur, double k0, double eta0, int ndir, const double* r_hat,
                 const double* theta_hat, const double* phi_hat, double* f_theta, double* f_phi,
                 double* intensity);
int so_surface_fields(const double* V, const int* F, const int* FE, int nf, int ne, const double* J,
                      const double* M, int nobs, const double* obs, double freq, double eps_r, double mu_r,
                      double eps0, double mu0, int rule, double* E, double* H);

#ifdef __cplusplus
}
#endif
#endif
