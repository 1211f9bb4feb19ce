// Test and measurement infrastructure only (never the product): the
// reference's own GPU solver, solve_dielectric_dense
// (include/sie_mom/solvers/dielectric/dielectric_solver.hpp:92-96 ->
// src/sie_mom/solvers/dielectric/dielectric_solver.cu: its assembly kernels,
// cusolverDnZgetrf/Zgetrs and its residual), compiled for sm_100a from the
// reference's sources by oracle/Makefile (target ref_gpu) and called here
// on a caller's mesh, so the benchmark can time the reference's GPU path on
// the same box and the same system.

#include <chrono>
#include <complex>
#include <cstring>
#include <exception>
#include <string>

#include "sie_mom/excitation/excitation.hpp"
#include "sie_mom/solvers/dielectric/dielectric_solver.hpp"

namespace {
thread_local std::string g_error;
}

extern "C" {

const char* ref_gpu_last_error(void) { return g_error.c_str(); }

// T-PMCHWT solve of an x-polarised plane wave along +z (exterior). V: nv x 3,
// F, FE: nf x 3, E: ne x 2. currents_out: 2 ne complex (interior-oriented
// [J, M], physical). times_out[0..4]: device preparation, assembly, solve
// (factorization + triangular solves), residual, wall seconds of the call;
// times_out[5]: relative residual. Returns 0 or -1 (message in
// ref_gpu_last_error).
int ref_gpu_solve_dielectric(const double* V, int nv, const int* F, int nf, const int* E, const int* FE, int ne,
                             double frequency_hz, double eps_r_interior, int rule, double* currents_out,
                             double* times_out) {
    try {
        using namespace sie_mom;
        mesh::MeshData mesh;
        mesh.vertices.resize(nv);
        for (int i = 0; i < nv; ++i) mesh.vertices[i] = make_vec3(V[3 * i], V[3 * i + 1], V[3 * i + 2]);
        mesh.faces.resize(nf);
        mesh.faces_edges.resize(nf);
        for (int f = 0; f < nf; ++f) {
            mesh.faces[f] = {F[3 * f], F[3 * f + 1], F[3 * f + 2]};
            mesh.faces_edges[f] = {FE[3 * f], FE[3 * f + 1], FE[3 * f + 2]};
        }
        mesh.edges.resize(ne);
        for (int e = 0; e < ne; ++e) mesh.edges[e] = {E[2 * e], E[2 * e + 1]};
        solvers::DielectricOptions o;
        o.frequency_hz = frequency_hz;
        o.interior.relative_permittivity = eps_r_interior;
        o.quadrature_rule = rule;
        excitation::PlaneWaveExcitation pw;
        const auto src = excitation::prepare_source(excitation::SourceSpec(pw), o.frequency_hz, o.interior,
                                                    o.exterior, o.vacuum_permittivity, o.vacuum_permeability);
        const auto t0 = std::chrono::steady_clock::now();
        const auto res = solvers::solve_dielectric_dense(mesh, o, src);
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::memcpy(currents_out, res.physical_currents.data(), sizeof(double) * 2 * res.physical_currents.size());
        times_out[0] = res.metrics.device_preparation_seconds;
        times_out[1] = res.metrics.assembly_seconds;
        times_out[2] = res.metrics.solve_seconds;
        times_out[3] = res.metrics.residual_seconds;
        times_out[4] = wall;
        times_out[5] = res.metrics.relative_residual;
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

}  // extern "C"
