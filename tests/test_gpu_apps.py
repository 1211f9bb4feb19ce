"""GPU: the incident-field entry point against the oracle, and the
anisotropic_sphere_app drop-in end to end (OBJ + face_tensors.bin in,
currents.bin, metrics JSON and field CSVs out) against the library calls it
is built on."""

import json
import math

import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def test_incident_fields_match_oracle(gpu_ctx, oracle_lib):
    import sieb200
    o = sieb200.GstcSieOptions(frequency_hz=C0, interior=sieb200.IsotropicMedium(3.0, 1.5))
    rng = np.random.default_rng(4)
    P = rng.uniform(-1, 1, (50, 3))
    eps0, mu0 = o.vacuum_permittivity, o.vacuum_permeability
    omega = 2 * math.pi * C0
    cases = [
        (sieb200.PlaneWaveExcitation(electric_amplitude=(0, 2.0, 0), propagation_direction=(3.0, 0, 0)),
         dict(kind=0, a=[0, 2.0, 0], b=[3.0, 0, 0]), 1.0, 1.0),
        (sieb200.DipoleExcitation(effective_moment=(0.2, 0, 1), position=(0.1, 0.05, 0), is_magnetic=True,
                                  region=sieb200.INTERIOR),
         dict(kind=1, a=[0.2, 0, 1], b=[0.1, 0.05, 0], is_magnetic=1), 3.0, 1.5),
        (sieb200.DipoleExcitation(effective_moment=(0, 1, 0), position=(0, 0, 0.2), region=sieb200.INTERIOR),
         dict(kind=1, a=[0, 1, 0], b=[0, 0, 0.2]), 3.0, 1.5),
    ]
    for src, spec, er, mr in cases:
        E, H = sieb200.incident_fields(P, src, o, ctx=gpu_ctx)
        k = omega * math.sqrt(mu0 * mr * eps0 * er)
        eta = math.sqrt(mu0 * mr / (eps0 * er))
        Eo, Ho = O.incident_fields(oracle_lib, spec, k, eta, P)
        assert rel_err(E, Eo) < 1e-12 and rel_err(H, Ho) < 1e-12


def test_anisotropic_sphere_app_end_to_end(tmp_path, gpu_ctx):
    import sieb200
    from sieb200.apps.anisotropic_sphere_app import main
    from sieb200.io import read_physical_currents, save_face_tensors
    mesh = sieb200.icosphere(0.5, 1)
    sieb200.save_obj(mesh, tmp_path / "sphere.obj")
    rng = np.random.default_rng(8)
    t = 0.3 * (rng.standard_normal((mesh.num_faces, 32)) + 1j * rng.standard_normal((mesh.num_faces, 32)))
    save_face_tensors(tmp_path / "face_tensors.bin", t)
    out = tmp_path / "run"
    argv = ["anisotropic_sphere_app", "--mesh", str(tmp_path / "sphere.obj"), "--tensors",
            str(tmp_path / "face_tensors.bin"), "--output-dir", str(out), "--frequency-hz", str(C0),
            "--epsilon-r-interior", "2", "--mu-r-interior", "1", "--epsilon-r-exterior", "1", "--mu-r-exterior", "1",
            "--quadrature-rule", "5", "--basis", "face",
            "--case", "pw", "--plane-wave", "exterior", "1", "0", "0", "0", "0", "1",
            "--case", "dip", "--dipole", "interior", "electric", "0", "0", "1", "0.05", "0", "0",
            "--zx-grid-size", "4", "--radial-points", "5"]
    assert main(argv) == 0
    batch = json.loads((out / "batch_metrics.json").read_text())
    assert batch["case_ids"] == ["pw", "dip"] and batch["solver"]["matrix_dimension"] == 4 * mesh.num_edges
    o = sieb200.GstcSieOptions(frequency_hz=C0, interior=sieb200.IsotropicMedium(2.0, 1.0), quadrature_rule=5,
                               basis="face")
    m2 = sieb200.load_obj(tmp_path / "sphere.obj")
    cases = [sieb200.GstcExcitationCase(exterior=sieb200.PlaneWaveExcitation()),
             sieb200.GstcExcitationCase(interior=sieb200.DipoleExcitation(effective_moment=(0, 0, 1),
                                                                          position=(0.05, 0, 0)))]
    ref = sieb200.solve_gstc_dense_batch(m2, t, o, cases, ctx=gpu_ctx)
    for cid, r, case in zip(["pw", "dip"], ref, cases):
        d = out / "cases" / cid
        cur = read_physical_currents(d / "currents.bin")
        assert rel_err(cur, r.currents) < 1e-12
        sm = json.loads((d / "solver_metrics.json").read_text())
        assert sm["solver"]["residual_computed"] and sm["solver"]["scaled_relative_residual"] < 1e-10
        # physical field on the radial cut = incident - surface integrals of the region's currents
        rows = np.loadtxt(d / "fields" / "sie_physical_radial.csv", delimiter=",", skiprows=1)
        assert rows.shape == (5, 17)
        P, reg = rows[:, 1:4], rows[:, 4].astype(int)
        E_csv = rows[:, 5:11:2] + 1j * rows[:, 6:12:2]
        ne = m2.num_edges
        blocks = [cur[b * ne:(b + 1) * ne] for b in range(4)]
        for region, (j, mm, medium, src) in {1: (blocks[0], blocks[1], o.interior, case.interior),
                                             2: (blocks[2], blocks[3], o.exterior, case.exterior)}.items():
            sel = reg == region
            if not sel.any():
                continue
            Q, _ = sieb200.evaluate_surface_integral_fields(m2, j, mm, P[sel], C0, medium, 5, ctx=gpu_ctx)
            inc = sieb200.incident_fields(P[sel], src, o, ctx=gpu_ctx)[0] if src is not None else 0.0
            assert rel_err(E_csv[sel], inc - Q) < 1e-12
        assert (d / "fields" / "sie_interior_representation_zx.csv").is_file()


def test_pec_sphere_app_end_to_end(tmp_path, gpu_ctx):
    import sieb200
    from sieb200.apps.pec_sphere_app import main
    mesh = sieb200.icosphere(0.5, 1)
    sieb200.save_obj(mesh, tmp_path / "sphere.obj")
    out = tmp_path / "run"
    argv = ["pec_sphere_app", "--mesh", str(tmp_path / "sphere.obj"), "--output-dir", str(out),
            "--frequency-hz", str(C0), "--formulation", "n-efie", "--quadrature-rule", "5",
            "--export-matrix", "--zx-grid-size", "4", "--radial-points", "6"]
    assert main(argv) == 0
    m2 = sieb200.load_obj(tmp_path / "sphere.obj")
    o = sieb200.PecOptions(frequency_hz=C0, quadrature_rule=5, formulation="NEfie")
    r = sieb200.solve_pec_dense(m2, o, sieb200.PlaneWaveExcitation(), ctx=gpu_ctx)
    rows = np.loadtxt(out / "currents.csv", delimiter=",", skiprows=1)
    assert rel_err(rows[:, 1] + 1j * rows[:, 2], r.currents) < 1e-12
    assert np.allclose(rows[:, 3], np.abs(rows[:, 1] + 1j * rows[:, 2]), rtol=1e-15)
    Z = np.load(out / "matrix.npy")
    assert rel_err(Z, sieb200.assemble_matrix(m2, o, ctx=gpu_ctx)) < 1e-15
    f = np.loadtxt(out / "radial_fields.csv", delimiter=",", skiprows=1)
    assert f.shape == (6, 16)
    P = f[:, :3]
    Q, _ = sieb200.evaluate_surface_integral_fields(m2, r.currents, None, P, C0, o.exterior, 5,
                                                    o.vacuum_permittivity, o.vacuum_permeability, ctx=gpu_ctx)
    inc, _ = sieb200.incident_fields(P, sieb200.PlaneWaveExcitation(), o, ctx=gpu_ctx)
    E = f[:, 4:10:2] + 1j * f[:, 5:11:2]
    assert rel_err(E, inc - Q) < 1e-11  # the CSV carries 13 significant digits
    # --currents-file: the saved J2 gives the same field files without a solve
    out2 = tmp_path / "fields_only"
    assert main(["pec_sphere_app", "--mesh", str(tmp_path / "sphere.obj"), "--output-dir", str(out2),
                 "--frequency-hz", str(C0), "--quadrature-rule", "5", "--currents-file", str(out / "currents.csv"),
                 "--zx-grid-size", "4", "--radial-points", "6"]) == 0
    assert (out2 / "radial_fields.csv").read_text() == (out / "radial_fields.csv").read_text()
    assert (out2 / "zx_fields.csv").read_text() == (out / "zx_fields.csv").read_text()
