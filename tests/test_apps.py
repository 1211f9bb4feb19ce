"""CPU: the anisotropic_sphere_app drop-in (sieb200/apps) — argument parsing,
validation and messages of anisotropic_sphere_app.cpp:128-324, the file
formats (face_tensors.bin, currents.bin, OBJ), observation sampling and the
JSON / CSV writers. The solve itself runs in tests/test_gpu_apps.py."""

import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
APP = ROOT / "sie-gstc-2026_b200" / "bin" / "anisotropic_sphere_app"
BASE = ["app", "--mesh", "m.obj", "--tensors", "t.bin", "--output-dir", "out", "--frequency-hz", "1e9",
        "--epsilon-r-interior", "2", "--mu-r-interior", "1", "--epsilon-r-exterior", "1", "--mu-r-exterior", "1"]


def _parse(extra):
    from sieb200.apps.anisotropic_sphere_app import parse_arguments
    return parse_arguments(BASE + extra)


def test_parse_cases_and_sources():
    a = _parse(["--case", "pw", "--plane-wave", "exterior", "1", "0", "0", "0", "0", "1",
                "--case", "dip_1", "--dipole", "interior", "magnetic", "0", "0", "1", "0.1", "0", "0",
                "--plane-wave", "exterior", "0", "1", "0", "1", "0", "0",
                "--basis", "face", "--quadrature-rule", "7", "--no-residual", "--zx-grid-size", "4"])
    assert [c.id for c in a.cases] == ["pw", "dip_1"]
    assert a.cases[0].interior is None and a.cases[0].exterior.region == 2
    d = a.cases[1].interior
    assert d.is_magnetic and tuple(d.position) == (0.1, 0.0, 0.0) and d.region == 1
    assert a.basis == "face" and a.quadrature_rule == 7 and not a.compute_residual and a.zx_grid_size == 4
    assert a.frequency_hz == 1e9 and a.epsilon_r_interior == 2.0


@pytest.mark.parametrize("extra,message", [
    ([], "at least one --case is required"),
    (["--plane-wave", "exterior", "1", "0", "0", "0", "0", "1"], "--plane-wave requires a preceding --case"),
    (["--case", "a", "--plane-wave", "exterior", "1", "0", "0", "0", "0", "1",
      "--plane-wave", "exterior", "1", "0", "0", "0", "0", "1"], "duplicate source region in case a"),
    (["--case", "A"], "invalid case ID: A"),
    (["--case", "a", "--plane-wave", "exterior", "1", "0", "0", "0", "0", "1", "--case", "a"],
     "duplicate case ID: a"),
    (["--case", "a"], "case a requires an excitation"),
    (["--case", "a", "--dipole", "interior", "x", "0", "0", "1", "0", "0", "0"],
     "dipole type must be electric or magnetic"),
    (["--case", "a", "--dipole", "inside"], "source region must be interior or exterior"),
    # require_value names argv[index], the last token read (cli_helpers.hpp:16-21)
    (["--case", "a", "--plane-wave", "exterior", "1", "0"], "missing value for option 0"),
    (["--case"], "missing value for option --case"),
    (["--frequency-hz", "1e9x"], "invalid numeric value for --frequency-hz: 1e9x"),
    (["--quadrature-rule", "7.5"], "invalid integer value for --quadrature-rule: 7.5"),
    (["--basis", "cartesian"], "--basis must be 'spherical' or 'face', got: cartesian"),
    (["--bogus"], "unknown option: --bogus"),
])
def test_parse_errors_match_reference_messages(extra, message):
    with pytest.raises(ValueError) as e:
        _parse(extra)
    assert str(e.value) == message


@pytest.mark.parametrize("extra,message", [
    (["--quadrature-rule", "21"], "--quadrature-rule must be in [1, 20]"),
    (["--zx-grid-size", "5"], "--zx-grid-size must be an even integer greater than one"),
    (["--zx-span-radii", "1"], "--zx-span-radii must be greater than one"),
    (["--radial-points", "1"], "--radial-points must be at least two"),
    (["--radial-min-radii", "1"], "--radial-min-radii must lie strictly between zero and one"),
    (["--radial-max-radii", "0.5"], "--radial-max-radii must be greater than one"),
    (["--singularity-threshold-lambda0", "0"], "--singularity-threshold-lambda0 must be positive"),
    (["--mu-r-exterior", "-1"], "all relative material parameters must be positive"),
])
def test_range_checks_match_reference_messages(extra, message):
    with pytest.raises(ValueError) as e:
        _parse(["--case", "a", "--plane-wave", "exterior", "1", "0", "0", "0", "0", "1"] + extra)
    assert str(e.value) == message


def test_command_line_exit_codes():
    r = subprocess.run([sys.executable, str(APP), "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.startswith("Usage:")
    r = subprocess.run([sys.executable, str(APP), "--mesh", "x"], capture_output=True, text=True)
    assert r.returncode == 2
    assert r.stderr.startswith("anisotropic_sphere_app: --tensors is required")
    assert "Required options:" in r.stdout


def test_observation_samples_geometry():
    from sieb200.apps.anisotropic_sphere_app import Arguments, make_observation_samples
    a = Arguments(zx_grid_size=4, radial_points=5, zx_span_radii=2.0, radial_min_radii=0.5,
                  radial_max_radii=1.5, radial_theta_degrees=90.0, radial_phi_degrees=90.0)
    s = make_observation_samples(a, 0.5)
    assert s.points.shape == (21, 3) and s.zx_count == 16
    assert np.allclose(s.points[0], [-1.0, 0.0, -1.0]) and np.allclose(s.points[15], [1.0, 0.0, 1.0])
    assert np.all(s.points[:16, 1] == 0.0)
    r = np.linalg.norm(s.points[16:], axis=1)
    assert np.allclose(r, [0.25, 0.375, 0.5, 0.625, 0.75])
    assert np.allclose(s.points[16:, 0], 0.0, atol=1e-16)  # phi = 90 deg: along +y
    assert list(s.regions[16:]) == [1, 1, 2, 2, 2]  # strictly inside -> region 1


def test_face_tensor_files(tmp_path):
    from sieb200.io import load_face_tensors, save_face_tensors
    rng = np.random.default_rng(0)
    t = rng.standard_normal((6, 32)) + 1j * rng.standard_normal((6, 32))
    save_face_tensors(tmp_path / "t64.bin", t)
    assert np.array_equal(load_face_tensors(tmp_path / "t64.bin", 6), t)
    save_face_tensors(tmp_path / "t32.bin", t, single=True)
    assert np.array_equal(load_face_tensors(tmp_path / "t32.bin", 6), t.astype(np.complex64).astype(np.complex128))
    with pytest.raises(RuntimeError, match="Tensor file size mismatch. Expected 1792 or 3584 bytes, got 3072"):
        load_face_tensors(tmp_path / "t64.bin", 7)
    with pytest.raises(RuntimeError, match="Could not open tensor file"):
        load_face_tensors(tmp_path / "missing.bin", 6)


def test_currents_file_round_trip(tmp_path):
    from sieb200.io import read_physical_currents, write_physical_currents
    c = np.array([1 + 2j, -3.5 + 0.25j])
    write_physical_currents(tmp_path / "c.bin", c)
    raw = (tmp_path / "c.bin").read_bytes()
    assert len(raw) == 32 and np.array_equal(np.frombuffer(raw, "<f8"), [1.0, 2.0, -3.5, 0.25])
    assert np.array_equal(read_physical_currents(tmp_path / "c.bin"), c)


def test_obj_loader_checks(tmp_path):
    import sieb200
    p = tmp_path / "m.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 2 3 # comment\nf -3 -1 -2\nf 1/1/1 4//2 2\nf 3 4 1\n")
    m = sieb200.load_obj(p)
    assert m.faces.tolist() == [[0, 1, 2], [1, 3, 2], [0, 3, 1], [2, 3, 0]]
    for body, msg in [("v 0 0\n", ":1: vertex requires three coordinates"),
                      ("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 3 4\n", ":5: only triangular faces are supported"),
                      ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n", ":4: invalid face vertex index '0'"),
                      ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf -4 1 2\n", ":4: relative face vertex index is out of range"),
                      ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf /1 1 2\n", ":4: face has an empty vertex index"),
                      ("v 0 0 0\n", ": no faces")]:
        p.write_text(body)
        with pytest.raises(RuntimeError, match=msg):
            sieb200.load_obj(p)


def test_sphere_radius_inference():
    import sieb200
    m = sieb200.icosphere(0.3, 1)
    r = np.linalg.norm(m.vertices, axis=1)
    assert abs(sieb200.infer_sphere_radius(m) - r.mean()) < 1e-15 and abs(r.mean() - 0.3) < 1e-7
    m.vertices = m.vertices * np.array([1.0, 1.0, 1.01])
    with pytest.raises(RuntimeError, match="common spherical radius"):
        sieb200.infer_sphere_radius(m)


def test_metrics_and_field_writers(tmp_path):
    import sieb200
    from sieb200.apps.anisotropic_sphere_app import (ExcitationCase, ObservationSamples, write_batch_metrics,
                                                     write_field_csv, write_solver_metrics)
    m = sieb200.icosphere(0.5, 0)
    metrics = dict(matrix_dimension=120, dense_matrix_bytes=230400, assembly_seconds=0.5,
                   factorization_seconds=0.25, solve_seconds=1e-3, residual_seconds=0.125,
                   residual_computed=1, rhs_norm=3.0, absolute_residual=1e-14, relative_residual=2e-15,
                   maximum_coefficient=[1.0, 2.0, 3.0, 4.0])
    write_batch_metrics(tmp_path / "b.json", m, metrics, [ExcitationCase("a"), ExcitationCase("b")], "face", 0.75)
    b = json.loads((tmp_path / "b.json").read_text())
    assert b["artifact"] == "anisotropic_sphere_app_batch" and b["case_ids"] == ["a", "b"]
    assert b["mesh"] == {"vertex_count": 12, "face_count": 20, "edge_count": 30}
    assert b["solver"]["matrix_dimension"] == 120 and b["solver"]["basis"] == "face"
    assert b["solver"]["residual_matrix_assembly_seconds"] == 0.125
    cur = np.zeros(120, np.complex128)
    write_solver_metrics(tmp_path / "s.json", "a", cur, metrics, "face", 0.0)
    s = json.loads((tmp_path / "s.json").read_text())
    assert s["current_data"]["complex_value_count"] == 120 and s["current_data"]["path"] == "currents.bin"
    assert s["solver"]["maximum_m2_coefficient"] == 4.0 and s["solver"]["scaled_relative_residual"] == 2e-15
    metrics["residual_computed"] = 0
    write_solver_metrics(tmp_path / "s2.json", "a", cur, metrics, "face", 0.0)
    assert "scaled_relative_residual" not in json.loads((tmp_path / "s2.json").read_text())["solver"]
    obs = ObservationSamples(np.array([[0.1, 0.0, -0.0], [1.0, 2.0, 3.0]]), np.array([1, 2]), 1)
    E = np.array([[1 + 2j, 0, 0], [0, 0, complex(0.0, -0.5)]])
    H = np.array([[0, 1e-3, 0], [0, 0, 0]], dtype=complex)
    write_field_csv(tmp_path / "f.csv", obs, (E, H), 1, 1)
    lines = (tmp_path / "f.csv").read_text().splitlines()
    assert lines[0].startswith("point_index,x,y,z,region,Ex_real")
    assert lines[1] == "0,1,2,3,2,0,0,0,0,0,-0.5,0,0,0,0,0,0"


# ------------------------------------------------------------ pec_sphere_app
PEC_BASE = ["pec", "--mesh", "m.obj", "--output-dir", "out", "--frequency-hz", "3e8"]


def test_pec_parse_and_messages():
    from sieb200.apps.pec_sphere_app import parse
    a = parse(PEC_BASE + ["--formulation", "n", "--ntl-form", "line", "--line-quadrature-points", "12",
                          "--zx-grid-size", "0", "--radial-points", "7", "--frequency-hz", "2e8Hz"])
    assert (a.formulation, a.ntl_form, a.line_quadrature_points) == ("NEfie", "Line", 12)
    assert a.zx_grid_size == 0 and a.radial_points == 7 and a.frequency_hz == 2e8  # stod takes the prefix
    for extra, msg in [(["--formulation", "x"], "--formulation must be t-efie, n-efie, or n-mfie"),
                       (["--ntl-form", "area"], "--ntl-form must be surface or line"),
                       (["--zx-grid-size", "1"], "invalid field sampling range or point count"),
                       (["--radial-max-radii", "0.01"], "invalid field sampling range or point count"),
                       (["--currents-file", "c.csv", "--no-fields"], "--currents-file requires field evaluation"),
                       (["--currents-file", "c.csv", "--export-matrix"],
                        "--export-matrix requires solving, not --currents-file"),
                       (["--quadrature-rule", "x"], "stoi"),
                       (["--zz"], "unknown option: --zz"),
                       (["--mesh"], "missing option value")]:
        with pytest.raises(ValueError) as e:
            parse(PEC_BASE + extra)
        assert str(e.value) == msg
    with pytest.raises(ValueError, match="are required"):
        parse(["pec", "--mesh", "m.obj"])


def test_pec_matrix_npy_and_currents_csv(tmp_path):
    from sieb200.apps.pec_sphere_app import read_currents, write_matrix_npy
    rng = np.random.default_rng(1)
    Z = rng.standard_normal((5, 5)) + 1j * rng.standard_normal((5, 5))
    write_matrix_npy(tmp_path / "m.npy", Z)
    raw = (tmp_path / "m.npy").read_bytes()
    assert raw[:8] == b"\x93NUMPY\x01\x00" and (10 + int.from_bytes(raw[8:10], "little")) % 16 == 0
    back = np.load(tmp_path / "m.npy")
    assert np.array_equal(back, Z) and back.flags["F_CONTIGUOUS"]
    c = tmp_path / "c.csv"
    c.write_text("edge,J2_real,J2_imag,J2_abs\n0,1.5,-2,2.5\n1,0,1e-3,1e-3\n")
    assert np.array_equal(read_currents(str(c), 2), [1.5 - 2j, 1e-3j])
    with pytest.raises(RuntimeError, match="edge count does not match mesh"):
        read_currents(str(c), 3)
    c.write_text("edge,J2_real,J2_imag,J2_abs\n1,1.5,-2,2.5\n")
    with pytest.raises(RuntimeError, match="invalid current CSV row"):
        read_currents(str(c), 1)
    c.write_text("edge,J2\n")
    with pytest.raises(RuntimeError, match="unexpected current CSV header"):
        read_currents(str(c), 0)


def test_pec_observations():
    from sieb200.apps.pec_sphere_app import Arguments, make_observations
    a = Arguments(zx_grid_size=3, radial_points=3, radial_min_radii=0.0, radial_max_radii=2.0,
                  radial_theta_degrees=0.0)
    o = make_observations(a, 1.0)
    assert o.zx_count == 9 and o.points.shape == (12, 3)
    assert np.allclose(o.points[4], [0, 0, 0]) and o.regions[4] == 1 and o.regions[0] == 2
    assert np.allclose(o.points[9:, 2], [0.0, 1.0, 2.0]) and list(o.regions[9:]) == [1, 2, 2]
    o = make_observations(Arguments(zx_grid_size=0, radial_points=0), 1.0)
    assert o.points.shape == (0, 3)


def _fake_library(monkeypatch, ne_blocks):
    """Stand-ins for the GPU calls, so that run() is exercised on the CPU."""
    import sieb200
    from sieb200 import solvers

    class _Ctx:
        pass

    monkeypatch.setattr(sieb200, "default_context", lambda: _Ctx())

    def solve_batch(mesh, tensors, options, cases, ctx=None):
        assert tensors.shape == (mesh.num_faces, 32) and options.basis in ("face", "spherical")
        n = ne_blocks * mesh.num_edges
        metrics = dict(matrix_dimension=n, dense_matrix_bytes=16 * n * n, assembly_seconds=0.5,
                       factorization_seconds=0.25, solve_seconds=0.125, residual_seconds=0.0625,
                       residual_computed=1, rhs_norm=2.0, absolute_residual=2e-15, relative_residual=1e-15,
                       maximum_coefficient=[1.0, 2.0, 3.0, 4.0])
        return [solvers.SolveResult(np.arange(n) * (1 + 1j) * (c + 1), dict(metrics)) for c in range(len(cases))]

    def solve_pec(mesh, options, source, ctx=None):
        return solve_batch(mesh, np.zeros((mesh.num_faces, 32)), sieb200.GstcSieOptions(), [None])[0]

    monkeypatch.setattr(sieb200, "solve_gstc_dense_batch", solve_batch)
    monkeypatch.setattr(sieb200, "solve_pec_dense", solve_pec)
    monkeypatch.setattr(sieb200, "assemble_matrix",
                        lambda mesh, options, ctx=None: np.eye(mesh.num_edges, dtype=complex))
    monkeypatch.setattr(sieb200, "evaluate_surface_integral_fields",
                        lambda mesh, j, m, P, *a, **k: (np.ones((len(P), 3), complex), np.zeros((len(P), 3), complex)))
    monkeypatch.setattr(sieb200, "incident_fields",
                        lambda P, src, options, ctx=None: (3 * np.ones((len(P), 3), complex),
                                                           np.ones((len(P), 3), complex)))


def test_anisotropic_run_writes_the_reference_file_set(tmp_path, monkeypatch, capsys):
    import sieb200
    from sieb200.apps.anisotropic_sphere_app import main
    from sieb200.io import read_physical_currents, save_face_tensors
    _fake_library(monkeypatch, 4)
    mesh = sieb200.icosphere(0.5, 0)
    sieb200.save_obj(mesh, tmp_path / "s.obj")
    save_face_tensors(tmp_path / "t.bin", np.zeros((mesh.num_faces, 32)), single=True)
    out = tmp_path / "run"
    rc = main(["app", "--mesh", str(tmp_path / "s.obj"), "--tensors", str(tmp_path / "t.bin"), "--output-dir",
               str(out), "--frequency-hz", "1e8", "--epsilon-r-interior", "2", "--mu-r-interior", "1",
               "--epsilon-r-exterior", "1", "--mu-r-exterior", "1", "--case", "a",
               "--plane-wave", "exterior", "1", "0", "0", "0", "0", "1", "--case", "b",
               "--dipole", "interior", "electric", "0", "0", "1", "0", "0", "0",
               "--zx-grid-size", "4", "--radial-points", "3"])
    assert rc == 0
    assert json.loads((out / "batch_metrics.json").read_text())["solver"]["matrix_dimension"] == 120
    for c, case in enumerate(("a", "b")):
        d = out / "cases" / case
        assert np.array_equal(read_physical_currents(d / "currents.bin"), np.arange(120) * (1 + 1j) * (c + 1))
        assert json.loads((d / "solver_metrics.json").read_text())["case_id"] == case
        for rep in ("interior_representation", "exterior_representation", "physical"):
            assert len((d / "fields" / f"sie_{rep}_zx.csv").read_text().splitlines()) == 17
            assert len((d / "fields" / f"sie_{rep}_radial.csv").read_text().splitlines()) == 4
        rows = np.loadtxt(d / "fields" / "sie_physical_radial.csv", delimiter=",", skiprows=1)
        # incident (3) minus surface integral (1) in the source's region, 0 - 1 elsewhere
        inside = rows[:, 4] == 1
        expect_inside = 2.0 if case == "b" else -1.0
        expect_outside = 2.0 if case == "a" else -1.0
        assert np.all(rows[inside, 5] == expect_inside) and np.all(rows[~inside, 5] == expect_outside)
    assert "Starting dense CUDA solve..." in capsys.readouterr().out


def test_pec_run_writes_the_reference_file_set(tmp_path, monkeypatch):
    import sieb200
    from sieb200.apps.pec_sphere_app import main
    _fake_library(monkeypatch, 1)
    mesh = sieb200.icosphere(0.5, 0)
    sieb200.save_obj(mesh, tmp_path / "s.obj")
    out = tmp_path / "run"
    assert main(["pec", "--mesh", str(tmp_path / "s.obj"), "--output-dir", str(out), "--frequency-hz", "1e8",
                 "--export-matrix", "--zx-grid-size", "2", "--radial-points", "2"]) == 0
    lines = (out / "currents.csv").read_text().splitlines()
    assert lines[0] == "edge,J2_real,J2_imag,J2_abs" and lines[2] == "1,1,1,1.4142135623730951"
    assert np.array_equal(np.load(out / "matrix.npy"), np.eye(30))
    assert (out / "matrix_edges.csv").read_text().splitlines()[0] == "edge,vertex_a,vertex_b"
    f = (out / "radial_fields.csv").read_text().splitlines()
    assert f[1].split(",")[4] == "2.000000000000e+00" and len(f) == 3
    assert len((out / "zx_fields.csv").read_text().splitlines()) == 5
