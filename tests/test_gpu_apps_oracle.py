"""GPU: the two application drop-ins end to end, their output files checked
against the oracle (the C restatement of the reference's assembly,
excitation, incident-field and surface-integral routines) rather than against
this library's own calls.

* anisotropic_sphere_app: currents.bin of a plane-wave case and an interior
  dipole case against the oracle's FP64 solution (M blocks x eta0), and the
  physical radial field cut (incident minus the surface integrals of the
  region's currents) against the oracle's fields of those currents;
* pec_sphere_app (N-EFIE): currents.csv against the oracle's FP64 solution,
  matrix.npy against the oracle's matrix, the radial field cut against the
  oracle's incident minus surface-integral field.

Tolerances: currents 1e-10 (FP64 solves), matrices 1e-12, fields 1e-10
(the GSTC app writes 17 digits) and 1e-9 (the PEC app writes 13 digits)."""

import json
import math

import numpy as np
import pytest

from conftest import rel_err
from oracle import oracle as O

pytestmark = pytest.mark.gpu
C0 = 299792458.0


def test_anisotropic_sphere_app_against_oracle(tmp_path, gpu_ctx, oracle_lib):
    import sieb200
    from sieb200.apps.anisotropic_sphere_app import main
    from sieb200.io import read_physical_currents, save_face_tensors
    mesh = sieb200.icosphere(0.5, 1)
    sieb200.save_obj(mesh, tmp_path / "sphere.obj")
    rng = np.random.default_rng(18)
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
    m2 = sieb200.load_obj(tmp_path / "sphere.obj")
    ne = m2.num_edges
    s = O.kernel_scalars(2, C0, eps_r=(2.0, 1.0))
    Zo = O.assemble(oracle_lib, 2, m2, 5, s, tensors=t)
    omega = 2 * math.pi * C0
    eta0 = math.sqrt(s["mu0"] / s["eps0"])
    media = {1: (2.0, 1.0), 2: (1.0, 1.0)}
    specs = {"pw": dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2),
             "dip": dict(kind=1, a=[0, 0, 1], b=[0.05, 0, 0], is_magnetic=0, region=1)}
    for cid, spec in specs.items():
        er, mr = media[spec["region"]]
        k = omega * math.sqrt(s["mu0"] * mr * s["eps0"] * er)
        eta = math.sqrt(s["mu0"] * mr / (s["eps0"] * er))
        bo = O.rhs(oracle_lib, 2, m2, 5, spec, k, eta, s["mu0"], s["eps0"])
        xo = np.linalg.solve(Zo, bo)
        xo[ne:2 * ne] *= eta0
        xo[3 * ne:] *= eta0
        d = out / "cases" / cid
        cur = read_physical_currents(d / "currents.bin")
        assert np.linalg.norm(cur - xo) / np.linalg.norm(xo) < 1e-10
        rows = np.loadtxt(d / "fields" / "sie_physical_radial.csv", delimiter=",", skiprows=1)
        P, reg = rows[:, 1:4], rows[:, 4].astype(int)
        E_csv = rows[:, 5:11:2] + 1j * rows[:, 6:12:2]
        blocks = [xo[b * ne:(b + 1) * ne] for b in range(4)]
        for region in (1, 2):
            sel = reg == region
            if not sel.any():
                continue
            j, mm = (blocks[0], blocks[1]) if region == 1 else (blocks[2], blocks[3])
            er, mr = media[region]
            Q, _ = O.surface_fields(oracle_lib, m2, j, mm, P[sel], C0, er, mr, s["eps0"], s["mu0"], 5)
            if spec["region"] == region:
                k = omega * math.sqrt(s["mu0"] * mr * s["eps0"] * er)
                eta = math.sqrt(s["mu0"] * mr / (s["eps0"] * er))
                inc, _ = O.incident_fields(oracle_lib, spec, k, eta, P[sel])
            else:
                inc = 0.0
            ref = inc - Q
            assert np.abs(E_csv[sel] - ref).max() <= 1e-10 * np.abs(ref).max()


def test_pec_sphere_app_against_oracle(tmp_path, gpu_ctx, oracle_lib):
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
    s = O.kernel_scalars(0, C0)
    Zo = O.assemble(oracle_lib, 0, m2, 5, s, variant=1)
    assert rel_err(np.load(out / "matrix.npy"), Zo) < 1e-12
    k = s["omega"] * math.sqrt(s["mu0"] * s["eps0"])
    eta = math.sqrt(s["mu0"] / s["eps0"])
    spec = dict(kind=0, a=[1, 0, 0], b=[0, 0, 1], region=2)
    bo = O.rhs(oracle_lib, 0, m2, 5, spec, k, eta, s["mu0"], s["eps0"], variant=1)
    xo = np.linalg.solve(Zo, bo)
    rows = np.loadtxt(out / "currents.csv", delimiter=",", skiprows=1)
    cur = rows[:, 1] + 1j * rows[:, 2]
    assert np.linalg.norm(cur - xo) / np.linalg.norm(xo) < 1e-10
    f = np.loadtxt(out / "radial_fields.csv", delimiter=",", skiprows=1)
    P = f[:, :3]
    Q, _ = O.surface_fields(oracle_lib, m2, xo, None, P, C0, 1.0, 1.0, s["eps0"], s["mu0"], 5)
    inc, _ = O.incident_fields(oracle_lib, spec, k, eta, P)
    E = f[:, 4:10:2] + 1j * f[:, 5:11:2]
    ref = inc - Q
    assert np.abs(E - ref).max() <= 1e-9 * np.abs(ref).max()
