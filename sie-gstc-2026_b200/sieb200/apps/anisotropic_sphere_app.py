"""Drop-in for applications/anisotropic_gstc_sphere/anisotropic_sphere_app.cpp
on the sieb200 C ABI: the same flags, validation and messages, the same
inputs (strict triangular OBJ mesh, face_tensors.bin) and the same outputs
under --output-dir:

    batch_metrics.json
    cases/<id>/currents.bin          [J1, M1, J2, M2] physical, complex128 LE
    cases/<id>/solver_metrics.json
    cases/<id>/fields/sie_{interior_representation,exterior_representation,physical}_{zx,radial}.csv

so the repository's Python workflows (sie_gstc_sphere.py, via --executable)
run unchanged. One extension: --solver selects the dense method (default
lu_cusolver, the reference's LU; mixed_ir the tensor-core LU refined to
--tolerance).
"""

from __future__ import annotations

import math
import re
import sys
import time
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional

import numpy as np

from .cli import INTERIOR, parse_integer, parse_real, parse_region, parse_vector, require_value

PROGRAM = "anisotropic_sphere_app"


@dataclass
class ExcitationCase:
    id: str
    interior: Optional[object] = None
    exterior: Optional[object] = None


@dataclass
class Arguments:
    mesh_path: str = ""
    tensor_path: str = ""
    output_directory: str = ""
    frequency_hz: float = 0.0
    epsilon_r_interior: float = 0.0
    mu_r_interior: float = 0.0
    epsilon_r_exterior: float = 0.0
    mu_r_exterior: float = 0.0
    cases: list = field(default_factory=list)
    quadrature_rule: int = 17
    singularity_threshold_lambda0: float = 0.1
    basis: str = "spherical"
    compute_residual: bool = True
    evaluate_fields: bool = True
    zx_grid_size: int = 200
    zx_span_radii: float = 2.0
    radial_points: int = 300
    radial_theta_degrees: float = 45.0
    radial_phi_degrees: float = 0.0
    radial_min_radii: float = 0.05
    radial_max_radii: float = 2.0
    solver: str = "lu_cusolver"
    tolerance: float = 1e-10


class UsageExit(Exception):
    """--help: usage printed, exit status 0."""


def usage(program: str) -> str:
    return (
        "Usage:\n  " + program + " [options]\n\n"
        "Required options:\n"
        "  --mesh PATH                         Strict triangular OBJ mesh\n"
        "  --tensors PATH                      Per-face GSTC tensor binary\n"
        "  --output-dir PATH                   Shared run directory\n"
        "  --frequency-hz VALUE                Frequency in hertz\n"
        "  --epsilon-r-interior VALUE          Interior relative permittivity\n"
        "  --mu-r-interior VALUE               Interior relative permeability\n"
        "  --epsilon-r-exterior VALUE          Exterior relative permittivity\n"
        "  --mu-r-exterior VALUE               Exterior relative permeability\n"
        "\nSimulation cases (repeat --case; one source per region):\n"
        "  --case ID                           Start an independent RHS case\n"
        "  --dipole REGION TYPE PX PY PZ X Y Z  Real effective moment and position (m)\n"
        "  --plane-wave REGION EX EY EZ DX DY DZ  Real E0 and propagation direction\n"
        "  REGION: interior or exterior; TYPE: electric or magnetic\n\n"
        "Optional numerical controls:\n"
        "  --basis {spherical,face}            Local tangent basis for GSTC tensors (default: spherical)\n"
        "  --quadrature-rule VALUE             Dunavant rule (default: 17)\n"
        "  --singularity-threshold-lambda0 V   Threshold/lambda0 (default: 0.1)\n"
        "  --no-residual                       Skip residual reassembly\n"
        "  --no-fields                         Skip 2D and radial field evaluation\n"
        "  --solver {lu_cusolver,lu_fp64,mixed_ir}  Dense method (default: lu_cusolver)\n"
        "  --tolerance V                       mixed_ir refinement target (default: 1e-10)\n\n"
        "Optional field sampling:\n"
        "  --zx-grid-size VALUE                Even points per ZX axis (default: 200)\n"
        "  --zx-span-radii VALUE               ZX half-span/a (default: 2)\n"
        "  --radial-points VALUE               Radial samples (default: 300)\n"
        "  --radial-theta-degrees VALUE        Radial-cut theta (default: 45)\n"
        "  --radial-phi-degrees VALUE          Radial-cut phi (default: 0)\n"
        "  --radial-min-radii VALUE            Minimum r/a (default: 0.05)\n"
        "  --radial-max-radii VALUE            Maximum r/a (default: 2)\n"
        "  -h, --help                          Show this message\n")


_REAL_OPTIONS = {
    "--frequency-hz": "frequency_hz", "--epsilon-r-interior": "epsilon_r_interior",
    "--mu-r-interior": "mu_r_interior", "--epsilon-r-exterior": "epsilon_r_exterior",
    "--mu-r-exterior": "mu_r_exterior", "--singularity-threshold-lambda0": "singularity_threshold_lambda0",
    "--zx-span-radii": "zx_span_radii", "--radial-theta-degrees": "radial_theta_degrees",
    "--radial-phi-degrees": "radial_phi_degrees", "--radial-min-radii": "radial_min_radii",
    "--radial-max-radii": "radial_max_radii", "--tolerance": "tolerance",
}
_INT_OPTIONS = {"--quadrature-rule": "quadrature_rule", "--zx-grid-size": "zx_grid_size",
                "--radial-points": "radial_points"}
_CASE_ID = re.compile(r"[a-z0-9][a-z0-9_-]*")


def parse_arguments(argv: list[str]) -> Arguments:
    """anisotropic_sphere_app.cpp:128-324; argv[0] is the program name."""
    import sieb200
    a = Arguments()
    i = 1
    while i < len(argv):
        option = argv[i]
        if option == "--mesh":
            a.mesh_path, i = require_value(argv, i)
        elif option == "--tensors":
            a.tensor_path, i = require_value(argv, i)
        elif option == "--output-dir":
            a.output_directory, i = require_value(argv, i)
        elif option in _REAL_OPTIONS:
            text, i = require_value(argv, i)
            setattr(a, _REAL_OPTIONS[option], parse_real(text, option))
        elif option in _INT_OPTIONS:
            text, i = require_value(argv, i)
            setattr(a, _INT_OPTIONS[option], parse_integer(text, option))
        elif option == "--case":
            text, i = require_value(argv, i)
            a.cases.append(ExcitationCase(text))
        elif option in ("--dipole", "--plane-wave"):
            if not a.cases:
                raise ValueError(f"{option} requires a preceding --case")
            text, i = require_value(argv, i)
            region = parse_region(text)
            slot = "interior" if region == INTERIOR else "exterior"
            if getattr(a.cases[-1], slot) is not None:
                raise ValueError("duplicate source region in case " + a.cases[-1].id)
            if option == "--dipole":
                kind, i = require_value(argv, i)
                if kind not in ("electric", "magnetic"):
                    raise ValueError("dipole type must be electric or magnetic")
                moment, i = parse_vector(argv, i, option)
                position, i = parse_vector(argv, i, option)
                src = sieb200.DipoleExcitation(effective_moment=moment, position=position,
                                               is_magnetic=kind == "magnetic", region=region)
            else:
                amplitude, i = parse_vector(argv, i, option)
                direction, i = parse_vector(argv, i, option)
                src = sieb200.PlaneWaveExcitation(electric_amplitude=amplitude, propagation_direction=direction,
                                                  region=region)
            setattr(a.cases[-1], slot, src)
        elif option == "--basis":
            text, i = require_value(argv, i)
            if text not in ("spherical", "face"):
                raise ValueError("--basis must be 'spherical' or 'face', got: " + text)
            a.basis = text
        elif option == "--solver":
            a.solver, i = require_value(argv, i)
            if a.solver not in ("lu_cusolver", "lu_fp64", "mixed_ir"):
                raise ValueError("--solver must be lu_cusolver, lu_fp64 or mixed_ir")
        elif option == "--no-residual":
            a.compute_residual = False
        elif option == "--no-fields":
            a.evaluate_fields = False
        elif option in ("--help", "-h"):
            raise UsageExit()
        else:
            raise ValueError("unknown option: " + option)
        i += 1

    if not a.mesh_path:
        raise ValueError("--mesh is required")
    if not a.tensor_path:
        raise ValueError("--tensors is required")
    if not a.output_directory:
        raise ValueError("--output-dir is required")
    if not a.frequency_hz > 0:
        raise ValueError("--frequency-hz must be positive")
    if not (a.epsilon_r_interior > 0 and a.mu_r_interior > 0 and a.epsilon_r_exterior > 0
            and a.mu_r_exterior > 0):
        raise ValueError("all relative material parameters must be positive")
    if not a.cases:
        raise ValueError("at least one --case is required")
    seen = set()
    for c in a.cases:
        if not _CASE_ID.fullmatch(c.id):
            raise ValueError("invalid case ID: " + c.id)
        if c.id in seen:
            raise ValueError("duplicate case ID: " + c.id)
        seen.add(c.id)
        if c.interior is None and c.exterior is None:
            raise ValueError("case " + c.id + " requires an excitation")
    if not 1 <= a.quadrature_rule <= 20:
        raise ValueError("--quadrature-rule must be in [1, 20]")
    if not a.singularity_threshold_lambda0 > 0:
        raise ValueError("--singularity-threshold-lambda0 must be positive")
    if a.zx_grid_size < 2 or a.zx_grid_size % 2 != 0:
        raise ValueError("--zx-grid-size must be an even integer greater than one")
    if not a.zx_span_radii > 1:
        raise ValueError("--zx-span-radii must be greater than one")
    if a.radial_points < 2:
        raise ValueError("--radial-points must be at least two")
    if not 0 < a.radial_min_radii < 1:
        raise ValueError("--radial-min-radii must lie strictly between zero and one")
    if not a.radial_max_radii > 1:
        raise ValueError("--radial-max-radii must be greater than one")
    return a


@dataclass
class ObservationSamples:
    points: np.ndarray
    regions: np.ndarray
    zx_count: int


def make_observation_samples(a: Arguments, sphere_radius: float) -> ObservationSamples:
    """ZX grid (y = 0) then the radial cut (anisotropic_sphere_app.cpp:357-398);
    region 1 strictly inside the sphere radius, else 2."""
    n = a.zx_grid_size
    span = a.zx_span_radii * sphere_radius
    den = float(n - 1)
    pts = []
    for zi in range(n):
        z = -span + 2.0 * span * zi / den
        for xi in range(n):
            x = -span + 2.0 * span * xi / den
            pts.append((x, 0.0, z))
    theta = a.radial_theta_degrees * math.pi / 180.0
    phi = a.radial_phi_degrees * math.pi / 180.0
    st = math.sin(theta)
    rden = float(a.radial_points - 1)
    for k in range(a.radial_points):
        r = (a.radial_min_radii + (a.radial_max_radii - a.radial_min_radii) * k / rden) * sphere_radius
        pts.append((r * st * math.cos(phi), r * st * math.sin(phi), r * math.cos(theta)))
    P = np.array(pts, dtype=np.float64)
    regions = np.where(np.sqrt((P * P).sum(axis=1)) < sphere_radius, 1, 2).astype(np.int32)
    return ObservationSamples(P, regions, n * n)


def evaluate_field_representations(mesh, options, currents, observations: ObservationSamples,
                                   case: ExcitationCase, ctx=None):
    """Interior, exterior and physical fields: incident minus the surface
    integrals of each region's currents (anisotropic_sphere_app.cpp:403-465)."""
    import sieb200
    ne = mesh.num_edges
    if currents.size != 4 * ne:
        raise RuntimeError("physical current vector does not contain four RWG blocks")
    j1, m1, j2, m2 = (currents[b * ne:(b + 1) * ne] for b in range(4))
    P = observations.points
    eps0, mu0 = options.vacuum_permittivity, options.vacuum_permeability
    qi = sieb200.evaluate_surface_integral_fields(mesh, j1, m1, P, options.frequency_hz, options.interior,
                                                  options.quadrature_rule, eps0, mu0, ctx=ctx)
    qe = sieb200.evaluate_surface_integral_fields(mesh, j2, m2, P, options.frequency_hz, options.exterior,
                                                  options.quadrature_rule, eps0, mu0, ctx=ctx)
    zero = (np.zeros_like(qi[0]), np.zeros_like(qi[1]))
    ii = sieb200.incident_fields(P, case.interior, options, ctx=ctx) if case.interior is not None else zero
    ie = sieb200.incident_fields(P, case.exterior, options, ctx=ctx) if case.exterior is not None else zero
    interior = (ii[0] - qi[0], ii[1] - qi[1])
    exterior = (ie[0] - qe[0], ie[1] - qe[1])
    inside = (observations.regions == 1)[:, None]
    physical = (np.where(inside, interior[0], exterior[0]), np.where(inside, interior[1], exterior[1]))
    return {"interior_representation": interior, "exterior_representation": exterior, "physical": physical}


def _g(x: float) -> str:
    """A double as the C++ streams print it with setprecision(17)."""
    return f"{x:.17g}"


def write_field_csv(path: Path, observations: ObservationSamples, fields, offset: int, count: int) -> None:
    E, H = fields
    lines = ["point_index,x,y,z,region,Ex_real,Ex_imag,Ey_real,Ey_imag,Ez_real,Ez_imag,"
             "Hx_real,Hx_imag,Hy_real,Hy_imag,Hz_real,Hz_imag"]
    for local in range(count):
        k = offset + local
        p = observations.points[k]
        row = [str(local), _g(p[0]), _g(p[1]), _g(p[2]), str(int(observations.regions[k]))]
        for c in range(3):
            row += [_g(E[k, c].real), _g(E[k, c].imag)]
        for c in range(3):
            row += [_g(H[k, c].real), _g(H[k, c].imag)]
        lines.append(",".join(row))
    path.write_text("\n".join(lines) + "\n")


def write_field_outputs(directory: Path, observations: ObservationSamples, fields) -> None:
    fdir = directory / "fields"
    fdir.mkdir(parents=True, exist_ok=True)
    n = observations.points.shape[0]
    for name in ("interior_representation", "exterior_representation", "physical"):
        write_field_csv(fdir / f"sie_{name}_zx.csv", observations, fields[name], 0, observations.zx_count)
        write_field_csv(fdir / f"sie_{name}_radial.csv", observations, fields[name], observations.zx_count,
                        n - observations.zx_count)


def write_solver_metrics(path: Path, case_id: str, currents, metrics: dict, basis: str,
                         rhs_seconds: float) -> None:
    """solver_metrics.json with the reference's keys (anisotropic_sphere_app.cpp:551-607).
    The batched solve assembles the right-hand sides together with the matrix
    (both inside matrix_assembly_seconds), so run() reports rhs_assembly_seconds 0."""
    mc = metrics["maximum_coefficient"]
    text = ("{\n"
            "  \"schema_version\": 2,\n"
            "  \"artifact\": \"anisotropic_sphere_app_solution\",\n"
            f"  \"case_id\": \"{case_id}\",\n"
            "  \"batch_metrics\": \"../../batch_metrics.json\",\n"
            "  \"phasor_convention\": \"exp(+j omega t)\",\n"
            "  \"scaling\": \"eta0\",\n"
            f"  \"basis\": \"{basis}\",\n"
            "  \"current_data\": {\n"
            "    \"path\": \"currents.bin\",\n"
            "    \"ordering\": \"J1, M1, J2, M2; one block per RWG edge\",\n"
            "    \"precision\": \"complex128\",\n"
            "    \"byte_order\": \"little-endian\",\n"
            "    \"complex_encoding\": \"interleaved real-imaginary float64\",\n"
            "    \"physical_currents\": true,\n"
            f"    \"complex_value_count\": {currents.size}\n"
            "  },\n"
            "  \"solver\": {\n"
            f"    \"rhs_assembly_seconds\": {_g(rhs_seconds)},\n"
            f"    \"residual_seconds\": {_g(metrics['residual_seconds'])},\n"
            f"    \"residual_computed\": {'true' if metrics['residual_computed'] else 'false'},\n"
            f"    \"scaled_rhs_norm\": {_g(metrics['rhs_norm'])},\n"
            f"    \"maximum_j1_coefficient\": {_g(mc[0])},\n"
            f"    \"maximum_m1_coefficient\": {_g(mc[1])},\n"
            f"    \"maximum_j2_coefficient\": {_g(mc[2])},\n"
            f"    \"maximum_m2_coefficient\": {_g(mc[3])}")
    if metrics["residual_computed"]:
        text += (f",\n    \"scaled_absolute_residual\": {_g(metrics['absolute_residual'])}"
                 f",\n    \"scaled_relative_residual\": {_g(metrics['relative_residual'])}\n")
    else:
        text += "\n"
    text += "  }\n}\n"
    path.write_text(text)


def write_batch_metrics(path: Path, mesh, metrics: dict, cases, basis: str, preparation_seconds: float) -> None:
    """batch_metrics.json with the reference's keys (anisotropic_sphere_app.cpp:609-652);
    device_preparation_seconds is the host loading of mesh and records."""
    ids = ", ".join(f'"{c.id}"' for c in cases)
    text = ("{\n"
            "  \"schema_version\": 2,\n"
            "  \"artifact\": \"anisotropic_sphere_app_batch\",\n"
            f"  \"case_ids\": [{ids}],\n"
            "  \"mesh\": {\n"
            f"    \"vertex_count\": {mesh.vertices.shape[0]},\n"
            f"    \"face_count\": {mesh.num_faces},\n"
            f"    \"edge_count\": {mesh.num_edges}\n"
            "  },\n"
            "  \"solver\": {\n"
            "    \"method\": \"dense_lu_batch\",\n"
            "    \"scaling\": \"eta0\",\n"
            f"    \"basis\": \"{basis}\",\n"
            f"    \"case_count\": {len(cases)},\n"
            f"    \"matrix_dimension\": {metrics['matrix_dimension']},\n"
            f"    \"dense_matrix_bytes\": {metrics['dense_matrix_bytes']},\n"
            f"    \"device_preparation_seconds\": {_g(preparation_seconds)},\n"
            f"    \"matrix_assembly_seconds\": {_g(metrics['assembly_seconds'])},\n"
            f"    \"factorization_seconds\": {_g(metrics['factorization_seconds'])},\n"
            f"    \"solve_seconds\": {_g(metrics['solve_seconds'])},\n"
            f"    \"residual_matrix_assembly_seconds\": {_g(metrics['residual_seconds'])}\n"
            "  }\n}\n")
    path.write_text(text)


def run(a: Arguments, out=None) -> int:
    """anisotropic_sphere_app.cpp:676-775 on the C ABI."""
    out = out if out is not None else sys.stdout
    import sieb200
    from ..io import load_face_tensors, write_physical_currents
    t_prep = time.perf_counter()
    mesh = sieb200.load_obj(a.mesh_path)
    tensors = load_face_tensors(a.tensor_path, mesh.num_faces)
    N = 4 * mesh.num_edges
    gib = N * N * 16 / 1024.0 ** 3
    print("Loaded spherical GSTC SIE inputs\n"
          f"  basis: {a.basis}\n  vertices: {mesh.vertices.shape[0]}\n  faces: {mesh.num_faces}\n"
          f"  edges: {mesh.num_edges}\n  tensor_records: {tensors.shape[0]}\n  matrix_dimension: {N}\n"
          f"  dense_matrix_gib: {gib:.3f}\nStarting dense CUDA solve...", file=out, flush=True)
    options = sieb200.GstcSieOptions(
        frequency_hz=a.frequency_hz,
        interior=sieb200.IsotropicMedium(a.epsilon_r_interior, a.mu_r_interior),
        exterior=sieb200.IsotropicMedium(a.epsilon_r_exterior, a.mu_r_exterior),
        quadrature_rule=a.quadrature_rule, singularity_threshold_lambda0=a.singularity_threshold_lambda0,
        tensors_are_uniform=False, compute_residual=a.compute_residual, basis=a.basis,
        solver=a.solver, tolerance=a.tolerance)
    observations = None
    if a.evaluate_fields:
        observations = make_observation_samples(a, sieb200.infer_sphere_radius(mesh))
    ctx = sieb200.default_context()
    cases = [sieb200.GstcExcitationCase(interior=c.interior, exterior=c.exterior) for c in a.cases]
    preparation = time.perf_counter() - t_prep
    results = sieb200.solve_gstc_dense_batch(mesh, tensors, options, cases, ctx=ctx)
    root = Path(a.output_directory)
    root.mkdir(parents=True, exist_ok=True)
    m0 = results[0].metrics
    write_batch_metrics(root / "batch_metrics.json", mesh, m0, a.cases, a.basis, preparation)
    print(f"Spherical anisotropic GSTC SIE\n  basis: {a.basis}\n  cases: {len(a.cases)}\n"
          f"  matrix_dimension: {N}\n  matrix_assembly_seconds: {m0['assembly_seconds']:.6e}\n"
          f"  factorization_seconds: {m0['factorization_seconds']:.6e}\n"
          f"  solve_seconds: {m0['solve_seconds']:.6e}", file=out)
    for c, r in zip(a.cases, results):
        d = root / "cases" / c.id
        d.mkdir(parents=True, exist_ok=True)
        write_physical_currents(d / "currents.bin", r.currents)
        write_solver_metrics(d / "solver_metrics.json", c.id, r.currents, r.metrics, a.basis, 0.0)
        print(f"Case {c.id}\n  outputs: {d}", file=out)
        if r.metrics["residual_computed"]:
            print(f"  scaled_relative_residual: {r.metrics['relative_residual']:.6e}", file=out)
        if observations is not None:
            t0 = time.perf_counter()
            fields = evaluate_field_representations(mesh, options, r.currents, observations, c, ctx=ctx)
            write_field_outputs(d, observations, fields)
            print(f"  observation_points: {observations.points.shape[0]}\n"
                  f"  field_evaluation_and_output_seconds: {time.perf_counter() - t0:.6e}", file=out)
    return 0


def main(argv: Optional[list[str]] = None) -> int:
    argv = list(sys.argv if argv is None else argv)
    program = argv[0] if argv else PROGRAM
    try:
        a = parse_arguments(argv)
    except UsageExit:
        print(usage(program), end="")
        return 0
    except (ValueError, RuntimeError) as e:
        print(f"{PROGRAM}: {e}\n", file=sys.stderr, flush=True)
        print(usage(program), end="")
        return 2
    try:
        return run(a)
    except Exception as e:  # the reference reports every std::exception and exits 1
        print(f"{PROGRAM}: {e}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
