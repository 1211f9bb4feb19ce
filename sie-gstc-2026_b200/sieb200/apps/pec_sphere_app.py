"""Drop-in for applications/pec_sphere/pec_sphere_app.cpp on the sieb200 C
ABI: T-EFIE, N-EFIE (surface or line nTL form) or N-MFIE for a PEC sphere lit
by a unit x-polarised plane wave travelling +z in region 2. Same flags,
messages and outputs under --output-dir: currents.csv (edge, J2 re/im/abs),
zx_fields.csv and radial_fields.csv (incident minus the surface integrals),
matrix.npy and matrix_edges.csv with --export-matrix; --currents-file
evaluates the fields of a saved currents.csv without solving.
"""

from __future__ import annotations

import math
import re
import sys
from dataclasses import dataclass
from pathlib import Path
from typing import Optional

import numpy as np

_STOD = re.compile(r"\s*[+-]?((\d+\.?\d*|\.\d+)([eE][+-]?\d+)?|inf(inity)?|nan)", re.IGNORECASE)
_STOI = re.compile(r"\s*[+-]?\d+")


def _stod(text: str) -> float:
    """std::stod: the longest numeric prefix; no prefix -> invalid_argument."""
    m = _STOD.match(text)
    if m is None:
        raise ValueError("stod")
    return float(m.group(0))


def _stoi(text: str) -> int:
    m = _STOI.match(text)
    if m is None:
        raise ValueError("stoi")
    v = int(m.group(0))
    if not -2**31 <= v < 2**31:
        raise ValueError("stoi")
    return v


@dataclass
class Arguments:
    mesh_path: str = ""
    output_directory: str = ""
    currents_file: str = ""
    frequency_hz: float = 0.0
    epsilon_r_exterior: float = 1.0
    mu_r_exterior: float = 1.0
    formulation: str = "TEfie"
    ntl_form: str = "Surface"
    line_quadrature_points: int = 20
    quadrature_rule: int = 7
    singularity_threshold_lambda0: float = 0.1
    compute_residual: bool = True
    export_matrix: bool = False
    evaluate_fields: bool = True
    zx_grid_size: int = 80
    zx_span_radii: float = 2.0
    radial_points: int = 100
    radial_theta_degrees: float = 45.0
    radial_phi_degrees: float = 0.0
    radial_min_radii: float = 0.05
    radial_max_radii: float = 2.0


class UsageExit(Exception):
    pass


def usage(name: str) -> str:
    return ("Usage: " + name + " --mesh PATH --output-dir PATH --frequency-hz HZ [options]\n"
            "  --epsilon-r-exterior V          Default: 1\n"
            "  --mu-r-exterior V               Default: 1\n"
            "  --formulation [t-efie|n-efie|n-mfie]  Default: t-efie; t/n aliases accepted\n"
            "  --ntl-form [surface|line]       N-EFIE only; Form B or A, default: surface\n"
            "  --line-quadrature-points N      N-EFIE Form A only, default: 20\n"
            "  --quadrature-rule N             Dunavant rule, default: 7\n"
            "  --singularity-threshold-lambda0 V  Default: 0.1\n"
            "  --no-residual                   Skip the matrix residual\n"
            "  --export-matrix                 Save the pre-LU complex matrix as matrix.npy\n"
            "  --currents-file PATH            Evaluate saved J2 without solving again\n"
            "  --no-fields                     Skip field evaluation\n"
            "  --zx-grid-size N                ZX points per axis, default: 80; 0 skips grid\n"
            "  --zx-span-radii V               ZX half-span in sphere radii, default: 2\n"
            "  --radial-points N               Radial samples, default: 100; 0 skips cut\n"
            "  --radial-theta-degrees V        Radial theta, default: 45\n"
            "  --radial-phi-degrees V          Radial phi, default: 0\n"
            "  --radial-min-radii V            Minimum r/a, default: 0.05\n"
            "  --radial-max-radii V            Maximum r/a, default: 2\n"
            "Source: unit x-polarized plane wave traveling +z in region 2.\n")


_REALS = {"--frequency-hz": "frequency_hz", "--epsilon-r-exterior": "epsilon_r_exterior",
          "--mu-r-exterior": "mu_r_exterior", "--singularity-threshold-lambda0": "singularity_threshold_lambda0",
          "--zx-span-radii": "zx_span_radii", "--radial-theta-degrees": "radial_theta_degrees",
          "--radial-phi-degrees": "radial_phi_degrees", "--radial-min-radii": "radial_min_radii",
          "--radial-max-radii": "radial_max_radii"}
_INTS = {"--line-quadrature-points": "line_quadrature_points", "--quadrature-rule": "quadrature_rule",
         "--zx-grid-size": "zx_grid_size", "--radial-points": "radial_points"}


def parse(argv: list[str]) -> Arguments:
    """pec_sphere_app.cpp:65-144."""
    a = Arguments()
    i = 1

    def value_after() -> str:
        nonlocal i
        i += 1
        if i >= len(argv):
            raise ValueError("missing option value")
        return argv[i]

    while i < len(argv):
        option = argv[i]
        if option in ("--help", "-h"):
            raise UsageExit()
        elif option == "--mesh":
            a.mesh_path = value_after()
        elif option == "--output-dir":
            a.output_directory = value_after()
        elif option in _REALS:
            setattr(a, _REALS[option], _stod(value_after()))
        elif option in _INTS:
            setattr(a, _INTS[option], _stoi(value_after()))
        elif option == "--formulation":
            v = value_after()
            forms = {"t": "TEfie", "t-efie": "TEfie", "n": "NEfie", "n-efie": "NEfie", "n-mfie": "NMfie"}
            if v not in forms:
                raise ValueError("--formulation must be t-efie, n-efie, or n-mfie")
            a.formulation = forms[v]
        elif option == "--ntl-form":
            v = value_after()
            if v not in ("surface", "line"):
                raise ValueError("--ntl-form must be surface or line")
            a.ntl_form = "Surface" if v == "surface" else "Line"
        elif option == "--no-residual":
            a.compute_residual = False
        elif option == "--export-matrix":
            a.export_matrix = True
        elif option == "--currents-file":
            a.currents_file = value_after()
        elif option == "--no-fields":
            a.evaluate_fields = False
        else:
            raise ValueError("unknown option: " + option)
        i += 1
    if not a.mesh_path or not a.output_directory or not a.frequency_hz > 0:
        raise ValueError("--mesh, --output-dir, and positive --frequency-hz are required")
    if (a.zx_grid_size < 0 or a.zx_grid_size == 1 or a.radial_points < 0 or a.radial_points == 1
            or not a.zx_span_radii > 0 or not a.radial_min_radii >= 0
            or not a.radial_max_radii > a.radial_min_radii):
        raise ValueError("invalid field sampling range or point count")
    if a.currents_file and not a.evaluate_fields:
        raise ValueError("--currents-file requires field evaluation")
    if a.currents_file and a.export_matrix:
        raise ValueError("--export-matrix requires solving, not --currents-file")
    return a


def options_of(a: Arguments):
    import sieb200
    return sieb200.PecOptions(frequency_hz=a.frequency_hz,
                              exterior=sieb200.IsotropicMedium(a.epsilon_r_exterior, a.mu_r_exterior),
                              quadrature_rule=a.quadrature_rule,
                              singularity_threshold_lambda0=a.singularity_threshold_lambda0,
                              compute_residual=a.compute_residual, formulation=a.formulation,
                              ntl_form=a.ntl_form, line_quadrature_points=a.line_quadrature_points)


def write_matrix_npy(path: Path, Z: np.ndarray) -> None:
    """NumPy 1.0 format, complex128, Fortran order, header padded to 16 bytes
    (pec_sphere_app.cpp:150-181)."""
    n = Z.shape[0]
    header = "{'descr': '<c16', 'fortran_order': True, 'shape': (" + f"{n}, {n}" + "), }"
    while (10 + len(header) + 1) % 16 != 0:
        header += " "
    header += "\n"
    body = np.asfortranarray(Z, dtype=np.complex128).tobytes(order="F")
    path.write_bytes(b"\x93NUMPY\x01\x00" + len(header).to_bytes(2, "little") + header.encode() + body)


def sphere_radius(mesh) -> float:
    r = np.sqrt((np.asarray(mesh.vertices) ** 2).sum(axis=1))
    s = 0.0
    for v in r:  # sequential sum, as the reference accumulates
        s += float(v)
    return s / r.size


@dataclass
class Observations:
    points: np.ndarray
    regions: np.ndarray
    zx_count: int


def make_observations(a: Arguments, radius: float) -> Observations:
    """pec_sphere_app.cpp:197-228."""
    pts, reg = [], []
    if a.zx_grid_size > 0:
        span = a.zx_span_radii * radius
        n = a.zx_grid_size
        for iz in range(n):
            z = span * (2.0 * iz / (n - 1) - 1.0)
            for ix in range(n):
                x = span * (2.0 * ix / (n - 1) - 1.0)
                pts.append((x, 0.0, z))
                reg.append(1 if math.hypot(x, z) < radius else 2)
    zx = len(pts)
    if a.radial_points > 0:
        theta = a.radial_theta_degrees * math.pi / 180.0
        phi = a.radial_phi_degrees * math.pi / 180.0
        for step in range(a.radial_points):
            f = step / (a.radial_points - 1)
            r = radius * (a.radial_min_radii + f * (a.radial_max_radii - a.radial_min_radii))
            pts.append((r * math.sin(theta) * math.cos(phi), r * math.sin(theta) * math.sin(phi),
                        r * math.cos(theta)))
            reg.append(1 if r < radius else 2)
    return Observations(np.array(pts, dtype=np.float64).reshape(-1, 3), np.array(reg, dtype=np.int32), zx)


def read_currents(path: str, edge_count: int) -> np.ndarray:
    """pec_sphere_app.cpp:230-256."""
    try:
        lines = Path(path).read_text().splitlines()
    except OSError:
        raise RuntimeError("cannot open " + str(path)) from None
    if not lines or lines[0] != "edge,J2_real,J2_imag,J2_abs":
        raise RuntimeError("unexpected current CSV header: " + str(path))
    out = []
    for line in lines[1:]:
        parts = line.split(",")
        if len(parts) < 4 or _stoi(parts[0]) != len(out):
            raise RuntimeError("invalid current CSV row: " + line)
        re_, im = _stod(parts[1]), _stod(parts[2])
        if not (math.isfinite(re_) and math.isfinite(im)):
            raise RuntimeError("non-finite current CSV row: " + line)
        out.append(complex(re_, im))
    if len(out) != edge_count:
        raise RuntimeError("current CSV edge count does not match mesh")
    return np.array(out, dtype=np.complex128)


def _e(x: float) -> str:
    """std::scientific with setprecision(12)."""
    return f"{x:.12e}"


def write_field_csv(path: Path, obs: Observations, E: np.ndarray, H: np.ndarray, begin: int, end: int) -> None:
    lines = ["x,y,z,region,E_x_re,E_x_im,E_y_re,E_y_im,E_z_re,E_z_im,"
             "H_x_re,H_x_im,H_y_re,H_y_im,H_z_re,H_z_im"]
    for i in range(begin, end):
        p = obs.points[i]
        row = [_e(p[0]), _e(p[1]), _e(p[2]), str(int(obs.regions[i]))]
        for c in range(3):
            row += [_e(E[i, c].real), _e(E[i, c].imag)]
        for c in range(3):
            row += [_e(H[i, c].real), _e(H[i, c].imag)]
        lines.append(",".join(row))
    path.write_text("\n".join(lines) + "\n")


def evaluate_fields(mesh, j2: np.ndarray, a: Arguments, options, source, out=None, ctx=None) -> None:
    """Incident minus the surface integral of J2 (M = 0) in region 2's medium
    (pec_sphere_app.cpp:279-312)."""
    import sieb200
    out = out if out is not None else sys.stdout
    obs = make_observations(a, sphere_radius(mesh))
    print(f"Evaluating {obs.points.shape[0]} field points inside and outside the sphere...", file=out, flush=True)
    QE, QH = sieb200.evaluate_surface_integral_fields(mesh, j2, np.zeros_like(j2), obs.points, a.frequency_hz,
                                                      options.exterior, a.quadrature_rule,
                                                      options.vacuum_permittivity, options.vacuum_permeability,
                                                      ctx=ctx)
    IE, IH = sieb200.incident_fields(obs.points, source, options, ctx=ctx)
    E, H = IE - QE, IH - QH
    root = Path(a.output_directory)
    if obs.zx_count > 0:
        write_field_csv(root / "zx_fields.csv", obs, E, H, 0, obs.zx_count)
        print(f"zx_fields_csv=\"{root / 'zx_fields.csv'}\"", file=out)
    if obs.points.shape[0] > obs.zx_count:
        write_field_csv(root / "radial_fields.csv", obs, E, H, obs.zx_count, obs.points.shape[0])
        print(f"radial_fields_csv=\"{root / 'radial_fields.csv'}\"", file=out)


def run(a: Arguments, out=None) -> int:
    """pec_sphere_app.cpp:317-388 on the C ABI."""
    out = out if out is not None else sys.stdout
    import sieb200
    mesh = sieb200.load_obj(a.mesh_path)
    options = options_of(a)
    source = sieb200.PlaneWaveExcitation(electric_amplitude=(1.0, 0.0, 0.0), propagation_direction=(0.0, 0.0, 1.0),
                                         region=sieb200.EXTERIOR)
    root = Path(a.output_directory)
    root.mkdir(parents=True, exist_ok=True)
    ctx = sieb200.default_context()
    if a.currents_file:
        evaluate_fields(mesh, read_currents(a.currents_file, mesh.num_edges), a, options, source, out, ctx)
        return 0
    print({"NMfie": "N-MFIE: (1/2 M - nTK2)(J2) = <f x n, H_inc,2>",
           "NEfie": "N-EFIE: i*omega*mu2*nTL2(J2) = <f x n, E_inc,2>",
           "TEfie": "T-EFIE: i*omega*mu2*TL2(J2) = <f, E_inc,2>"}[a.formulation], file=out)
    print(f"mesh=\"{a.mesh_path}\" faces={mesh.num_faces} edges={mesh.num_edges}\n"
          f"quadrature_rule={a.quadrature_rule} singularity_threshold_lambda0={a.singularity_threshold_lambda0:g}",
          file=out)
    if a.formulation == "NMfie":
        print("operator_quadrature=Form A nTK (zero 1D points)", file=out)
    if a.formulation == "NEfie":
        print("ntl_form=" + ("line (Form A)" if a.ntl_form == "Line" else "surface (Form B)"), file=out)
    r = sieb200.solve_pec_dense(mesh, options, source, ctx=ctx)
    m = r.metrics
    print(f"matrix_dimension={m['matrix_dimension']}\nassembly_seconds={m['assembly_seconds']:.9g}\n"
          f"solve_seconds={m['solve_seconds']:.9g}\nmaximum_abs_J2={m['maximum_coefficient'][0]:.9g}", file=out)
    if m["residual_computed"]:
        print(f"relative_residual={m['relative_residual']:.9g}", file=out)
    if a.export_matrix:
        write_matrix_npy(root / "matrix.npy", sieb200.assemble_matrix(mesh, options, ctx=ctx))
        print(f"matrix_npy=\"{root / 'matrix.npy'}\"", file=out)
        edges = ["edge,vertex_a,vertex_b"] + [f"{e},{v[0]},{v[1]}" for e, v in enumerate(mesh.edges)]
        (root / "matrix_edges.csv").write_text("\n".join(edges) + "\n")
        print(f"matrix_edges_csv=\"{root / 'matrix_edges.csv'}\"", file=out)
    rows = ["edge,J2_real,J2_imag,J2_abs"] + [f"{e},{v.real:.17g},{v.imag:.17g},{abs(v):.17g}"
                                              for e, v in enumerate(r.currents)]
    (root / "currents.csv").write_text("\n".join(rows) + "\n")
    print(f"currents_csv=\"{root / 'currents.csv'}\"", file=out)
    if a.evaluate_fields:
        evaluate_fields(mesh, r.currents, a, options, source, out, ctx)
    return 0


def main(argv: Optional[list[str]] = None) -> int:
    argv = list(sys.argv if argv is None else argv)
    try:
        a = parse(argv)
    except UsageExit:
        print(usage(argv[0] if argv else "pec_sphere_app"), end="")
        return 0
    except (ValueError, RuntimeError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    try:
        return run(a)
    except Exception as e:  # the reference reports every std::exception and exits 1
        print(f"Error: {e}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
