"""CPU: the C-ABI library loads, exports everything include/sieb200.h declares,
and its host-side logic (rules, edge numbering, defaults, validation) works
without a GPU."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import GoldenMesh

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "sieb200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sieb200_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import sieb200
    lib = sieb200.lib()
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # and the Python binding knows every one of them
    assert set(names) <= set(sieb200.exported_symbols()), set(names) - set(sieb200.exported_symbols())


def test_library_is_in_tree_and_built_for_sm100a():
    import sieb200
    p = sieb200.library_path()
    assert p.exists() and p.parent.name == "sieb200"
    data = p.read_bytes()
    assert b"sm_100a" in data or b"sm_100" in data


def test_quadrature_rule_abi_matches_golden(golden):
    import sieb200
    lib = sieb200.lib()
    for rule in range(1, 21):
        n = lib.sieb200_quadrature_rule(rule, None, None)
        p = np.zeros(2 * n, np.float32)
        w = np.zeros(n, np.float32)
        assert lib.sieb200_quadrature_rule(rule, p.ctypes.data, w.ctypes.data) == n
        assert np.array_equal(p, golden[f"rule{rule}_points"])
        assert np.array_equal(w, golden[f"rule{rule}_weights"])
    assert lib.sieb200_quadrature_rule(0, None, None) == -1
    assert lib.sieb200_quadrature_rule(21, None, None) == -1


def test_build_edges_matches_reference_numbering(golden):
    import sieb200
    for name in ("L0", "L1r05"):
        g = GoldenMesh(golden, name)
        edges, fe = sieb200.build_edges(g.faces)
        assert np.array_equal(edges, g.edges) and np.array_equal(fe, g.faces_edges)


def test_options_defaults_follow_reference():
    from sieb200 import _lib
    pec = _lib.default_options(_lib.PEC_EFIE)
    assert pec.quadrature_rule == 7 and pec.vacuum_permittivity == 8.8541878128e-12
    assert pec.vacuum_permeability == 1.25663706212e-6 and pec.singularity_threshold_lambda0 == 0.1
    die = _lib.default_options(_lib.PMCHWT)
    assert die.quadrature_rule == 17
    gst = _lib.default_options(_lib.GSTC)
    assert gst.quadrature_rule == 17 and gst.vacuum_permittivity == 8.8541878188e-12
    assert gst.vacuum_permeability == 1.25663706127e-6 and gst.basis == 0


def _call_solve(mesh, **over):
    from sieb200 import _lib
    o = _lib.default_options(_lib.PEC_EFIE)
    o.frequency_hz = 299792458.0
    for k, v in over.items():
        setattr(o, k, v)
    src = _lib.Source()
    src.kind, src.region = 0, 2
    src.a[:] = [1.0, 0.0, 0.0]
    src.b[:] = [0.0, 0.0, 1.0]
    out = np.zeros(mesh.num_edges, np.complex128)
    m = _lib.Metrics()
    return _lib.lib().sieb200_solve_pec_dense(None, ctypes.byref(mesh.as_c()), ctypes.byref(o),
                                              ctypes.byref(src), out.ctypes.data, ctypes.byref(m))


@pytest.mark.parametrize("field,value,msg", [
    ("frequency_hz", 0.0, "frequency must be positive"),
    ("quadrature_rule", 21, "Dunavant quadrature rule must be in [1, 20]"),
    ("singularity_threshold_lambda0", 0.0, "singularity threshold"),
    ("eps_r_exterior", -1.0, "permittivities and permeabilities must be positive"),
    ("vacuum_permittivity", 0.0, "vacuum permittivity and permeability must be positive"),
])
def test_validation_errors_mirror_reference(field, value, msg):
    import sieb200
    from sieb200 import _lib
    mesh = sieb200.icosphere(1.0, 0)
    assert _call_solve(mesh, **{field: value}) == _lib.INVALID_ARG
    assert msg in _lib.lib().sieb200_last_error().decode()


@pytest.mark.parametrize("over,msg", [
    (dict(variant=3), "unknown formulation variant"),
    (dict(ntl_form=2), "unknown nTL integral form"),
    (dict(variant=2, ntl_form=1), "line nTL form requires N-EFIE"),
    (dict(variant=0, ntl_form=1), "line nTL form requires N-EFIE"),
    (dict(variant=1, ntl_form=1, line_quadrature_points=0), "Gauss-Legendre point count must be in [1, 20]"),
    (dict(variant=1, ntl_form=1, line_quadrature_points=21), "Gauss-Legendre point count must be in [1, 20]"),
])
def test_variant_validation_mirrors_reference(over, msg):
    # pec_solver.cu:91-97: checked before any device work (null context here)
    import sieb200
    from sieb200 import _lib
    mesh = sieb200.icosphere(1.0, 0)
    assert _call_solve(mesh, **over) == _lib.INVALID_ARG
    assert msg in _lib.lib().sieb200_last_error().decode()
    assert "context" not in _lib.lib().sieb200_last_error().decode()


def test_null_context_is_rejected_after_validation():
    import sieb200
    from sieb200 import _lib
    mesh = sieb200.icosphere(1.0, 0)
    assert _call_solve(mesh) == _lib.INVALID_ARG
    assert "context" in _lib.lib().sieb200_last_error().decode()


def test_python_layer_rejects_bad_inputs():
    import sieb200
    mesh = sieb200.icosphere(1.0, 0)
    with pytest.raises(ValueError):
        sieb200.solvers.to_c_options(sieb200.PecOptions(frequency_hz=1.0, solver="nope"), 0)
    with pytest.raises(ValueError):
        sieb200.solvers._tensor_array(mesh, np.zeros(31), True)
    with pytest.raises(ValueError):
        sieb200.solvers.to_c_options(sieb200.GstcSieOptions(frequency_hz=1.0, basis="polar"), 2)


def test_header_compiles_as_c_and_links(tmp_path):
    # A plain C caller (what a reference-side binding compiles against) built
    # with gcc against include/sieb200.h and the in-tree library: struct
    # layout, defaults of the variant fields and two host-only entry points.
    import subprocess
    import sieb200
    src = tmp_path / "caller.c"
    src.write_text(r"""
#include <stddef.h>
#include <stdio.h>
#include "sieb200.h"
int main(void) {
    sieb200_options o;
    if (sieb200_options_default(SIEB200_PMCHWT, &o) != SIEB200_OK) return 1;
    if (o.variant != SIEB200_VARIANT_T || o.ntl_form != SIEB200_NTL_SURFACE || o.line_quadrature_points != 20)
        return 2;
    if (o.quadrature_rule != 17 || o.solver != SIEB200_SOLVER_LU_CUSOLVER) return 3;
    if (sieb200_quadrature_rule(20, NULL, NULL) != 79) return 4;
    const int32_t faces[12] = {0, 1, 2, 0, 3, 1, 1, 3, 2, 2, 3, 0};
    int32_t edges[24], fe[12];
    int64_t ne = 0;
    if (sieb200_build_edges(faces, 4, edges, fe, &ne) != SIEB200_OK || ne != 6) return 5;
    if (sieb200_version() != SIEB200_ABI_VERSION) return 6;
    printf("%d %zu %zu %zu\n", sieb200_version(), sizeof(sieb200_options), sizeof(sieb200_sweep_instance),
           offsetof(sieb200_sweep_instance, currents_out));
    return 0;
}
""")
    lib = sieb200.library_path()
    exe = tmp_path / "caller"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", str(ROOT / "include"), str(src), "-o", str(exe),
                        str(lib), f"-Wl,-rpath,{lib.parent}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stderr)
    import ctypes
    from sieb200 import _lib
    assert int(r.stdout.split()[1]) == ctypes.sizeof(_lib.Options)
    assert int(r.stdout.split()[2]) == ctypes.sizeof(_lib.SweepInstance)
    assert int(r.stdout.split()[3]) == _lib.SweepInstance.currents_out.offset


def test_sweep_validation_without_gpu_work():
    """The sweep refuses empty input and a zero lane count before any work."""
    import ctypes
    import sieb200
    from sieb200 import _lib
    lib = _lib.lib()
    arr = (_lib.SweepInstance * 1)()
    assert lib.sieb200_solve_gstc_sweep(None, arr, 1, 1, None) == _lib.INVALID_ARG
    assert lib.sieb200_solve_gstc_sweep(None, arr, 0, 1, None) == _lib.INVALID_ARG
    secs = ctypes.c_double()
    assert lib.sieb200_solve_gstc_sweep(None, None, 1, 1, ctypes.byref(secs)) == _lib.INVALID_ARG
    _ = sieb200  # the package exposes the call as solve_gstc_sweep_batched
