"""The oracle's library-free sphere generators (used by the reference arm of
the benchmark and by the config-size parity checks) give exactly the meshes
the library generates: vertices bit-equal, faces, edges and the face-edge map
equal."""

import numpy as np
import pytest


@pytest.mark.parametrize("kind,args", [("geodesic_sphere", (0.5, 10)), ("geodesic_sphere", (1.0, 12)),
                                       ("icosphere", (1.0, 3)), ("icosphere", (0.5, 1))])
def test_oracle_mesh_equals_library_mesh(kind, args):
    import sieb200
    from oracle import oracle as O
    a = getattr(O, kind)(*args)
    b = getattr(sieb200, kind)(*args)
    assert np.array_equal(a.vertices, b.vertices)
    assert np.array_equal(a.faces, b.faces)
    assert np.array_equal(a.edges, b.edges)
    assert np.array_equal(a.faces_edges, b.faces_edges)
