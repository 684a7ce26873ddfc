"""The package's box-mesh generator against the reference's generateBox + Mesh::build arrays."""
import numpy as np

from conftest import load_golden, golden_names
from voluma_b200 import mesh as vm
import pytest

KEYS = {"owner": "owner", "neighbour": "neighbour", "V": "V", "C": "C", "Sf": "Sf", "magSf": "magSf", "Cf": "Cf",
        "d": "d", "w": "w", "deltaCoeffs": "deltaCoeffs", "ndc": "ndc", "corrVecs": "corrVecs",
        "skewVecs": "skewVecs", "patchStart": "patch_start", "patchSize": "patch_size"}


@pytest.mark.parametrize("name", golden_names())
def test_box_mesh_matches_reference(name):
    g = load_golden(name)
    M = vm.box_mesh(tuple(g["spec_n"]), tuple(g["spec_lo"]), tuple(g["spec_hi"]), tuple(g["spec_periodic"]),
                    bool(g["spec_two_d"]), tuple(g["spec_beta"]), points=g.get("points"))
    assert (M["n_cells"], M["n_internal_faces"], M["n_faces"]) == (g["n_cells"], g["n_internal_faces"], g["n_faces"])
    for rk, mk in KEYS.items():
        a, b = g[rk], M[mk]
        assert a.shape == b.shape, rk
        if a.dtype.kind == "i":
            assert np.array_equal(a, b), rk
        else:
            # bit-identical except through libm tanh in stretched boxes
            np.testing.assert_allclose(b, a, rtol=1e-13, atol=1e-15, err_msg=rk)
    assert M["skewed"] == bool(g["sizes"][6])
    assert M["empty_dir"] == int(g["sizes"][5])


def test_jitter_keeps_boundary():
    n = (6, 5, 4)
    p0 = vm.box_points(n)
    p1 = vm.jitter_interior(p0, n, 0.2, 1)
    P0 = p0.reshape(5, 6, 7, 3)
    P1 = p1.reshape(5, 6, 7, 3)
    for sl in [(0,), (-1,), (slice(None), 0), (slice(None), -1), (slice(None), slice(None), 0),
               (slice(None), slice(None), -1)]:
        assert np.array_equal(P0[sl], P1[sl])
    assert not np.array_equal(P0[1:-1, 1:-1, 1:-1], P1[1:-1, 1:-1, 1:-1])


def test_poisson_matrix_row_sums():
    M = vm.box_mesh((5, 4, 3), periodic=(1, 1, 1))
    d, up = vm.poisson_matrix(M, ref_cell=None)
    y = np.zeros(M["n_cells"])
    np.add.at(y, M["owner"][:M["n_internal_faces"]], up)
    np.add.at(y, M["neighbour"], up)
    np.testing.assert_allclose(d + y, 0.0, atol=1e-12)
