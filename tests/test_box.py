"""Box-mesh detection behind the structured level-0 kernels (host only, no GPU): the face arrays of
generateBox meshes are recognised with their shape and periodicity, every golden mesh is one, and
face arrays that are not exactly a box's are refused."""
import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import mesh as vm


@pytest.mark.parametrize("n,periodic,two_d,layout", [
    ((8, 8, 8), (1, 1, 1), False, True),
    ((7, 5, 3), (0, 0, 0), False, True),      # odd x extent: padding slots inside the colour groups
    ((16, 16, 1), (0, 0, 0), True, True),     # 2D cavity
    ((6, 4, 4), (1, 0, 1), False, True),      # channel-like: periodic x and z
    ((5, 4, 4), (1, 0, 0), False, False),     # odd periodic extent: three colours, general layout
    ((4, 3, 2), (0, 0, 0), False, True),
])
def test_box_shapes_are_detected(n, periodic, two_d, layout):
    m = vm.box_mesh(n, periodic=periodic, two_d=two_d)
    b = vb.box_shape(m["n_cells"], m["owner"], m["neighbour"], m["magSf"], m["ndc"])
    assert b is not None
    assert b["n"] == tuple(n)
    assert b["periodic"] == tuple(bool(p) and not (d == 2 and two_d) for d, p in enumerate(periodic))
    assert b["layout"] == layout


def test_golden_meshes_are_boxes(golden):
    b = vb.box_shape(golden["n_cells"], golden["owner"], golden["neighbour"][:golden["n_internal_faces"]],
                     golden["magSf"], golden["ndc"])
    assert b is not None and int(np.prod(b["n"])) == golden["n_cells"]


def test_non_box_face_arrays_are_refused():
    m = vm.box_mesh((6, 5, 4))
    own, nei = m["owner"][:m["n_internal_faces"]].copy(), m["neighbour"].copy()
    # two faces swapped: same graph, not the box's face order
    own[[3, 4]], nei[[3, 4]] = own[[4, 3]], nei[[4, 3]]
    assert vb.box_shape(m["n_cells"], own, nei) is None
    # one face removed
    o2, n2 = m["owner"][:m["n_internal_faces"] - 1], m["neighbour"][:-1]
    assert vb.box_shape(m["n_cells"], o2, n2) is None
    # a periodic direction of two cells: its cyclic faces duplicate the internal ones
    p = vm.box_mesh((2, 4, 4), periodic=(1, 0, 0))
    assert vb.box_shape(p["n_cells"], p["owner"][:p["n_internal_faces"]], p["neighbour"]) is None
