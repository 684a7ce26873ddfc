"""The C-ABI library: it loads, exports every entry point include/voluma_b200.h declares, and its
host-only parts (the GAMG topology the device uses) agree with the reference - no GPU needed."""
import os
import re

import numpy as np

from conftest import ROOT, golden_hierarchy, has_gpu
import voluma_b200 as vb
from voluma_b200 import _ffi
from oracle import restate as ro


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "voluma_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vlm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = vb.load()
    decl = declared_symbols()
    assert len(decl) >= 20
    for name in decl:
        assert hasattr(L, name), name
    assert sorted(_ffi.EXPORTS) == decl


def test_topology_matches_reference_hierarchy(golden):
    t = vb.topology(golden["n_cells"], golden["owner"], golden["neighbour"], golden["magSf"], golden["ndc"])
    ref_h = golden_hierarchy(golden)
    assert len(t) == len(ref_h)
    for a, b in zip(t, ref_h):
        for f in ("l", "u", "weight", "agg", "faceMap", "faceFlip"):
            assert np.array_equal(a[f], b[f]), f


def test_topology_colouring_is_proper_and_matches_oracle(golden):
    t = vb.topology(golden["n_cells"], golden["owner"], golden["neighbour"], golden["magSf"], golden["ndc"])
    o = ro.hierarchy(golden, colours=True)
    for a, b in zip(t, o):
        assert np.array_equal(a["colour"], b["colour"])
        assert a["ncolours"] == b["ncolours"]
        c = a["colour"]
        assert np.all(c[a["l"]] != c[a["u"]])  # no face joins two cells of one colour


def test_topology_rejects_self_coupled_faces():
    own = np.array([0, 1], np.int32)
    nei = np.array([1, 1], np.int32)
    try:
        vb.topology(2, own, nei, np.ones(2), np.ones(2))
        raise AssertionError("expected an error")
    except vb.VlmError as e:
        assert e.name == "BAD_ARG"


def test_context_without_device_fails_cleanly():
    if has_gpu():
        return
    try:
        vb.Context(0)
        raise AssertionError("expected NO_DEVICE")
    except vb.VlmError as e:
        assert e.name in ("NO_DEVICE", "CUDA")


def test_topology_matches_reference_on_skewed_meshes():
    """The library's agglomeration (coarse faces numbered by first occurrence without hashing)
    against the reference's own buildHierarchy on jittered graded meshes, 3D with a periodic
    direction and 2D."""
    import pytest
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("reference library not built here")
    from voluma_b200 import mesh as vm
    for n, per, two_d, seed in (((13, 11, 9), (0, 1, 0), False, 3), ((41, 29, 1), (0, 0, 0), True, 4)):
        pts = vm.jitter_interior(vm.box_points(n, beta=(0.7, 0.0, 0.9 if not two_d else 0.0)), n, 0.2, seed)
        M = vm.box_mesh(n, periodic=per, points=pts, two_d=two_d)
        R = ref.RefMesh(n, periodic=per, points=pts, two_d=two_d)
        t = vb.topology(M["n_cells"], M["owner"], M["neighbour"], M["magSf"], M["ndc"])
        h = R.gamg_levels()
        assert len(t) == len(h)
        for a, b in zip(t, h):
            for f in ("l", "u", "weight", "agg", "faceMap", "faceFlip"):
                assert np.array_equal(a[f], b[f].astype(a[f].dtype)), f
