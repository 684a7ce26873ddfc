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
