"""Device-side GAMG agglomeration (vlm_mesh_register_ex with VLM_MESH_DEVICE_AGGLOMERATION,
csrc/aggl.cu) against its CPU restatement (oracle/vlm_oracle.c, vo_hier_build_matching): the
parallel handshake matching gives the same hierarchy (cells, faces, aggregates) on every golden mesh
and on device-built boxes, and GAMG-PCG on it converges as the restatement's solve of the same
schedule does (iterations +-1, relative L2 <= 1e-10 at equal work)."""
import os

import numpy as np
import pytest

import voluma_b200 as vb
from oracle import restate as ro
from voluma_b200 import mesh as vm

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")
NAMES = ["periodic8", "walls7x5x3", "cavity16", "stretched6x9x5", "jitter10x8x6", "periodic24"]


def golden(name):
    g = dict(np.load(os.path.join(HERE, f"{name}.npz")))
    g["n_cells"] = int(g["sizes"][0])
    g["patch_start"], g["patch_size"] = g["patchStart"], g["patchSize"]
    g["two_d"], g["empty_dir"] = int(g["sizes"][4]), int(g["sizes"][5])
    return g


def ctrl(**kw):
    base = dict(solver="PCG", preconditioner="GAMG", tolerance=0.0, relTol=1e-8, maxIter=2000, smoother="mcgs-jacobi")
    base.update(kw)
    return vb.SolverControls(**base)


def same_hierarchy(m, oracle_levels):
    dev = m.gamg_levels()
    assert [L["n"] for L in dev] == [L["n"] for L in oracle_levels]
    for k, (a, b) in enumerate(zip(dev, oracle_levels)):
        assert np.array_equal(a["l"], b["l"]) and np.array_equal(a["u"], b["u"]), k
        if k + 1 < len(dev):
            assert np.array_equal(a["agg"], b["agg"]), k


@pytest.mark.parametrize("name", NAMES)
def test_device_hierarchy_equals_restatement(name):
    g = golden(name)
    m = vb.Mesh.from_arrays(g, agglomeration="device")
    same_hierarchy(m, ro.hierarchy(g, matching=True))
    m.close()


@pytest.mark.parametrize("n", [(40, 24, 1), (20, 18, 16)])
def test_device_hierarchy_on_boxes(n):
    # a uniform box: every coupling equal, so the pairing rests on the pair hash alone
    b = vm.box_mesh(n, two_d=n[2] == 1, periodic=(1, 0, 0))
    m = vb.Mesh.from_arrays(b, agglomeration="device")
    same_hierarchy(m, ro.hierarchy(b, matching=True))
    m.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_agglomeration_solve_matches_restatement(name, precision):
    g = golden(name)
    m = vb.Mesh.from_arrays(g, agglomeration="device")
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(precision=precision))
    m.close()
    xo, po = ro.solve(g, g["diag"], g["upper"], None, g["b"], g["x0"], "PCG", "GAMG", 0.0, 1e-8, 2000,
                      smoother="mcgs-jacobi", coarse=1, matching=True)
    assert p.converged and po["converged"]
    assert abs(p.iterations - po["iterations"]) <= 1
    if p.iterations != po["iterations"]:
        xo, pk = ro.solve(g, g["diag"], g["upper"], None, g["b"], g["x0"], "PCG", "GAMG", 0.0, 0.0, p.iterations,
                          smoother="mcgs-jacobi", coarse=1, matching=True)
    tol = 1e-10 if precision == "fp64" else 1e-6
    assert np.linalg.norm(x - xo) <= tol * np.linalg.norm(xo)


def test_unknown_registration_flag():
    g = golden("periodic8")
    with pytest.raises(ValueError):
        vb.Mesh.from_arrays(g, agglomeration="elsewhere")


def test_device_hierarchy_disconnected_and_isolated_cells():
    """Two disconnected boxes and a cell without faces: the matching never pairs across components,
    the isolated cell is an aggregate of its own on every level, and the hierarchy equals the
    restatement's."""
    a = vm.box_mesh((9, 7, 1), two_d=True)
    b = vm.box_mesh((6, 5, 4))
    na, nb = a["n_cells"], b["n_cells"]
    nIa, nIb = len(a["neighbour"]), len(b["neighbour"])
    own = np.concatenate([a["owner"][:nIa], b["owner"][:nIb] + na]).astype(np.int32)
    nei = np.concatenate([a["neighbour"], b["neighbour"] + na]).astype(np.int32)
    magSf = np.concatenate([a["magSf"][:nIa], b["magSf"][:nIb]])
    ndc = np.concatenate([a["ndc"][:nIa], b["ndc"][:nIb]])
    m = dict(n_cells=na + nb + 1, owner=own, neighbour=nei, magSf=magSf, ndc=ndc)
    mesh = vb.Mesh(m["n_cells"], own, nei, magSf, ndc, agglomeration="device")
    H = ro.hierarchy(m, matching=True)
    same_hierarchy(mesh, H)
    for k in range(len(H) - 1):
        agg = H[k]["agg"]
        n = H[k]["n"]
        # the last cell of every level is the isolated one (numbered by its first cell, it comes last)
        assert np.count_nonzero(agg == agg[n - 1]) == 1
    # a Poisson-like system on it: every component solvable (diagonal dominance for the isolated cell)
    up = -magSf * ndc
    d = np.zeros(m["n_cells"])
    np.add.at(d, own, -up)
    np.add.at(d, nei, -up)
    d[0] *= 2.0
    d[na] *= 2.0
    d[-1] = 1.0
    rng = np.random.default_rng(3)
    bvec = rng.standard_normal(m["n_cells"])
    x = np.zeros(m["n_cells"])
    p = vb.solve_ldu(mesh, d, up, None, bvec, x, ctrl())
    xo, po = ro.solve(m, d, up, None, bvec, np.zeros(m["n_cells"]), "PCG", "GAMG", 0.0, 1e-8, 2000,
                      smoother="mcgs-jacobi", coarse=1, matching=True)
    assert p.converged and abs(p.iterations - po["iterations"]) <= 1
    mesh.close()
