"""The oracle pinned against the reference: the C restatement (oracle/vlm_oracle.c) must reproduce
the reference's own outputs stored in tests/golden/ bit for bit, and, where the reference library
was built here (oracle/_ref), agree with it live on fresh inputs."""
import os

import numpy as np
import pytest

from conftest import golden_hierarchy, perf_dict
from oracle import restate as ro

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_exact_sum_properties():
    # test_mesh.cpp:13-28: order independence and exact cancellation
    assert ro.exact_sum([1e20, 1.0, -1e20]) == 1.0
    rng = np.random.default_rng(1)
    v = rng.standard_normal(10000) * np.exp(rng.uniform(-30, 30, 10000))
    assert ro.exact_sum(v) == ro.exact_sum(v[::-1]) == ro.exact_sum(rng.permutation(v))
    assert ro.exact_sum([]) == 0.0
    assert np.isnan(ro.exact_sum([1.0, np.nan]))
    assert ro.exact_sum([np.inf, 1.0]) == np.inf


def test_exact_sum_golden(golden):
    assert ro.exact_sum(golden["b"]) == golden["exact_sum_b"]
    assert ro.exact_sum(golden["exact_spread"]) == golden["exact_spread_sum"]


def test_amul_golden(golden):
    y = ro.amul(golden, golden["diag"], golden["upper"], None, golden["amul_x"])
    assert np.array_equal(y, golden["amul_y"])


def test_hierarchy_golden(golden):
    ref_h = golden_hierarchy(golden)
    h = ro.hierarchy(golden)
    assert len(h) == len(ref_h)
    for a, b in zip(h, ref_h):
        for f in ("l", "u", "weight", "agg", "faceMap", "faceFlip"):
            assert np.array_equal(a[f], b[f]), f


def test_vcycle_gs_golden(golden):
    w = ro.gamg_apply(golden, golden["diag"], golden["upper"], None, golden["b"], smoother="gs", coarse=0)
    assert np.array_equal(w, golden["vcycle_w"])


@pytest.mark.parametrize("key,solver,prec,exact,asym", [
    ("pcg_diag_repro", "PCG", "diagonal", True, False),
    ("pcg_diag", "PCG", "diagonal", False, False),
    ("pcg_gamg", "PCG", "GAMG", False, False),
    ("bicg_diag_repro", "PBiCGStab", "diagonal", True, True),
    ("bicg_gamg", "PBiCGStab", "GAMG", False, True),
])
def test_solve_golden(golden, key, solver, prec, exact, asym):
    lower = golden["lower_asym"] if asym else None
    x, perf = ro.solve(golden, golden["diag"], golden["upper"], lower, golden["b"], golden["x0"], solver, prec,
                       0.0, 1e-8, 2000, exact=exact)
    ref_perf = perf_dict(golden[key + "_perf"])
    assert np.array_equal(x, golden[key + "_x"])
    assert perf == ref_perf


@pytest.mark.parametrize("key,solver,prec,asym,rtol,max_iter,sweeps", [
    ("bicg_dilu", "PBiCGStab", "DILU", True, 1e-8, 2000, 1),
    ("pcg_dic", "PCG", "DIC", False, 1e-8, 2000, 1),
    ("gs", "GaussSeidel", "none", False, 1e-3, 300, 2),
    ("sgs", "symGaussSeidel", "none", True, 1e-3, 300, 1),
    ("jac", "Jacobi", "none", False, 1e-3, 300, 3),
])
def test_dilu_and_relaxation_golden(golden, key, solver, prec, asym, rtol, max_iter, sweeps):
    """DIC/DILU (LinearSolver.cpp:56-107) and GaussSeidel/symGaussSeidel/Jacobi (:238-278) restated:
    the reference's solutions, residuals and iteration counts bit for bit."""
    lower = golden["lower_asym"] if asym else None
    x, perf = ro.solve(golden, golden["diag"], golden["upper"], lower, golden["b"], golden["x0"], solver, prec,
                       0.0, rtol, max_iter, n_sweeps=sweeps)
    assert np.array_equal(x, golden[key + "_x"])
    assert perf == perf_dict(golden[key + "_perf"])


def test_precond_apply_properties(golden):
    """DILU on a symmetric matrix is DIC; M^-1 applied to M-products: w = M^-1 r is linear."""
    g = golden
    r = g["b"]
    w1 = ro.precond_apply(g, g["diag"], g["upper"], None, r, "DIC")
    assert np.array_equal(w1, ro.precond_apply(g, g["diag"], g["upper"], g["upper"], r, "DILU"))
    w2 = ro.precond_apply(g, g["diag"], g["upper"], None, 2.0 * r, "DIC")
    assert np.allclose(w2, 2.0 * w1, rtol=1e-13, atol=0)
    wd = ro.precond_apply(g, g["diag"], g["upper"], None, r, "diagonal")
    assert np.array_equal(wd, 1.0 / g["diag"] * r)


def test_oracle_live_against_reference():
    """Fresh random inputs through both the reference build and the restatement."""
    ref = pytest.importorskip("oracle.ref")
    if not ref.available():
        pytest.skip("reference library not built here")
    from voluma_b200 import mesh as vm
    n = (9, 7, 6)
    pts = vm.jitter_interior(vm.box_points(n, beta=(0.8, 0, 1.1)), n, 0.15, 11)
    R = ref.RefMesh(n, periodic=(0, 1, 0), points=pts)
    M = vm.box_mesh(n, periodic=(0, 1, 0), points=pts)
    d, up = vm.poisson_matrix(M)
    rng = np.random.default_rng(5)
    b = rng.standard_normal(M["n_cells"])
    for prec in ("diagonal", "GAMG"):
        xr, pr = R.solve(d, up, None, b, np.zeros(M["n_cells"]), "PCG", prec, 0.0, 1e-9, 500)
        xo, po = ro.solve(M, d, up, None, b, np.zeros(M["n_cells"]), "PCG", prec, 0.0, 1e-9, 500)
        assert np.array_equal(xr, xo) and pr == po


@pytest.mark.parametrize("name", ["periodic8", "walls7x5x3", "cavity16", "jitter10x8x6", "periodic24"])
def test_matching_hierarchy_is_a_maximal_pairing(name):
    """The parallel matching's restatement (the device agglomeration's definition): on every level
    of every pass each aggregate is a pair of neighbours or a pair with cells that had no unpaired
    neighbour left, every cell has one aggregate, coarse faces are the distinct aggregate pairs in
    (lower, upper) order, and the coarse weights are the fine weights' sums."""
    z = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    z["n_cells"] = int(z["sizes"][0])
    H = ro.hierarchy(z, matching=True, merge=1)
    for k in range(len(H) - 1):
        L, C = H[k], H[k + 1]
        agg = L["agg"]
        assert agg.min() == 0 and agg.max() == C["n"] - 1
        sizes = np.bincount(agg, minlength=C["n"])
        assert sizes.min() >= 1
        # coarse faces: sorted distinct pairs
        keys = C["l"].astype(np.int64) * (1 << 32) + C["u"]
        assert np.all(np.diff(keys) > 0) and np.all(C["l"] < C["u"])
        a, b = agg[L["l"]], agg[L["u"]]
        inter = a != b
        pairs = set(zip(np.minimum(a, b)[inter].tolist(), np.maximum(a, b)[inter].tolist()))
        assert pairs == set(zip(C["l"].tolist(), C["u"].tolist()))
        w = np.zeros(len(C["l"]))
        np.add.at(w, L["faceMap"][inter], L["weight"][inter])
        assert np.allclose(w, C["weight"], rtol=1e-14, atol=0)
        # the cells paired in the matching: a pair shares a face
        for c in np.nonzero(sizes == 2)[0][:200]:
            i, j = np.nonzero(agg == c)[0]
            assert np.any((L["l"] == i) & (L["u"] == j))
