"""DIC/DILU preconditioning and the relaxation solvers on the device against the oracle and the
reference's own results (tests/golden: PBiCGStab/DILU, PCG/DIC, GaussSeidel, symGaussSeidel and
Jacobi runs of the reference's solveLdu).

The level-scheduled kernels apply every row's terms in the reference's order, so
  * one preconditioner application is compared bit for bit with the oracle
    (the oracle itself reproduces the reference's solves bit for bit, tests/test_oracle.py);
  * relaxation solves (whose iterates involve no reduction) give the reference's iterate bit for
    bit at the same iteration count, and its residuals within 1e-12 relative (the device's
    compensated sums round differently from the reference's plain double sums);
  * Krylov solves with DIC/DILU agree with the reference within +-1 iteration, meet the tolerance
    in the true residual, and match its solution within 1e-10 (PCG/DIC) or 1e-6 (PBiCGStab/DILU,
    whose iterates amplify the reductions' rounding to the solver tolerance).
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden, perf_dict
import voluma_b200 as vb
from oracle import restate as ro

pytestmark = pytest.mark.gpu

_meshes = {}


def device_mesh(name):
    if name not in _meshes:
        g = load_golden(name)
        _meshes[name] = (g, vb.Mesh.from_arrays(g))
    return _meshes[name]


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("prec,asym", [("DILU", True), ("DIC", False), ("DILU", False), ("diagonal", True),
                                       ("none", False)])
def test_precond_apply_bitwise(name, prec, asym):
    g, m = device_mesh(name)
    lower = g["lower_asym"] if asym else None
    w = vb.precond_apply(m, g["diag"], g["upper"], lower, g["b"], prec)
    assert np.array_equal(w, ro.precond_apply(g, g["diag"], g["upper"], lower, g["b"], prec))


@pytest.mark.parametrize("name", golden_names())
def test_dilu_apply_twice_is_deterministic(name):
    g, m = device_mesh(name)
    w1 = vb.precond_apply(m, g["diag"], g["upper"], g["lower_asym"], g["b"], "DILU")
    w2 = vb.precond_apply(m, g["diag"], g["upper"], g["lower_asym"], g["b"], "DILU")
    assert np.array_equal(w1, w2)


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("key,solver,prec,asym", [("bicg_dilu", "PBiCGStab", "DILU", True),
                                                  ("pcg_dic", "PCG", "DIC", False)])
def test_krylov_dilu_matches_reference(name, key, solver, prec, asym):
    g, m = device_mesh(name)
    x = g["x0"].copy()
    lower = g["lower_asym"] if asym else None
    p = vb.solve_ldu(m, g["diag"], g["upper"], lower, g["b"], x,
                     vb.SolverControls(solver, prec, 0.0, 1e-8, 2000))
    ref = perf_dict(g[key + "_perf"])
    assert abs(p.iterations - ref["iterations"]) <= 1
    assert p.converged == ref["converged"]
    # the true residual of the device solution meets the tolerance (normalised as in solveLdu)
    lo = g["upper"] if lower is None else lower
    true_res = np.abs(g["b"] - ro.amul(g, g["diag"], g["upper"], lo, x)).sum() / p.normFactor
    assert true_res <= 1.01e-8 * p.initialResidual
    # PCG/DIC stays close to the reference's iterate; PBiCGStab amplifies the rounding difference
    # of the reductions (compensated on the device, plain in the reference) to the solver tolerance
    assert rel(x, g[key + "_x"]) <= (1e-10 if solver == "PCG" else 1e-6)


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("key,solver,asym,rtol,max_iter,sweeps", [
    ("gs", "GaussSeidel", False, 1e-3, 300, 2),
    ("sgs", "symGaussSeidel", True, 1e-3, 300, 1),
    ("jac", "Jacobi", False, 1e-3, 300, 3),
])
def test_relaxation_solvers_match_reference(name, key, solver, asym, rtol, max_iter, sweeps):
    g, m = device_mesh(name)
    x = g["x0"].copy()
    lower = g["lower_asym"] if asym else None
    p = vb.solve_ldu(m, g["diag"], g["upper"], lower, g["b"], x,
                     vb.SolverControls(solver, "none", 0.0, rtol, max_iter, nSweeps=sweeps))
    ref = perf_dict(g[key + "_perf"])
    assert p.iterations == ref["iterations"]
    assert np.array_equal(x, g[key + "_x"])
    assert abs(p.finalResidual - ref["finalResidual"]) <= 1e-12 * ref["finalResidual"]
    assert p.converged == ref["converged"]


def test_relaxation_reproducible_mode_is_jacobi_bitwise():
    """CFD_REPRODUCIBLE: GaussSeidel -> Jacobi with exact sums (LinearSolver.cpp:141): the oracle's
    run, residuals included, bit for bit."""
    g, m = device_mesh("periodic8")
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x,
                     vb.SolverControls("GaussSeidel", "none", 0.0, 1e-3, 200, nSweeps=2, reproducible=True))
    xo, po = ro.solve(g, g["diag"], g["upper"], None, g["b"], g["x0"], "GaussSeidel", "none", 0.0, 1e-3, 200,
                      exact=True, n_sweeps=2)
    assert np.array_equal(x, xo)
    assert p.iterations == po["iterations"] and p.finalResidual == po["finalResidual"]
    assert p.normFactor == po["normFactor"]


def test_relaxation_needs_a_sweep():
    g, m = device_mesh("periodic8")
    x = g["x0"].copy()
    with pytest.raises(vb.VlmError) as e:
        vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x,
                     vb.SolverControls("GaussSeidel", "none", 0.0, 1e-3, 10, nSweeps=0))
    assert e.value.name == "BAD_ARG"


def test_dilu_batch_matches_solo():
    """A batch of uneven systems: each system's DILU-preconditioned solve equals its solo solve."""
    names = ("walls7x5x3", "cavity16", "jitter10x8x6")
    gs = [load_golden(n) for n in names]
    batch = vb.Mesh.batch(gs)
    diag = np.concatenate([g["diag"] for g in gs])
    upper = np.concatenate([g["upper"] for g in gs])
    lower = np.concatenate([g["lower_asym"] for g in gs])
    b = np.concatenate([g["b"] for g in gs])
    x = np.concatenate([g["x0"] for g in gs])
    perfs = vb.solve_ldu(batch, diag, upper, lower, b, x, vb.SolverControls("PBiCGStab", "DILU", 0.0, 1e-8, 2000))
    off = 0
    for name, g, p in zip(names, gs, perfs):
        _, ms = device_mesh(name)
        xs = g["x0"].copy()
        ps = vb.solve_ldu(ms, g["diag"], g["upper"], g["lower_asym"], g["b"], xs,
                          vb.SolverControls("PBiCGStab", "DILU", 0.0, 1e-8, 2000))
        assert np.array_equal(x[off:off + g["n_cells"]], xs)
        assert p.iterations == ps.iterations
        off += g["n_cells"]


def test_wide_system_uses_a_cooperative_group():
    """48^3 box: levels up to ~1700 rows wide, so one system is swept by a co-resident group of CTAs
    with the bounded global barrier; the result is still the natural-order one, bit for bit."""
    from voluma_b200 import mesh as vm
    msh = vm.box_mesh((48, 48, 48), hi=(1.0, 1.0, 1.0), periodic=(0, 0, 0))
    diag, upper = vm.poisson_matrix(msh)
    rng = np.random.default_rng(5)
    nI = msh["n_internal_faces"]
    lower = upper * (0.8 + 0.4 * rng.random(nI))
    r = rng.standard_normal(msh["n_cells"])
    m = vb.Mesh.from_arrays(msh)
    w = vb.precond_apply(m, diag, upper, lower, r, "DILU")
    assert np.array_equal(w, ro.precond_apply(msh, diag, upper, lower, r, "DILU"))
    x = np.zeros(msh["n_cells"])
    p = vb.solve_ldu(m, diag, upper, None, r, x, vb.SolverControls("symGaussSeidel", "none", 0.0, 1e-12, 4,
                                                                     nSweeps=2))
    xo, po = ro.solve(msh, diag, upper, None, r, np.zeros(msh["n_cells"]), "symGaussSeidel", "none", 0.0, 1e-12, 4,
                      n_sweeps=2)
    assert p.iterations == po["iterations"] == 4
    assert np.array_equal(x, xo)


def test_group_barrier_gives_up_when_a_cta_never_arrives():
    """Failure path of the bounded group barrier (dilu.cuh group_sync): with every CTA present the
    barriers all pass; with one CTA returning before its first arrival, the others' wait runs out
    after the spin limit, the kernel ends with status TIMEOUT, and the context stays usable."""
    st, passed = vb.barrier_check(6, 1 << 22, absent_cta=-1, rounds=5)
    assert st == "OK" and np.all(passed == 5)
    st, passed = vb.barrier_check(6, 2000, absent_cta=3, rounds=5)
    assert st == "TIMEOUT"
    assert np.all(passed == 0)  # nobody got through the first barrier
    st, passed = vb.barrier_check(4, 1 << 22, absent_cta=-1, rounds=3)
    assert st == "OK" and np.all(passed == 3)
