"""Parity of the CUDA path (through the C ABI) with the oracle and the reference's own results.

Tolerances: integer/topology results and row-ordered arithmetic are compared bit for bit; whole
solves are compared at relative L2 <= 1e-10 with iteration counts equal (reference algorithm) or
within +-1; mixed precision is checked against its own stated bound (true FP64 residual below
relTol, solution within 1e-6 relative of the FP64 solve)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, perf_dict
import voluma_b200 as vb
from voluma_b200 import mesh as vm
from oracle import restate as ro

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


_meshes = {}


def device_mesh(name):
    if name not in _meshes:
        g = load_golden(name)
        g["patch_start"], g["patch_size"] = g["patchStart"], g["patchSize"]
        g["two_d"], g["empty_dir"] = int(g["sizes"][4]), int(g["sizes"][5])
        _meshes[name] = (g, vb.Mesh.from_arrays(g))
    return _meshes[name]


def ctrl(**kw):
    base = dict(solver="PCG", preconditioner="diagonal", tolerance=0.0, relTol=1e-8, maxIter=2000)
    base.update(kw)
    return vb.SolverControls(**base)


def oracle_iterate(m, d, up, b, x0, xo, po, iterations, smoother="mcgs-jacobi"):
    """The oracle's solution after exactly `iterations` PCG+GAMG iterations: its converged solution
    when the counts agree, else the same schedule run to that count (tolerances 0).  Near relTol
    1e-8 one iteration moves the solution by up to 2e-7 relative on these systems, so a +-1 count
    is compared at equal work."""
    if iterations == po["iterations"]:
        return xo
    xk, pk = ro.solve(m, d, up, None, b, x0, "PCG", "GAMG", 0.0, 0.0, iterations, smoother=smoother, coarse=1)
    assert pk["iterations"] == iterations
    return xk


def true_residual(m, d, up, lo, b, x):
    return np.abs(b - ro.amul(m, d, up, lo, x)).sum()


@pytest.mark.parametrize("name", golden_names())
def test_amul_bitwise(name):
    g, m = device_mesh(name)
    y = vb.amul(m, g["diag"], g["upper"], None, g["amul_x"])
    assert np.array_equal(y, g["amul_y"])
    lo = g["lower_asym"]
    assert np.array_equal(vb.amul(m, g["diag"], g["upper"], lo, g["amul_x"]),
                          ro.amul(g, g["diag"], g["upper"], lo, g["amul_x"]))


@pytest.mark.parametrize("name", golden_names())
def test_device_hierarchy_equals_reference(name):
    g, m = device_mesh(name)
    lv = m.gamg_levels()
    assert len(lv) == int(g["nlevels"])
    for k, L in enumerate(lv):
        assert np.array_equal(L["agg"], g[f"lev{k}_agg"])
        assert np.array_equal(L["l"], g[f"lev{k}_l"])


def test_exact_sum_bitwise():
    g = load_golden("periodic24")
    assert vb.exact_sum(g["b"]) == g["exact_sum_b"]
    assert vb.exact_sum(g["exact_spread"]) == g["exact_spread_sum"]
    assert vb.exact_sum([1e20, 1.0, -1e20]) == 1.0
    rng = np.random.default_rng(2)
    v = rng.standard_normal(300000) * np.exp(rng.uniform(-300, 300, 300000))
    assert vb.exact_sum(v) == ro.exact_sum(v) == vb.exact_sum(v[::-1])
    assert np.isnan(vb.exact_sum([1.0, np.nan])) and vb.exact_sum([np.inf, 2.0]) == np.inf


@pytest.mark.parametrize("name", golden_names())
def test_pcg_diagonal_reproducible_bitwise(name):
    """CFD_REPRODUCIBLE mode: exact sums + the reference's operation order -> the reference's
    solution bit for bit, same iteration count and residuals."""
    g, m = device_mesh(name)
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(reproducible=True))
    ref = perf_dict(g["pcg_diag_repro_perf"])
    assert p.iterations == ref["iterations"]
    assert p.converged == ref["converged"]
    assert np.array_equal(x, g["pcg_diag_repro_x"])
    assert p.initialResidual == ref["initialResidual"] and p.finalResidual == ref["finalResidual"]
    assert p.normFactor == ref["normFactor"] and p.residualSum == ref["residualSum"]


@pytest.mark.parametrize("name", golden_names())
def test_pcg_diagonal_matches_reference(name):
    g, m = device_mesh(name)
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl())
    ref = perf_dict(g["pcg_diag_perf"])
    assert abs(p.iterations - ref["iterations"]) <= 1
    assert rel(x, g["pcg_diag_x"]) <= 1e-10


@pytest.mark.parametrize("name", golden_names())
def test_vcycle_mcgs_matches_oracle(name):
    g, m = device_mesh(name)
    w = vb.gamg_apply(m, g["diag"], g["upper"], None, g["b"], smoother="mcgs")
    wo = ro.gamg_apply(g, g["diag"], g["upper"], None, g["b"], smoother="mcgs", coarse=1)
    assert rel(w, wo) <= 1e-14


@pytest.mark.parametrize("name", golden_names())
def test_vcycle_jacobi_matches_oracle(name):
    g, m = device_mesh(name)
    w = vb.gamg_apply(m, g["diag"], g["upper"], None, g["b"], smoother="jacobi")
    wo = ro.gamg_apply(g, g["diag"], g["upper"], None, g["b"], smoother="jacobi", coarse=1)
    assert rel(w, wo) <= 1e-14


@pytest.mark.parametrize("name", golden_names())
def test_vcycle_mcgs_jacobi_matches_oracle(name):
    g, m = device_mesh(name)
    w = vb.gamg_apply(m, g["diag"], g["upper"], None, g["b"], smoother="mcgs-jacobi")
    wo = ro.gamg_apply(g, g["diag"], g["upper"], None, g["b"], smoother="mcgs-jacobi", coarse=1)
    assert rel(w, wo) <= 1e-14


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("smoother", ["mcgs", "mcgs-jacobi", "jacobi"])
def test_pcg_gamg_matches_oracle(name, smoother):
    g, m = device_mesh(name)
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(preconditioner="GAMG", smoother=smoother))
    xo, po = ro.solve(g, g["diag"], g["upper"], None, g["b"], g["x0"], "PCG", "GAMG", 0.0, 1e-8, 2000,
                      smoother=smoother, coarse=1)
    assert abs(p.iterations - po["iterations"]) <= 1
    assert p.converged and po["converged"]
    assert rel(x, oracle_iterate(g, g["diag"], g["upper"], g["b"], g["x0"], xo, po, p.iterations, smoother)) <= 1e-10
    # against the reference's sequential-GS GAMG: same tolerance reached, counts reported
    ref = perf_dict(g["pcg_gamg_perf"])
    assert true_residual(g, g["diag"], g["upper"], None, g["b"], x) <= 1e-8 * ref["residualSum"] * 1.0001
    if smoother != "jacobi":
        assert abs(p.iterations - ref["iterations"]) <= 3


@pytest.mark.parametrize("name", golden_names())
def test_pbicgstab_diagonal_reproducible_bitwise(name):
    g, m = device_mesh(name)
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], g["lower_asym"], g["b"], x,
                     ctrl(solver="PBiCGStab", reproducible=True))
    ref = perf_dict(g["bicg_diag_repro_perf"])
    assert p.iterations == ref["iterations"]
    assert p.converged == ref["converged"]
    assert np.array_equal(x, g["bicg_diag_repro_x"])


@pytest.mark.parametrize("name", golden_names())
def test_pbicgstab_gamg(name):
    g, m = device_mesh(name)
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], g["lower_asym"], g["b"], x,
                     ctrl(solver="PBiCGStab", preconditioner="GAMG"))
    xo, po = ro.solve(g, g["diag"], g["upper"], g["lower_asym"], g["b"], g["x0"], "PBiCGStab", "GAMG", 0.0, 1e-8,
                      2000, smoother="mcgs-jacobi", coarse=1)
    assert p.converged
    assert abs(p.iterations - po["iterations"]) <= 1


@pytest.mark.parametrize("name", golden_names())
def test_mixed_precision_reaches_fp64_tolerance(name):
    """FP32 V-cycle inside the FP64 PCG recurrence: same tolerance, same iteration count (+-1),
    solution within 1e-6 relative of the FP64 solve (the stated error bound)."""
    g, m = device_mesh(name)
    x64 = g["x0"].copy()
    p64 = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x64, ctrl(preconditioner="GAMG"))
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(preconditioner="GAMG", precision="mixed"))
    assert p.converged
    assert abs(p.iterations - p64.iterations) <= 1
    assert p.finalResidual < 1e-8 * p.initialResidual
    r = true_residual(g, g["diag"], g["upper"], None, g["b"], x)
    assert r / p.normFactor < 1e-8 * p.initialResidual * 1.0001
    assert rel(x, x64) <= 1e-6


@pytest.mark.parametrize("name", ["periodic8", "walls7x5x3", "jitter10x8x6"])
def test_mixed_defect_correction_converges(name):
    """FP32 inner PCG+GAMG inside FP64 defect correction reaches the FP64 tolerance."""
    g, m = device_mesh(name)
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(preconditioner="GAMG", precision="mixed-dc"))
    assert p.converged and p.outerIterations >= 1
    r = true_residual(g, g["diag"], g["upper"], None, g["b"], x)
    assert r / p.normFactor < 1e-8 * p.initialResidual * 1.0001


def test_deterministic_bitwise():
    g, m = device_mesh("periodic24")
    xs = []
    for _ in range(3):
        x = g["x0"].copy()
        vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(preconditioner="GAMG"))
        xs.append(x)
    assert np.array_equal(xs[0], xs[1]) and np.array_equal(xs[1], xs[2])


def test_single_level_system_is_a_direct_solve():
    M = vm.box_mesh((4, 4, 2))
    d, up = vm.poisson_matrix(M)
    m = vb.Mesh.from_arrays(M)
    assert len(m.gamg_levels()) == 1
    b = np.random.default_rng(3).standard_normal(M["n_cells"])
    x = np.zeros(M["n_cells"])
    p = vb.solve_ldu(m, d, up, None, b, x, ctrl(preconditioner="GAMG"))
    assert p.converged and p.iterations <= 2


def test_already_converged_does_no_iteration():
    g, m = device_mesh("periodic8")
    x = g["x0"].copy()
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(tolerance=10.0))
    assert p.iterations == 0 and p.converged
    assert np.array_equal(x, g["x0"])


def test_errors_follow_the_reference():
    g, m = device_mesh("periodic8")
    x = g["x0"].copy()
    with pytest.raises(vb.VlmError) as e:
        vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(solver="BiCG"))
    assert e.value.name == "UNSUPPORTED"
    with pytest.raises(vb.VlmError) as e:
        vb.solve_ldu(m, g["diag"], g["upper"], g["lower_asym"], g["b"], x, ctrl())
    assert e.value.name == "UNSUPPORTED" and "symmetric" in str(e.value)
    with pytest.raises(vb.VlmError) as e:
        vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(preconditioner="ILU"))
    assert e.value.name == "UNSUPPORTED"


def test_nonfinite_rhs_is_reported_not_hung():
    g, m = device_mesh("periodic8")
    b = g["b"].copy()
    b[5] = np.nan
    x = np.zeros(g["n_cells"])
    p = vb.solve_ldu(m, g["diag"], g["upper"], None, b, x, ctrl(preconditioner="GAMG"))
    assert p.status == 5 and not p.converged


def test_singular_coarsest_matrix_raises():
    g, m = device_mesh("periodic8")
    x = np.zeros(g["n_cells"])
    with pytest.raises(vb.VlmError) as e:
        vb.solve_ldu(m, np.zeros(g["n_cells"]), np.zeros(g["n_internal_faces"]), None, g["b"], x,
                     ctrl(preconditioner="GAMG", maxIter=3))
    assert e.value.name == "SINGULAR"


def test_64cubed_gamg_against_oracle():
    M = vm.box_mesh((64, 64, 64), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    d, up = vm.poisson_matrix(M)
    b = np.random.default_rng(9).standard_normal(M["n_cells"])
    b -= b.mean()
    m = vb.Mesh.from_arrays(M)
    x = np.zeros(M["n_cells"])
    p = vb.solve_ldu(m, d, up, None, b, x, ctrl(preconditioner="GAMG"))
    xo, po = ro.solve(M, d, up, None, b, np.zeros(M["n_cells"]), "PCG", "GAMG", 0.0, 1e-8, 2000,
                      smoother="mcgs-jacobi", coarse=1)
    assert abs(p.iterations - po["iterations"]) <= 1
    assert rel(x, oracle_iterate(M, d, up, b, np.zeros(M["n_cells"]), xo, po, p.iterations)) <= 1e-10


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_box_level0_matches_general_layout(name, precision, monkeypatch):
    """Every golden mesh is a box; level 0 runs the structured box kernels unless a periodic extent
    is odd (stretched6x9x5: three colours, the general layout).  The same solve on the general SELL
    layout (VLM_BOX=0 at registration) gives the same iterates - bit for bit where the two layouts
    place the rows alike (even x extent), else to rounding (odd x extent: the box layout has padding
    slots, so the reductions' partial sums are grouped differently)."""
    g, m = device_mesh(name)
    shape = vb.box_shape(g["n_cells"], g["owner"][:g["n_internal_faces"]], g["neighbour"][:g["n_internal_faces"]])
    assert shape is not None
    assert shape["layout"] == all(not p or n % 2 == 0 for n, p in zip(shape["n"], shape["periodic"]))
    monkeypatch.setenv("VLM_BOX", "0")
    m2 = vb.Mesh.from_arrays(g)
    monkeypatch.delenv("VLM_BOX")
    c = ctrl(preconditioner="GAMG", precision=precision)
    x1, x2 = g["x0"].copy(), g["x0"].copy()
    p1 = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x1, c)
    p2 = vb.solve_ldu(m2, g["diag"], g["upper"], None, g["b"], x2, c)
    assert p1.iterations == p2.iterations
    if shape["n"][0] % 2 == 0 or not shape["layout"]:
        assert np.array_equal(x1, x2) and p1.finalResidual == p2.finalResidual
    else:
        assert rel(x1, x2) <= 1e-12


@pytest.mark.parametrize("name", ["periodic24", "cavity16", "jitter10x8x6"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tail_launch_configurations_give_identical_results(name, precision):
    """The coarse V-cycle tail (one CTA or a thread-block cluster of 2, 4 or 8 CTAs per system, taking
    the levels below a row limit, or the whole V-cycle of a small system) only shapes launches: every
    configuration gives the solution of the per-level launches bit for bit."""
    g, _ = device_mesh(name)
    m = vb.Mesh.from_arrays(g)
    c = ctrl(preconditioner="GAMG", precision=precision)
    ref = None
    for cfg in [(1, 32, 1), (1, 256, 1), (1, 1, 4096), (2, 256, 1), (4, 1, 4096), (8, 4096, 1), (8, 1, 8192)]:
        m.set_tail(*cfg)
        x = g["x0"].copy()
        p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, c)
        if ref is None:
            ref = (x, p.iterations)
            assert p.converged
        assert p.iterations == ref[1] and np.array_equal(x, ref[0]), cfg


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["periodic24", "stretched6x9x5"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_coarse_launches_give_identical_results(name, precision):
    """The fused Jacobi-level launches (both pre-sweeps in one pass, residual with restriction,
    prolongation inside the first post-sweep) perform the unfused launches' row operations in the
    same order: every combination gives the unfused solution bit for bit, with and without the
    coarse tail."""
    g, _ = device_mesh(name)
    m = vb.Mesh.from_arrays(g)
    c = ctrl(preconditioner="GAMG", precision=precision)
    ref = None
    big = 1 << 40
    for tail in [(1, 32, 1), (1, 1, 1 << 30)]:
        m.set_tail(*tail)
        for fuse in [(0, 0, 0), (big, 0, 0), (0, big, 0), (0, 0, big), (big, big, big), (64, 64, 64)]:
            m.set_fusion(*fuse)
            assert m.fusion_config() == fuse
            x = g["x0"].copy()
            p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, c)
            if ref is None:
                ref = (x, p.iterations)
                assert p.converged
            assert p.iterations == ref[1] and np.array_equal(x, ref[0]), (tail, fuse)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["periodic24", "walls7x5x3"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_box_sweep_matches_colour_launches(name, precision, monkeypatch):
    """A box level-0 red-black sweep as one launch (first-colour pieces, then second-colour pieces
    that wait for the planes they read, across the periodic wrap) performs the two colour launches'
    row operations: the same solution bit for bit."""
    g, _ = device_mesh(name)
    out = []
    for fused in ("0", "1"):
        monkeypatch.setenv("VLM_BOX_FUSED", fused)
        m = vb.Mesh.from_arrays(g)
        x = g["x0"].copy()
        p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, ctrl(preconditioner="GAMG", precision=precision))
        out.append((x, p.iterations))
        m.close()
    assert out[0][1] == out[1][1] and np.array_equal(out[0][0], out[1][0])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["periodic24", "jitter10x8x6", "stretched6x9x5"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_shared_memory_tail_matches_global_tail(name, precision, monkeypatch):
    """The coarse tail with every operand in shared memory performs the global-memory tail's row
    operations in the same order: bit for bit, for tails that start at several levels."""
    g, _ = device_mesh(name)
    c = ctrl(preconditioner="GAMG", precision=precision)
    for rows in (32, 256, 1024):
        out = []
        for smem in ("0", "1"):
            monkeypatch.setenv("VLM_TAIL_SMEM", smem)
            m = vb.Mesh.from_arrays(g)
            m.set_tail(1, rows, 1)
            x = g["x0"].copy()
            p = vb.solve_ldu(m, g["diag"], g["upper"], None, g["b"], x, c)
            out.append((x, p.iterations))
            m.close()
        assert out[0][1] == out[1][1] and np.array_equal(out[0][0], out[1][0]), rows


@pytest.mark.gpu
@pytest.mark.parametrize("shape,periodic", [((32, 16, 8), (1, 1, 1)), ((64, 16, 6), (0, 0, 0)),
                                            ((32, 32, 12), (1, 0, 1)), ((64, 24, 4), (1, 1, 1))])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_streamed_product_matches_four_slot_kernel(shape, periodic, precision, monkeypatch):
    """The plane-streamed level-0 FP64 product (y-pencils of x-rows, z-planes staged in shared
    memory by bulk copies, runs of planes split across CTAs, periodic and wall boundaries) forms
    every row's terms in the four-slot kernel's order, and its dot differs only in how the per-CTA
    double-double partials are grouped: the same PCG iterates bit for bit, with GAMG and with the
    diagonal preconditioner."""
    M = vm.box_mesh(shape, hi=(1.0, 0.7, 0.5), periodic=periodic)
    d, up = vm.poisson_matrix(M)
    b = np.random.default_rng(3).standard_normal(M["n_cells"])
    b -= b.mean()
    out = {}
    for on in ("0", "1"):
        monkeypatch.setenv("VLM_BOX_STREAM", on)
        m = vb.Mesh.from_arrays(M)
        assert (m.stream_config()[2] > 0) == (on == "1")
        for pc in ("GAMG", "diagonal"):
            x = np.zeros(M["n_cells"])
            p = vb.solve_ldu(m, d, up, None, b, x, ctrl(preconditioner=pc, precision=precision))
            assert p.converged
            out[on, pc] = (x, p.iterations)
        m.close()
    for pc in ("GAMG", "diagonal"):
        assert out["0", pc][1] == out["1", pc][1]
        assert np.array_equal(out["0", pc][0], out["1", pc][0])


@pytest.mark.gpu
@pytest.mark.parametrize("shape,periodic", [((32, 32, 32), (1, 1, 1)), ((24, 16, 20), (0, 0, 0))])
def test_mixed_defect_correction_projects_the_reference_mode(shape, periodic):
    """With setReference, A = L + c e_ref e_ref^T (one row with a non-zero row sum): the defect
    correction solves the pure-Neumann L in FP32 with the constant mode projected out of every
    preconditioned residual and restores that mode in FP64, so it reaches relTol 1e-8 in at most
    three outer passes and within a few iterations of the FP64 solve (ten passes before)."""
    M = vm.box_mesh(shape, hi=(1.0, 0.8, 0.9), periodic=periodic)
    d, up = vm.poisson_matrix(M)
    b = np.random.default_rng(11).standard_normal(M["n_cells"])
    b -= b.mean()
    m = vb.Mesh.from_arrays(M)
    x64 = np.zeros(M["n_cells"])
    p64 = vb.solve_ldu(m, d, up, None, b, x64, ctrl(preconditioner="GAMG"))
    x = np.zeros(M["n_cells"])
    p = vb.solve_ldu(m, d, up, None, b, x, ctrl(preconditioner="GAMG", precision="mixed-dc"))
    m.close()
    assert p.converged and 1 <= p.outerIterations <= 3
    assert p.iterations <= p64.iterations + 5
    r = np.abs(b - ro.amul(M, d, up, None, x)).sum()
    assert r / p.normFactor < 1e-8 * p.initialResidual * 1.0001
    assert rel(x, x64) <= 1e-6


@pytest.mark.gpu
def test_mixed_defect_correction_without_reference_row():
    """Several rows with non-zero row sums (Dirichlet-like boundary rows): no single reference row,
    so nothing is projected and the plain defect correction runs; it still reaches relTol 1e-8."""
    M = vm.box_mesh((16, 12, 10), hi=(1.0, 0.8, 0.9))
    d, up = vm.poisson_matrix(M, ref_cell=None)
    d = d.copy()
    d[::7] *= 1.5
    b = np.random.default_rng(12).standard_normal(M["n_cells"])
    m = vb.Mesh.from_arrays(M)
    x = np.zeros(M["n_cells"])
    p = vb.solve_ldu(m, d, up, None, b, x, ctrl(preconditioner="GAMG", precision="mixed-dc"))
    m.close()
    assert p.converged and p.outerIterations >= 1
    r = np.abs(b - ro.amul(M, d, up, None, x)).sum()
    assert r / p.normFactor < 1e-8 * p.initialResidual * 1.0001


@pytest.mark.gpu
@pytest.mark.parametrize("shape,periodic", [((20, 16, 8), (1, 1, 1)), ((32, 16, 2), (0, 0, 0)), ((32, 9, 6), (0, 0, 0))])
def test_streamed_product_not_planned_where_it_cannot_apply(shape, periodic):
    """x rows of 10 slots (not whole 16-byte words), fewer than 3 planes, or no pencil height that
    divides ny (9): no streamed shape is planned, the four-slot product runs, and the solve matches
    the oracle's."""
    M = vm.box_mesh(shape, hi=(1.0, 0.7, 0.5), periodic=periodic)
    d, up = vm.poisson_matrix(M)
    b = np.random.default_rng(4).standard_normal(M["n_cells"])
    b -= b.mean()
    m = vb.Mesh.from_arrays(M)
    assert m.stream_config() == (0, 0, 0)
    x = np.zeros(M["n_cells"])
    p = vb.solve_ldu(m, d, up, None, b, x, ctrl(preconditioner="GAMG"))
    m.close()
    xo, po = ro.solve(M, d, up, None, b, np.zeros(M["n_cells"]), "PCG", "GAMG", 0.0, 1e-8, 2000,
                      smoother="mcgs-jacobi", coarse=1)
    assert p.converged and abs(p.iterations - po["iterations"]) <= 1
    assert rel(x, oracle_iterate(M, d, up, b, np.zeros(M["n_cells"]), xo, po, p.iterations)) <= 1e-10
