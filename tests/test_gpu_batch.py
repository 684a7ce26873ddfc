"""Batched solves: uneven systems in one device batch.  Reductions, convergence tests and coarse
solves are per system with a fixed partition, so every system's result must be bit-identical to
solving it alone (batch invariance), whatever else shares the launch."""
import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases
from voluma_b200 import mesh as vm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems():
    # uneven sizes, including a one-level system (4^3 = 64 cells) and a 2-level one
    rng = np.random.default_rng(11)
    out = []
    for n in (9, 4, 13, 6, 11, 5):
        m = cases.graded_jittered_box(n, float(rng.uniform(1, 8)), 0.2, int(rng.integers(1 << 30)))
        u = cases.fourier_velocity(m["Cf"], int(rng.integers(1 << 30)))
        out.append((m, cases.div_per_volume(m, cases.face_flux(m, u))))
    return out


def run_batch(systems, ctrl, n_non_orth=2):
    meshes = [m for m, _ in systems]
    B = vb.Mesh.batch(meshes)
    gamma = cases.batch_face_array(meshes, [np.ones(m["n_faces"]) for m in meshes])
    div = np.concatenate([d for _, d in systems])
    p = np.zeros(B.n_cells)
    perf, flux = vb.pressure_solve(B, gamma, div, p, ctrl, ref_cell=[0] * len(meshes), n_non_orth=n_non_orth,
                                   grad_scheme=1)
    ps = [p[B.cell_base[i]:B.cell_base[i + 1]] for i in range(len(meshes))]
    return perf, ps, cases.split_batch_faces(meshes, flux)


def run_solo(m, div, ctrl, n_non_orth=2):
    M = vb.Mesh.from_arrays(m)
    p = np.zeros(m["n_cells"])
    perf, flux = vb.pressure_solve(M, np.ones(m["n_faces"]), div, p, ctrl, ref_cell=0, n_non_orth=n_non_orth,
                                   grad_scheme=1)
    return perf, p, flux


@pytest.mark.parametrize("precision", ["", "mixed"])
def test_batch_invariance_pressure_loop(systems, precision):
    ctrl = vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 500, precision=precision)
    perf, ps, fluxes = run_batch(systems, ctrl)
    for i, (m, div) in enumerate(systems):
        sp, p, flux = run_solo(m, div, ctrl)
        assert [q.iterations for q in sp] == [row[i].iterations for row in perf]
        assert np.array_equal(ps[i], p), i
        assert np.array_equal(fluxes[i], flux), i
        assert all(row[i].converged for row in perf)


def test_batch_reproducible_mode_matches_solo(systems):
    ctrl = vb.SolverControls("PCG", "diagonal", 0.0, 1e-8, 3000, reproducible=True)
    perf, ps, _ = run_batch(systems, ctrl, n_non_orth=1)
    for i, (m, div) in enumerate(systems):
        _, p, _ = run_solo(m, div, ctrl, n_non_orth=1)
        assert np.array_equal(ps[i], p)


def test_batch_ldu_solve_matches_solo(systems):
    meshes = [m for m, _ in systems]
    B = vb.Mesh.batch(meshes)
    mats = [vm.poisson_matrix(m) for m in meshes]
    rng = np.random.default_rng(3)
    bs = [rng.standard_normal(m["n_cells"]) for m in meshes]
    x = np.zeros(B.n_cells)
    perf = vb.solve_ldu(B, np.concatenate([d for d, _ in mats]), np.concatenate([u for _, u in mats]), None,
                        np.concatenate(bs), x, vb.SolverControls("PCG", "GAMG", 0.0, 1e-9, 500))
    assert len(perf) == len(meshes)
    for i, m in enumerate(meshes):
        M = vb.Mesh.from_arrays(m)
        xs = np.zeros(m["n_cells"])
        ps = vb.solve_ldu(M, mats[i][0], mats[i][1], None, bs[i], xs, vb.SolverControls("PCG", "GAMG", 0.0, 1e-9, 500))
        assert ps.iterations == perf[i].iterations
        assert np.array_equal(x[B.cell_base[i]:B.cell_base[i + 1]], xs)


@pytest.mark.parametrize("precision", ["", "mixed"])
def test_pressure_corrector_graph_replays_the_direct_run(systems, precision):
    """The batched pressure corrector runs its first call directly and every later call of the same
    configuration as one captured graph (the passes' assembly kernels and solve loops in one launch):
    the replayed calls give the direct call's fields, flux and solver records bit for bit."""
    meshes = [m for m, _ in systems]
    B = vb.Mesh.batch(meshes)
    gamma = cases.batch_face_array(meshes, [np.ones(m["n_faces"]) for m in meshes])
    div = np.concatenate([d for _, d in systems])
    ctrl = vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 500, precision=precision)
    runs = []
    for _ in range(3):
        p = np.zeros(B.n_cells)
        perf, flux = vb.pressure_solve(B, gamma, div, p, ctrl, ref_cell=[0] * len(meshes), n_non_orth=2,
                                       grad_scheme=1)
        runs.append((p, flux, [[(q.iterations, q.finalResidual, q.initialResidual) for q in row] for row in perf]))
    for p, flux, rec in runs[1:]:
        assert np.array_equal(p, runs[0][0]) and np.array_equal(flux, runs[0][1])
        assert rec == runs[0][2]
