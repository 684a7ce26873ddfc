"""The headline system at its full size: the 128^3 periodic Taylor-Green pressure equation that
bench.py times (2,097,152 cells; laplacian(rAUf = 2e-3) minus the divergence of the predicted
flux, setReference(0)), solved from p = 0 to relTol 1e-8 by the device's GAMG-PCG in FP64 and in
mixed precision (FP32 V-cycle in the FP64 recurrence), against the oracle's restatement of the
same schedule (level-0 multicolour Gauss-Seidel, Jacobi coarse levels, explicit coarsest inverse):
iteration counts within +-1, solution within relative L2 1e-10 of the oracle's iterate at the
device's iteration count.  The reference's own sequential Gauss-Seidel GAMG takes 39 iterations
on this system; the device schedule takes 47 (its parallel smoother is weaker per sweep)."""
import numpy as np
import pytest

import bench
import voluma_b200 as vb
from oracle import restate as ro
from test_gpu_solve import oracle_iterate, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tgv128():
    m = vb.box_mesh_device((128, 128, 128), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    d, up, b = bench.assemble(m)
    x0 = np.zeros(m["n_cells"])
    xo, po = ro.solve(m, d, up, None, b, x0, "PCG", "GAMG", 0.0, 1e-8, 1000, smoother="mcgs-jacobi", coarse=1)
    return m, d, up, b, x0, xo, po, vb.Mesh.from_arrays(m)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tgv128_gamg_pcg_matches_oracle(tgv128, precision):
    m, d, up, b, x0, xo, po, mesh = tgv128
    nI = m["n_internal_faces"]
    assert vb.box_shape(m["n_cells"], m["owner"][:nI], m["neighbour"][:nI])["layout"]
    x = x0.copy()
    p = vb.solve_ldu(mesh, d, up, None, b, x, vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 1000, precision=precision))
    assert p.converged and po["converged"]
    assert abs(p.iterations - po["iterations"]) <= 1
    assert rel(x, oracle_iterate(m, d, up, b, x0, xo, po, p.iterations)) <= 1e-10


@pytest.fixture(scope="module")
def tgv128_device_agglomeration(tgv128):
    m, d, up, b, x0 = tgv128[:5]
    xo, po = ro.solve(m, d, up, None, b, x0, "PCG", "GAMG", 0.0, 1e-8, 1000, smoother="mcgs-jacobi", coarse=1,
                      matching=True)
    return xo, po, vb.Mesh.from_arrays(m, agglomeration="device")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_tgv128_device_agglomeration_matches_oracle(tgv128, tgv128_device_agglomeration, precision):
    """The same system on the device-built hierarchy (parallel matching) against the restatement of
    that hierarchy and schedule: iterations +-1 (42 on both), relative L2 1e-10 at equal work."""
    m, d, up, b, x0 = tgv128[:5]
    xo, po, mesh = tgv128_device_agglomeration
    x = x0.copy()
    p = vb.solve_ldu(mesh, d, up, None, b, x, vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 1000, precision=precision))
    assert p.converged and po["converged"]
    assert abs(p.iterations - po["iterations"]) <= 1
    if p.iterations != po["iterations"]:
        xo, _ = ro.solve(m, d, up, None, b, x0, "PCG", "GAMG", 0.0, 0.0, p.iterations, smoother="mcgs-jacobi",
                         coarse=1, matching=True)
    assert rel(x, xo) <= 1e-10
