"""Parity of the device assembly (fvm::laplacian with non-orthogonal correction, fvc::grad,
fvc::div, the pressure-corrector loop) with the reference's own results in tests/golden/.
The kernels gather over each cell's faces in ascending face order, so the comparison is bit
for bit."""
import numpy as np
import pytest

from conftest import golden_names
from test_gpu_solve import device_mesh, rel
import voluma_b200 as vb

pytestmark = pytest.mark.gpu

KEYS = ("diag", "upper", "source", "internalCoeffs", "boundarySource", "ffc")


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("scheme", [0, 1])
def test_laplacian_bitwise(name, scheme):
    g, m = device_mesh(name)
    nP = len(g["patchStart"])
    L = vb.laplacian(m, g["lap_gamma"], g["lap_psi"], g["lap_bctype"][:nP], g["lap_bcvalues"], True, scheme)
    for k in KEYS:
        assert np.array_equal(L[k], g[f"lap{scheme}_{k}"]), k
    assert L["hasFfc"] == bool(g[f"lap{scheme}_hasFfc"])


@pytest.mark.parametrize("name", golden_names())
@pytest.mark.parametrize("scheme", [0, 1])
def test_grad_bitwise(name, scheme):
    g, m = device_mesh(name)
    nP = len(g["patchStart"])
    gr = vb.grad(m, g["lap_psi"], g["lap_bctype"][:nP], g["lap_bcvalues"], scheme)
    assert np.array_equal(gr, g[f"grad{scheme}"])


@pytest.mark.parametrize("name", golden_names())
def test_div_matches_face_loop(name):
    g, m = device_mesh(name)
    F = np.random.default_rng(4).standard_normal(g["n_faces"])
    nI = g["n_internal_faces"]
    r = np.zeros(g["n_cells"])
    # Fvc.h:294-304: owner +F, neighbour -F, face order; then / V
    idx = np.stack([g["owner"][:nI], g["neighbour"]], 1).ravel()
    np.add.at(r, idx, np.stack([F[:nI], -F[:nI]], 1).ravel())
    np.add.at(r, g["owner"][nI:], F[nI:])
    assert np.array_equal(vb.div(m, F), r / g["V"])


@pytest.mark.parametrize("name", golden_names())
def test_pressure_loop_reproducible_bitwise(name):
    """laplacian (LS non-orthogonal correction) - divPhi, setReference(0), PCG/diagonal in
    CFD_REPRODUCIBLE mode, three passes: p and the final flux equal the reference's bit for bit."""
    g, m = device_mesh(name)
    p = np.zeros(g["n_cells"])
    ctrl = vb.SolverControls("PCG", "diagonal", 0.0, 1e-8, 3000, reproducible=True)
    perf, flux = vb.pressure_solve(m, g["ps_gamma"], g["ps_divphi"], p, ctrl, ref_cell=0, n_non_orth=2,
                                   grad_scheme=1)
    assert [q.iterations for q in perf] == [int(v) for v in g["ps_perf"][:, 4]]
    assert np.array_equal(p, g["ps_p"])
    assert np.array_equal(flux, g["ps_flux"])


@pytest.mark.parametrize("name", golden_names())
def test_pressure_loop_gamg(name):
    g, m = device_mesh(name)
    p = np.zeros(g["n_cells"])
    ctrl = vb.SolverControls("PCG", "GAMG", 0.0, 1e-8, 3000)
    perf, flux = vb.pressure_solve(m, g["ps_gamma"], g["ps_divphi"], p, ctrl, ref_cell=0, n_non_orth=2,
                                   grad_scheme=1)
    assert all(q.converged for q in perf)
    # both solutions satisfy relTol 1e-8; they agree to the solver tolerance
    assert rel(p, g["ps_p"]) <= 1e-5
    assert rel(flux, g["ps_flux"]) <= 1e-5


@pytest.mark.gpu
def test_scalar_boundary_types_checked():
    # a mixed boundary needs value fractions that only the flow step supplies, and unknown types are
    # refused: neither reaches a kernel
    from voluma_b200 import mesh as vm
    M = vm.box_mesh((6, 5, 4))
    m = vb.Mesh.from_arrays(M)
    nP = len(M["patch_start"])
    psi = np.linspace(0.0, 1.0, M["n_cells"])
    for t in (3, 4, 9, -1):
        with pytest.raises(vb.VlmError):
            vb.grad(m, psi, np.full(nP, t, np.int32))
        with pytest.raises(vb.VlmError):
            vb.laplacian(m, np.ones(M["n_faces"]), psi, np.full(nP, t, np.int32))
    # symmetry is a zero gradient for a scalar; a zero fixedGradient is too
    g0 = vb.grad(m, psi, np.zeros(nP, np.int32))
    assert np.array_equal(vb.grad(m, psi, np.full(nP, 2, np.int32)), g0)
    assert np.array_equal(vb.grad(m, psi, np.full(nP, 5, np.int32), np.zeros(M["n_faces"] - M["n_internal_faces"])), g0)
