"""The device incompressible step (vlm_flow_*, csrc/flow.cu) against the reference's own
IncompressibleFlow::step (fixtures in tests/golden/flow_cases.npz, made by make_flow_golden.py).

* CFD_REPRODUCIBLE mode (exact sums, diagonal preconditioning, as the reference swaps them): every
  field after several SIMPLE / PIMPLE steps, and the per-step residual history, bit for bit.
* Default mode (GAMG pressure, DILU momentum, compensated sums on the device): per-step figures
  within the solvers' tolerances of the reference's, and the converged 32x32 cavity within 2e-5 of
  the reference's converged fields, in the same number of SIMPLE iterations +-2 %.
"""
import os

import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "flow_cases.npz")


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


def flow_for(m, case):
    mesh = vb.Mesh.from_arrays(m)
    return mesh, vb.Flow(mesh, case)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run(m, case, n, dt=1.0, U0=None):
    mesh, fl = flow_for(m, case)
    fl.set_state(U0, None)
    hist = []
    for _ in range(n):
        i = fl.step(dt)
        hist.append([i["UInitialResidual"], i["pInitialResidual"], i["continuityError"]])
    U, p, phi = fl.state()
    fl.close()
    return U, p, phi, np.array(hist)


def test_cavity_reproducible_bitwise(gold):
    m, case = cases.lid_cavity(16, 100.0)
    case["reproducible"] = True
    U, p, phi, hist = run(m, case, 8)
    assert np.array_equal(hist, gold["cav16_repro_hist"][:, :3])
    assert np.array_equal(U, gold["cav16_repro_U"])
    assert np.array_equal(p, gold["cav16_repro_p"])
    assert np.array_equal(phi, gold["cav16_repro_phi"])


def test_taylor_green_reproducible_bitwise(gold):
    m, case, U0 = cases.taylor_green_flow(12)
    case["reproducible"] = True
    U, p, phi, hist = run(m, case, 4, dt=0.05, U0=U0)
    assert np.array_equal(hist, gold["tgv12_repro_hist"][:, :3])
    assert np.array_equal(U, gold["tgv12_repro_U"])
    assert np.array_equal(p, gold["tgv12_repro_p"])
    assert np.array_equal(phi, gold["tgv12_repro_phi"])


def test_default_mode_cavity_tracks_reference(gold):
    """SIMPLE with pressure solves stopped at relTol 0.05: the device GAMG (multicolour smoother)
    and the reference's (sequential Gauss-Seidel) stop at different partial solutions, so per-step
    figures agree to the solver tolerance, not to rounding."""
    m, case = cases.lid_cavity(16, 100.0)
    U, p, phi, hist = run(m, case, 8)
    ref = gold["cav16_hist"][:, :3]
    assert np.allclose(hist[:, :2], ref[:, :2], rtol=5e-3)
    assert np.all(hist[:, 2] < 3.0 * ref[:, 2] + 1e-12)
    assert rel(U, gold["cav16_U"]) < 5e-3


def test_default_mode_taylor_green_tracks_reference(gold):
    """PIMPLE whose momentum and final pressure solves converge to 1e-8 (normalised residual): the
    fields agree to a few times that tolerance."""
    m, case, U0 = cases.taylor_green_flow(12)
    U, p, phi, hist = run(m, case, 4, dt=0.05, U0=U0)
    ref = gold["tgv12_hist"][:, :3]
    assert np.allclose(hist[:, :2], ref[:, :2], rtol=1e-4)
    assert np.all(hist[:, 2] < 1e-8)
    assert rel(U, gold["tgv12_U"]) < 1e-5
    assert rel(phi, gold["tgv12_phi"]) < 1e-5


def test_cavity32_converges_like_reference(gold):
    m, case = cases.lid_cavity(32, 100.0)
    mesh, fl = flow_for(m, case)
    fl.set_state(None, None)
    its, last = fl.run_steady(3000, 1e-6)
    U, p, phi = fl.state()
    fl.close()
    ref_its = int(gold["cav32_iters"])
    assert abs(its - ref_its) <= max(2, int(0.02 * ref_its))
    assert last["UInitialResidual"] < 1e-6 and last["pInitialResidual"] < 1e-6
    assert rel(U, gold["cav32_U"]) < 2e-5
    assert rel(p - p.mean(), gold["cav32_p"] - gold["cav32_p"].mean()) < 2e-4


def test_flow_rejects_bad_settings():
    m, case = cases.lid_cavity(8, 100.0)
    mesh = vb.Mesh.from_arrays(m)
    bad = dict(case, div_scheme=9)
    with pytest.raises(vb.VlmError) as e:
        vb.Flow(mesh, bad)
    assert e.value.name == "BAD_ARG"
    nocentres = {k: v for k, v in m.items() if k not in ("C", "Cf")}
    mesh2 = vb.Mesh.from_arrays(nocentres)
    with pytest.raises(vb.VlmError) as e:
        vb.Flow(mesh2, case)  # linearUpwind needs the cell and face centres
    assert e.value.name == "BAD_ARG"


@pytest.fixture(scope="module")
def cav64():
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "flow_cavity64.npz"))
    return {k: z[k] for k in z.files}


def fnv1a(a):
    """The reference's field checksum (fieldChecksum, VtkWriter.cpp:81-99): 64-bit FNV-1a over the
    bytes of the doubles in cell order."""
    h = 0xcbf29ce484222325
    for byte in np.ascontiguousarray(a, np.float64).tobytes():
        h ^= byte
        h = (h * 0x100000001b3) & 0xffffffffffffffff
    return h


def test_cavity64_steady_like_reference(cav64):
    """The lid-driven cavity of cases/cavity/case.json (64x64, Re 100, steady SIMPLE to residualTol
    1e-6): the reference converges in 1161 iterations.  Default mode (device GAMG with its
    multicolour smoother): the iteration count within +-2 % of the reference's and the converged
    fields within 2e-5 (U) and 2e-4 (p, relative to its mean) of the reference's."""
    m, case = cases.lid_cavity(64, 100.0)
    mesh, fl = flow_for(m, case)
    fl.set_state(None, None)
    its, last = fl.run_steady(20000, 1e-6)
    U, p, phi = fl.state()
    fl.close()
    ref_its = int(cav64["cav64_iters"])
    assert ref_its == 1161
    assert abs(its - ref_its) <= int(0.02 * ref_its)
    assert last["UInitialResidual"] < 1e-6 and last["pInitialResidual"] < 1e-6
    assert rel(U, cav64["cav64_U"]) < 2e-5
    assert rel(p - p.mean(), cav64["cav64_p"] - cav64["cav64_p"].mean()) < 2e-4


def test_cavity64_reproducible_to_convergence_bitwise(cav64):
    """The same case in CFD_REPRODUCIBLE mode, run to convergence: the same iteration count and the
    converged fields bit for bit (so the reference's field checksums too)."""
    m, case = cases.lid_cavity(64, 100.0)
    case["reproducible"] = True
    mesh, fl = flow_for(m, case)
    fl.set_state(None, None)
    its, last = fl.run_steady(20000, 1e-6)
    U, p, phi = fl.state()
    fl.close()
    assert its == int(cav64["cav64_repro_iters"])
    assert np.array_equal(U, cav64["cav64_repro_U"]) and np.array_equal(p, cav64["cav64_repro_p"])
    assert fnv1a(U) == fnv1a(cav64["cav64_repro_U"]) and fnv1a(p) == fnv1a(cav64["cav64_repro_p"])
