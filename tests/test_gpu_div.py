"""The TVD-limited divergence schemes of the device momentum equation (limitedLinear k, vanLeer,
MUSCL, minmod; fvm::div, Fvm.h:47-137) against the reference's own IncompressibleFlow::step in
CFD_REPRODUCIBLE mode (fixtures tests/golden/flow_div_cases.npz, made by make_div_golden.py): fields
and residual histories bit for bit."""
import os

import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "flow_div_cases.npz")
SCHEMES = {"ll1": (4, 1.0), "ll05": (4, 0.5), "vanLeer": (5, 1.0), "MUSCL": (6, 1.0), "minmod": (7, 1.0)}


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


def run(m, case, n, dt=1.0, U0=None):
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_state(U0, None)
    hist = []
    for _ in range(n):
        i = fl.step(dt)
        hist.append([i["UInitialResidual"], i["pInitialResidual"], i["continuityError"]])
    U, p, phi = fl.state()
    fl.close()
    return U, p, phi, np.array(hist)


@pytest.mark.parametrize("tag", sorted(SCHEMES))
def test_cavity_limited_schemes_bitwise(gold, tag):
    code, k = SCHEMES[tag]
    m, case = cases.lid_cavity(16, 100.0)
    case = dict(case, div_scheme=code, div_coeff=k, reproducible=True)
    U, p, phi, hist = run(m, case, 6)
    assert np.array_equal(hist, gold[f"cav_{tag}_hist"][:, :3])
    assert np.array_equal(U, gold[f"cav_{tag}_U"])
    assert np.array_equal(p, gold[f"cav_{tag}_p"])
    assert np.array_equal(phi, gold[f"cav_{tag}_phi"])


def test_taylor_green_vanleer_bitwise(gold):
    m, case, U0 = cases.taylor_green_flow(12)
    case = dict(case, div_scheme=5, reproducible=True)
    U, p, phi, hist = run(m, case, 3, dt=0.05, U0=U0)
    assert np.array_equal(hist, gold["tgv_vanLeer_hist"][:, :3])
    assert np.array_equal(U, gold["tgv_vanLeer_U"])
    assert np.array_equal(phi, gold["tgv_vanLeer_phi"])


def test_schemes_differ(gold):
    # the limiters are active: different schemes give different fields
    assert not np.array_equal(gold["cav_vanLeer_U"], gold["cav_minmod_U"])
    assert not np.array_equal(gold["cav_ll1_U"], gold["cav_ll05_U"])
