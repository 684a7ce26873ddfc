"""The device incompressible step on skewed meshes (jittered boxes): the skew corrections of
fvm::div for linear / LUST (Fvm.h:83, 119-123), of rAUf and the Rhie-Chow HbyA_f with least-squares
gradients (IncompressibleFlow.cpp:252-282) and of the initial flux (IncompressibleFlow.cpp:36), against
the reference's own IncompressibleFlow::step in CFD_REPRODUCIBLE mode (fixtures
tests/golden/flow_skew_cases.npz, made by make_skew_golden.py): fields and residual histories bit for
bit."""
import os

import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden", "flow_skew_cases.npz")


def initial_field(C):
    x, y, z = C[:, 0], C[:, 1], C[:, 2]
    return np.stack([np.sin(np.pi * x) * np.cos(np.pi * y), -np.cos(np.pi * x) * np.sin(np.pi * y),
                     0.3 * np.sin(np.pi * z)], 1)


def transient(case):
    return dict(case, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0, div_scheme=1)


CASES = {
    "skew2d_lu": ((16, 16, 1), lambda c: dict(c, div_scheme=2), 6, 1.0, False),
    "skew2d_linear": ((16, 16, 1), lambda c: dict(c, div_scheme=1), 6, 1.0, False),
    "skew2d_lust": ((16, 16, 1), lambda c: dict(c, div_scheme=3), 4, 1.0, False),
    "skew3d": ((8, 8, 6), transient, 3, 0.05, True),
}


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


def run(tag, reproducible=True):
    n, tf, steps, dt, init = CASES[tag]
    m, case, _ = cases.skewed_cavity(n)
    case = dict(tf(case), reproducible=reproducible)
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_state(initial_field(m["C"]) if init else None, None)
    hist = []
    for _ in range(steps):
        i = fl.step(dt)
        hist.append([i["UInitialResidual"], i["pInitialResidual"], i["continuityError"]])
    U, p, phi = fl.state()
    fl.close()
    return U, p, phi, np.array(hist)


def test_cases_are_skewed():
    for n in ((16, 16, 1), (8, 8, 6)):
        m, _, _ = cases.skewed_cavity(n)
        assert m["skewed"]


def test_golden_skew_changes_the_answer(gold):
    # the corrections matter: linear and linearUpwind differ, and the fields are not those of the
    # unjittered cavity (which has no skew)
    assert not np.array_equal(gold["skew2d_lu_U"], gold["skew2d_linear_U"])
    assert np.abs(gold["skew2d_linear_U"]).max() > 0.1


@pytest.mark.gpu
@pytest.mark.parametrize("tag", sorted(CASES))
def test_skewed_cavity_bitwise(gold, tag):
    U, p, phi, hist = run(tag)
    assert np.array_equal(hist, gold[f"{tag}_hist"][:, :3])
    assert np.array_equal(U, gold[f"{tag}_U"])
    assert np.array_equal(p, gold[f"{tag}_p"])
    assert np.array_equal(phi, gold[f"{tag}_phi"])


@pytest.mark.gpu
def test_skewed_cavity_default_mode_close(gold):
    # default (fast) mode against the reference's default mode, within the solver tolerances
    # (U relTol 0.1, p relTol 0.05 per outer iteration)
    U, p, phi, hist = run("skew2d_lu", reproducible=False)
    ref = gold["skew2d_default_U"]
    assert np.abs(U - ref).max() < 5e-3 * np.abs(ref).max()
