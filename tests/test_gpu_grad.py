"""Gradient schemes of the device flow step: the least-squares mesh-default gradient (grad_scheme 1:
fvm::div and the laplacians' non-orthogonal correction, with every U / p boundary type as a value or a
normal-gradient constraint, Fvc.h:264-289) and the leastSquares / GaussSkew pressure gradient
(grad_p_scheme 1 / 2, Fvc.h:233-262), against the reference's own IncompressibleFlow::step in
CFD_REPRODUCIBLE mode (fixtures tests/golden/flow_grad_cases.npz, made by make_grad_golden.py): fields
and residual histories bit for bit."""
import os

import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden", "flow_grad_cases.npz")
TAGS = ("cav_ls_skew", "cav_ls_ls", "cav3d_ls_skew", "totalp_ls", "freestream_ls", "gradient_ls")


def initial_field(C):
    x, y, z = C[:, 0], C[:, 1], C[:, 2]
    return np.stack([np.sin(np.pi * x) * np.cos(np.pi * y), -np.cos(np.pi * x) * np.sin(np.pi * y),
                     0.3 * np.sin(np.pi * z)], 1)


def build(tag):
    if tag.startswith("cav"):
        n = (8, 8, 6) if tag.startswith("cav3d") else (16, 16, 1)
        m, case, _ = cases.skewed_cavity(n)
        if tag == "cav_ls_skew":
            return m, dict(case, div_scheme=2, grad_scheme=1, grad_p_scheme=2), None, 6, 1.0
        if tag == "cav_ls_ls":
            return m, dict(case, div_scheme=1, grad_scheme=1, grad_p_scheme=1), None, 4, 1.0
        c = dict(case, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0, div_scheme=1, grad_scheme=1,
                 grad_p_scheme=2)
        return m, c, initial_field(m["C"]), 3, 0.05
    if tag == "totalp_ls":
        m, case, U0 = cases.channel_total_pressure()
        return m, dict(case, grad_scheme=1, grad_p_scheme=2), U0, 6, 1.0
    if tag == "freestream_ls":
        m, case, U0 = cases.freestream_box()
        return m, dict(case, grad_scheme=1, grad_p_scheme=1), U0, 3, 0.02
    m, case, U0 = cases.channel_gradient()
    return m, dict(case, grad_scheme=1, grad_p_scheme=2), U0, 6, 1.0


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


def test_golden_schemes_change_the_skewed_answer(gold):
    for tag in ("cav_ls_skew", "cav_ls_ls", "cav3d_ls_skew"):
        assert np.abs(gold[f"{tag}_U"] - gold[f"{tag}_gaussU"]).max() > 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("tag", TAGS)
def test_gradient_schemes_bitwise(gold, tag):
    m, case, U0, steps, dt = build(tag)
    fl = vb.Flow(vb.Mesh.from_arrays(m), dict(case, reproducible=True))
    fl.set_state(U0, None)
    hist = []
    for _ in range(steps):
        i = fl.step(dt)
        hist.append([i["UInitialResidual"], i["pInitialResidual"], i["continuityError"]])
    U, p, phi = fl.state()
    fl.close()
    assert np.array_equal(np.array(hist), gold[f"{tag}_hist"][:, :3])
    for k, v in (("U", U), ("p", p), ("phi", phi)):
        assert np.array_equal(v, gold[f"{tag}_{k}"]), k


@pytest.mark.gpu
def test_gradient_scheme_codes_checked():
    m, case, _, _, _ = build("cav_ls_ls")
    for bad in (dict(grad_scheme=2), dict(grad_p_scheme=3)):
        with pytest.raises(vb.VlmError):
            vb.Flow(vb.Mesh.from_arrays(m), dict(case, **bad))
