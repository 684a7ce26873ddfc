"""Generates tests/golden/flow_grad_cases.npz from the reference itself: IncompressibleFlow::step with
the least-squares mesh-default gradient (gradScheme leastSquares, Mesh::setGradScheme: fvm::div and the
laplacians' non-orthogonal correction) and the leastSquares / GaussSkew pressure gradient (gradPScheme,
discretization/Fvc.h:209-291), as fvmFlow sets them for skewed meshes (apps/fvmFlow/fvmFlow.cpp:149-154);
compiled into oracle/_ref/libvlmref.so and driven by oracle/ref_flow.cpp, in CFD_REPRODUCIBLE mode:
  * cav_ls_skew: the 16 x 16 jittered lid cavity, linearUpwind, leastSquares + GaussSkew, 6 SIMPLE steps;
  * cav_ls_ls: the same with linear divergence, leastSquares + leastSquares, 4 steps;
  * cav3d_ls_skew: the 8 x 8 x 6 jittered cavity, transient Euler (nCorr 2), linear, leastSquares +
    GaussSkew, 3 steps of dt 0.05 from a smooth field;
  * totalp_ls: the total-pressure inlet channel (symmetry walls, pressureInletOutletVelocity,
    inletOutlet, totalPressure) with leastSquares + GaussSkew, 6 steps;
  * freestream_ls: the freestream vortex box with leastSquares + leastSquares, 3 steps of dt 0.02;
  * gradient_ls: the fixedGradient channel with leastSquares + GaussSkew, 6 steps.
Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_grad_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import cases  # noqa: E402


def initial_field(C):
    x, y, z = C[:, 0], C[:, 1], C[:, 2]
    return np.stack([np.sin(np.pi * x) * np.cos(np.pi * y), -np.cos(np.pi * x) * np.sin(np.pi * y),
                     0.3 * np.sin(np.pi * z)], 1)


def build(tag):
    """(mesh dict, RefMesh, case, U0, steps, dt) of one case."""
    if tag.startswith("cav"):
        n = (8, 8, 6) if tag.startswith("cav3d") else (16, 16, 1)
        m, case, pts = cases.skewed_cavity(n)
        R = ref.RefMesh(n, points=pts, two_d=n[2] == 1)
        if tag == "cav_ls_skew":
            return m, R, dict(case, div_scheme=2, grad_scheme=1, grad_p_scheme=2), None, 6, 1.0
        if tag == "cav_ls_ls":
            return m, R, dict(case, div_scheme=1, grad_scheme=1, grad_p_scheme=1), None, 4, 1.0
        c = dict(case, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0, div_scheme=1, grad_scheme=1,
                 grad_p_scheme=2)
        return m, R, c, initial_field(m["C"]), 3, 0.05
    if tag == "totalp_ls":
        m, case, U0 = cases.channel_total_pressure()
        R = ref.RefMesh((40, 10, 1), hi=(4.0, 1.0, 0.1), two_d=True)
        return m, R, dict(case, grad_scheme=1, grad_p_scheme=2), U0, 6, 1.0
    if tag == "freestream_ls":
        m, case, U0 = cases.freestream_box()
        R = ref.RefMesh((32, 16, 1), hi=(2.0, 1.0, 0.1), two_d=True)
        return m, R, dict(case, grad_scheme=1, grad_p_scheme=1), U0, 3, 0.02
    m, case, U0 = cases.channel_gradient()
    R = ref.RefMesh((40, 10, 1), hi=(4.0, 1.0, 0.1), two_d=True)
    return m, R, dict(case, grad_scheme=1, grad_p_scheme=2), U0, 6, 1.0


TAGS = ("cav_ls_skew", "cav_ls_ls", "cav3d_ls_skew", "totalp_ls", "freestream_ls", "gradient_ls")


def main():
    out = {}
    for tag in TAGS:
        m, R, case, U0, steps, dt = build(tag)
        U, p, phi, hist = R.flow_run(case, steps, dt=dt, U=U0, reproducible=True)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
        # the same case with the Gauss gradients, to show the schemes change the answer
        g = dict(case, grad_scheme=0, grad_p_scheme=0)
        Ug, _, _, _ = R.flow_run(g, steps, dt=dt, U=U0, reproducible=True)
        out[f"{tag}_gaussU"] = Ug
    np.savez_compressed(os.path.join(HERE, "flow_grad_cases.npz"), **out)
    print(sorted(out))


if __name__ == "__main__":
    main()
