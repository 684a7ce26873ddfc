"""Generates tests/golden/flow_skew_cases.npz from the reference itself: IncompressibleFlow::step on
skewed meshes (jittered boxes, Mesh::skewed), where the step adds the skew corrections of
fvm::div for linear / LUST (discretization/Fvm.h:83, 119-123), of rAUf and the Rhie-Chow HbyA_f with
least-squares gradients (solvers/IncompressibleFlow.cpp:252-282) and of the initial flux
(IncompressibleFlow.cpp:36); compiled into oracle/_ref/libvlmref.so and driven by oracle/ref_flow.cpp,
in CFD_REPRODUCIBLE mode:
  * skew2d_lu / skew2d_linear / skew2d_lust: the 16 x 16 jittered lid cavity, steady SIMPLE with
    linearUpwind / linear / LUST, 6 / 6 / 4 steps;
  * skew3d: the 8 x 8 x 6 jittered cavity, transient Euler, linear, nCorr 2, 3 steps of dt 0.05 from
    a smooth non-zero initial field;
  * skew2d_default: skew2d_lu in the reference's default (non-reproducible) mode.
Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_skew_golden.py
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


def transient(case):
    return dict(case, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0, div_scheme=1)


CASES = {
    # tag: (n, case transform, steps, dt, initial field)
    "skew2d_lu": ((16, 16, 1), lambda c: dict(c, div_scheme=2), 6, 1.0, False),
    "skew2d_linear": ((16, 16, 1), lambda c: dict(c, div_scheme=1), 6, 1.0, False),
    "skew2d_lust": ((16, 16, 1), lambda c: dict(c, div_scheme=3), 4, 1.0, False),
    "skew3d": ((8, 8, 6), transient, 3, 0.05, True),
}


def main():
    out = {}
    for tag, (n, tf, steps, dt, init) in CASES.items():
        m, case, pts = cases.skewed_cavity(n)
        R = ref.RefMesh(n, points=pts, two_d=n[2] == 1)
        assert R.skewed
        U0 = initial_field(m["C"]) if init else None
        U, p, phi, hist = R.flow_run(tf(case), steps, dt=dt, U=U0, reproducible=True)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
    m, case, pts = cases.skewed_cavity((16, 16, 1))
    R = ref.RefMesh((16, 16, 1), points=pts, two_d=True)
    U, p, phi, hist = R.flow_run(case, 6)
    out.update(skew2d_default_U=U, skew2d_default_p=p, skew2d_default_phi=phi, skew2d_default_hist=hist)
    np.savez_compressed(os.path.join(HERE, "flow_skew_cases.npz"), **out)
    print(sorted(out))


if __name__ == "__main__":
    main()
