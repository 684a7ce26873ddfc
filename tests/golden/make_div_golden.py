"""Generates tests/golden/flow_div_cases.npz from the reference itself: IncompressibleFlow::step with the
TVD-limited divergence schemes of fvm::div (Fvm.h:47-137: limitedLinear k, vanLeer, MUSCL, minmod),
compiled into oracle/_ref/libvlmref.so and driven by oracle/ref_flow.cpp, in CFD_REPRODUCIBLE mode:
the 16 x 16 lid cavity (6 SIMPLE steps) per scheme and the 12^3 Taylor-Green vortex with vanLeer
(3 PIMPLE steps).  Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_div_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import cases  # noqa: E402

SCHEMES = {"ll1": (4, 1.0), "ll05": (4, 0.5), "vanLeer": (5, 1.0), "MUSCL": (6, 1.0), "minmod": (7, 1.0)}


def main():
    out = {}
    m, case = cases.lid_cavity(16, 100.0)
    R = ref.RefMesh((16, 16, 1), hi=(1.0, 1.0, 0.1), two_d=True)
    for tag, (code, k) in SCHEMES.items():
        c = dict(case, div_scheme=code, div_coeff=k)
        U, p, phi, hist = R.flow_run(c, 6, reproducible=True)
        out.update({f"cav_{tag}_U": U, f"cav_{tag}_p": p, f"cav_{tag}_phi": phi, f"cav_{tag}_hist": hist})
    m, case, U0 = cases.taylor_green_flow(12)
    R = ref.RefMesh((12, 12, 12), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    c = dict(case, div_scheme=5)
    U, p, phi, hist = R.flow_run(c, 3, dt=0.05, U=U0, reproducible=True)
    out.update(tgv_vanLeer_U=U, tgv_vanLeer_p=p, tgv_vanLeer_phi=phi, tgv_vanLeer_hist=hist)
    np.savez_compressed(os.path.join(HERE, "flow_div_cases.npz"), **out)
    print(sorted(out))


if __name__ == "__main__":
    main()
