"""Generates tests/golden/flow_cases.npz from the reference itself: IncompressibleFlow::step
(solvers/IncompressibleFlow.cpp) compiled from the reference's own sources into oracle/_ref/libvlmref.so
and driven by oracle/ref_flow.cpp, on the lid-driven cavity (cases/cavity/case.json settings) and the
Taylor-Green vortex (fvmFlow transient defaults).  Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_flow_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import cases  # noqa: E402


def ref_mesh(m):
    nx, ny, nz = m["shape"]
    hi = (1.0, 1.0, 0.1) if m["two_d"] else (2 * np.pi,) * 3
    return ref.RefMesh((nx, ny, nz), hi=hi, periodic=m["periodic"], two_d=bool(m["two_d"]))


def main():
    out = {}
    # lid cavity 16x16: 8 SIMPLE iterations in CFD_REPRODUCIBLE mode and in the default mode
    m, case = cases.lid_cavity(16, 100.0)
    R = ref_mesh(m)
    for tag, repro in (("cav16_repro", True), ("cav16", False)):
        U, p, phi, hist = R.flow_run(case, 8, reproducible=repro)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
    # lid cavity 32x32 to convergence (residualTol 1e-6, fvmFlow.cpp:611-625)
    m, case = cases.lid_cavity(32, 100.0)
    R = ref_mesh(m)
    U, p, phi, hist = R.flow_run(case, 3000)
    conv = next(i + 1 for i in range(1, len(hist)) if hist[i, 0] < 1e-6 and hist[i, 1] < 1e-6)
    U, p, phi, hist = R.flow_run(case, conv)
    out.update(cav32_U=U, cav32_p=p, cav32_phi=phi, cav32_iters=np.array(conv))
    # Taylor-Green 12^3: 4 PIMPLE steps of dt = 0.05 (reproducible and default)
    m, case, U0 = cases.taylor_green_flow(12)
    R = ref_mesh(m)
    for tag, repro in (("tgv12_repro", True), ("tgv12", False)):
        U, p, phi, hist = R.flow_run(case, 4, dt=0.05, U=U0, reproducible=repro)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
    np.savez_compressed(os.path.join(HERE, "flow_cases.npz"), **out)
    print("cavity32 converged in", conv, "iterations")


if __name__ == "__main__":
    main()
