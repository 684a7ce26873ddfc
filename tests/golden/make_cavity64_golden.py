"""Generates tests/golden/flow_cavity64.npz from the reference itself: the 64x64 lid-driven cavity
(cases/cavity/case.json: Re 100, the fvmFlow steady defaults) run by the reference's own
IncompressibleFlow::step (compiled from its sources into oracle/_ref/libvlmref.so, driven by
oracle/ref_flow.cpp) to residualTol 1e-6 as fvmFlow's steady loop stops it (fvmFlow.cpp:611-625),
in the default mode and in CFD_REPRODUCIBLE mode.  Stores the converged U, p, phi and the iteration
counts, and the FNV-1a checksums the reference prints for U and p (VtkWriter.cpp:81-99).
Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_cavity64_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import cases  # noqa: E402


def fnv1a(a):
    """64-bit FNV-1a over the bytes of a double array (the reference's field checksum)."""
    h = 0xcbf29ce484222325
    for byte in np.ascontiguousarray(a, np.float64).tobytes():
        h ^= byte
        h = (h * 0x100000001b3) & 0xffffffffffffffff
    return h


def main():
    m, case = cases.lid_cavity(64, 100.0)
    R = ref.RefMesh((64, 64, 1), hi=(1.0, 1.0, 0.1), two_d=True)
    out = {}
    for tag, repro in (("cav64", False), ("cav64_repro", True)):
        U, p, phi, hist = R.flow_run(case, 20000, reproducible=repro, residual_tol=1e-6)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_iters": np.array(len(hist)),
                    f"{tag}_hist": hist})
        print(tag, "converged in", len(hist), "iterations; checksum U", f"{fnv1a(U):016x}", "p", f"{fnv1a(p):016x}")
    np.savez_compressed(os.path.join(HERE, "flow_cavity64.npz"), **out)


if __name__ == "__main__":
    main()
