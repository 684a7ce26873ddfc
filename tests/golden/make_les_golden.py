"""Generates tests/golden/flow_les_cases.npz from the reference itself: IncompressibleFlow::step with the
reference's Smagorinsky LES model (models/LESModels.cpp, built by TurbulenceModel::create from the
"turbulence" dictionary) and its mean-velocity / constant momentum forcing, compiled from the reference's
own sources into oracle/_ref/libvlmref.so and driven by oracle/ref_flow.cpp, on a small periodic channel
(voluma_b200.cases.channel at 8 x 12 x 6).  Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_les_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import cases  # noqa: E402

N = (8, 12, 6)
STEPS = 3


def channel_case(les, van_driest, forcing="meanVelocity"):
    m, case, model, U0, dt = cases.channel(N, les=les, van_driest=van_driest)
    model = dict(model, forcing=forcing)
    if forcing == "constant":
        model["force"] = (2e-3, 0.0, 0.0)
    return m, case, model, U0, dt


def main():
    beta = cases.channel_beta(N[1], 1.0 / 395.0)
    R = ref.RefMesh(N, hi=(2 * np.pi, 2.0, np.pi), periodic=(1, 0, 1), beta=(0, beta, 0), patch_types=[0, 0, 1, 1, 0, 0])
    out = {}
    runs = (("les_repro", True, False, "meanVelocity", True), ("lesvd_repro", True, True, "meanVelocity", True),
            ("lesvd", True, True, "meanVelocity", False), ("lam_repro", False, False, "meanVelocity", True),
            ("const_repro", False, False, "constant", True))
    for tag, les, vd, forcing, repro in runs:
        m, case, model, U0, dt = channel_case(les, vd, forcing)
        U, p, phi, hist, nut, gp = R.flow_run(case, STEPS, dt=dt, U=U0, reproducible=repro, model=model)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist, f"{tag}_nut": nut,
                    f"{tag}_gradP": np.array(gp)})
        print(tag, "gradP", gp, "max nut", nut.max(), "hist", hist[-1])
    np.savez_compressed(os.path.join(HERE, "flow_les_cases.npz"), **out)


if __name__ == "__main__":
    main()
