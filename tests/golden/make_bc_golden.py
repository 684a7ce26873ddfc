"""Generates tests/golden/flow_bc_cases.npz from the reference itself: IncompressibleFlow::step with
symmetry (slip) planes for U and p (SymmetryBC, field/BoundaryCondition.h:194-205 and
field/VolField.h:156-191), compiled into oracle/_ref/libvlmref.so and driven by oracle/ref_flow.cpp, in
CFD_REPRODUCIBLE mode:
  * slip2d: the 16 x 16 sheared slip cavity (leaning slip walls, one non-orthogonal corrector),
    6 SIMPLE steps;
  * slip2d_flat: the same without shear, 4 SIMPLE steps;
  * slip3d: the 8 x 8 x 6 sheared slip cavity (slip x and z walls), transient Euler with nCorr 2,
    3 steps of dt 0.05;
  * slip2d_default: slip2d in the reference's default (non-reproducible) mode;
  * inlet / inlet_backflow / inlet_transient: the 40 x 10 inlet-outlet channel (parabolic fixedValue
    inlet given face by face, inletOutlet outlet, InletOutletBC BoundaryCondition.h:263-287), steady
    SIMPLE 6 steps from U = (1, 0, 0) and from a field with backflow at the outlet, and transient
    Euler (nCorr 2, 3 steps of dt 0.02) from the backflow field;
  * freestream: a vortex carried through the 32 x 16 box with freestream U / freestreamPressure p on
    every side (FreestreamVelocityBC, FreestreamPressureBC, BoundaryCondition.h:289-320), transient
    Euler, 4 steps of dt 0.02;
  * gradient: the inlet-outlet channel with fixedGradient p at the inlet and fixedGradient U at the
    outlet (FixedGradientBC, BoundaryCondition.h:140-153), steady SIMPLE, 6 steps;
  * fluxp / fluxpo: the inlet-outlet channel with fixedFluxPressure p at the inlet / at the outlet
    (FixedFluxPressureBC, BoundaryCondition.h:155-163; IncompressibleFlow.cpp:17-29), steady SIMPLE,
    6 steps;
  * totalp: the total-pressure inlet of cases/channelInlet/totalPressure.json (TotalPressureBC with
    PressureInletOutletVelocityBC, BoundaryCondition.h:325-364), steady SIMPLE, 8 steps from rest;
  * robin / robin_walls / robin_gradient: the inlet-outlet channel with Robin U and p at the outlet
    (RobinBC, BoundaryCondition.h:166-192), also with Robin (partial-slip-like) U walls, and with a
    pure-gradient Robin (a = 0) outlet; steady SIMPLE, 6 steps; robin_transient: Euler, nCorr 2,
    3 steps of dt 0.02;
  * adv_euler / adv_backward / adv_far / adv_steady: the inlet-outlet channel with an advective U
    outlet (AdvectiveBC, BoundaryCondition.h:389-414, VolField.h:235-264) and p fixed there: PISO
    (nCorr 2) Euler 4 steps and backward 5 steps of dt 0.02, backward with the far-field relaxation
    (lInf 0.5 towards (0.8, 0.05, 0)), and steady SIMPLE 3 steps (zero gradient).
Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_bc_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import cases  # noqa: E402


def transient(case):
    return dict(case, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0)


CASES = {
    # tag: (n, shear, case transform, steps, dt)
    "slip2d": ((16, 16, 1), 0.3, dict, 6, 1.0),
    "slip2d_flat": ((16, 16, 1), 0.0, dict, 4, 1.0),
    "slip3d": ((8, 8, 6), 0.3, transient, 3, 0.05),
}


INLET = {
    # tag: (backflow, case transform, steps, dt)
    "inlet": (0.0, dict, 6, 1.0),
    "inlet_backflow": (0.5, dict, 6, 1.0),
    "inlet_transient": (0.5, lambda c: dict(c, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0), 3,
                        0.02),
}


# tag, steps, dt of the advective-outlet channels (advective_case builds them)
ADVECTIVE = (("adv_euler", 4, 0.02), ("adv_backward", 5, 0.02), ("adv_far", 5, 0.02), ("adv_steady", 3, 1.0))


def advective_case(tag):
    kw = {"adv_euler": dict(ddt_scheme=1), "adv_backward": dict(ddt_scheme=2),
          "adv_far": dict(ddt_scheme=2, far_field=(0.5, (0.8, 0.05, 0.0))), "adv_steady": dict(ddt_scheme=0)}[tag]
    m, case, U0 = cases.channel_advective(**kw)
    if tag == "adv_steady":
        case = dict(case, steady=True, n_corr=1, alpha_u=0.7, alpha_p=0.3)
    return m, case, U0


def main():
    out = {}
    for tag, (n, shear, tf, steps, dt) in CASES.items():
        m, case, pts = cases.slip_cavity(n, shear)
        R = ref.RefMesh(n, points=pts, two_d=n[2] == 1)
        U, p, phi, hist = R.flow_run(tf(case), steps, dt=dt, reproducible=True)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
    # the reference's default mode (DILU, GAMG with Gauss-Seidel) for the loose default-mode comparison
    m, case, pts = cases.slip_cavity((16, 16, 1), 0.3)
    R = ref.RefMesh((16, 16, 1), points=pts, two_d=True)
    U, p, phi, hist = R.flow_run(case, 6)
    out.update(slip2d_default_U=U, slip2d_default_p=p, slip2d_default_phi=phi, slip2d_default_hist=hist)
    for tag, (backflow, tf, steps, dt) in INLET.items():
        m, case, U0 = cases.channel_inlet((40, 10, 1), backflow=backflow)
        R = ref.RefMesh((40, 10, 1), hi=(4.0, 1.0, 0.1), two_d=True)
        U, p, phi, hist = R.flow_run(tf(case), steps, dt=dt, U=U0, reproducible=True)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
    m, case, U0 = cases.freestream_box()
    R = ref.RefMesh((32, 16, 1), hi=(2.0, 1.0, 0.1), two_d=True)
    U, p, phi, hist = R.flow_run(case, 4, dt=0.02, U=U0, reproducible=True)
    out.update(freestream_U=U, freestream_p=p, freestream_phi=phi, freestream_hist=hist)
    m, case, U0 = cases.channel_gradient()
    R = ref.RefMesh((40, 10, 1), hi=(4.0, 1.0, 0.1), two_d=True)
    U, p, phi, hist = R.flow_run(case, 6, U=U0, reproducible=True)
    out.update(gradient_U=U, gradient_p=p, gradient_phi=phi, gradient_hist=hist)
    m, case, U0 = cases.channel_flux_pressure()
    R = ref.RefMesh((40, 10, 1), hi=(4.0, 1.0, 0.1), two_d=True)
    U, p, phi, hist = R.flow_run(case, 6, U=U0, reproducible=True)
    out.update(fluxp_U=U, fluxp_p=p, fluxp_phi=phi, fluxp_hist=hist)
    m, case, U0 = cases.channel_flux_pressure(patch="xMax")
    U, p, phi, hist = R.flow_run(case, 6, U=U0, reproducible=True)
    out.update(fluxpo_U=U, fluxpo_p=p, fluxpo_phi=phi, fluxpo_hist=hist)
    m, case, U0 = cases.channel_total_pressure()
    U, p, phi, hist = R.flow_run(case, 8, U=U0, reproducible=True)
    out.update(totalp_U=U, totalp_p=p, totalp_phi=phi, totalp_hist=hist)
    for tag, kw, tf, steps, dt in (("robin", {}, dict, 6, 1.0), ("robin_walls", {"wall_ab": (2.0, 0.05)}, dict, 6, 1.0),
                                   ("robin_gradient", {"u_ab": (0.0, 1.0), "u_c": (0.02, 0.0, 0.0),
                                                       "p_ab": (0.0, 1.0), "p_c": 0.3}, dict, 6, 1.0),
                                   ("robin_transient", {}, transient, 3, 0.02)):
        m, case, U0 = cases.channel_robin(**kw)
        U, p, phi, hist = R.flow_run(tf(case), steps, dt=dt, U=U0, reproducible=True)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
    for tag, steps, dt in ADVECTIVE:
        m, case, U0 = advective_case(tag)
        U, p, phi, hist = R.flow_run(case, steps, dt=dt, U=U0, reproducible=True)
        out.update({f"{tag}_U": U, f"{tag}_p": p, f"{tag}_phi": phi, f"{tag}_hist": hist})
    np.savez_compressed(os.path.join(HERE, "flow_bc_cases.npz"), **out)
    print(sorted(out))


if __name__ == "__main__":
    main()
