"""Generates the restart fixtures from the reference itself (restart::write / restart::read of
io/Restart.cpp around IncompressibleFlow::step, compiled into oracle/_ref/libvlmref.so and driven by
oracle/ref_flow.cpp), in CFD_REPRODUCIBLE mode:

  tests/golden/restart_chan/   the 8 x 12 x 6 graded channel (Smagorinsky LES, mean-velocity forcing,
                               PIMPLE backward) after 3 steps: U, U_0, U_00, p, phi, phi_0, phi_00, nut,
                               state.txt
  tests/golden/restart_cav/    the 16 x 16 lid cavity (steady SIMPLE) after 4 steps: U, p, phi, state.txt
  tests/golden/restart_adv/    the 40 x 10 channel with an advective U outlet (PISO backward, dt 0.02)
                               after 3 steps: U, U_0, U_00, p, phi, phi_0, phi_00, state.txt (the
                               outlet condition's own history is not part of a restart)
  tests/golden/flow_restart_cases.npz   U, p, phi (and gradP) of the reference continuing 2 steps from
                               each directory

Run where the reference sources are present:
    make -C oracle REF=<reference tree> && python tests/golden/make_restart_golden.py
"""
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import cases  # noqa: E402

CHAN = (8, 12, 6)


def main():
    out = {}
    # channel: LES without damping (bit-exact on the device) + mean-velocity forcing
    beta = cases.channel_beta(CHAN[1], 1.0 / 395.0)
    R = ref.RefMesh(CHAN, hi=(2 * np.pi, 2.0, np.pi), periodic=(1, 0, 1), beta=(0, beta, 0),
                    patch_types=[0, 0, 1, 1, 0, 0])
    m, case, model, U0, dt = cases.channel(CHAN, les=True, van_driest=False)
    d = os.path.join(HERE, "restart_chan")
    shutil.rmtree(d, ignore_errors=True)
    R.flow_run(case, 3, dt=dt, U=U0, reproducible=True, model=model, write_restart=d)
    U, p, phi, _, nut, gp = R.flow_run(case, 2, dt=dt, U=U0, reproducible=True, model=model, read_restart=d)
    out.update(chan_U=U, chan_p=p, chan_phi=phi, chan_nut=nut, chan_gradP=np.array(gp))
    # cavity: steady SIMPLE, no old time levels
    m, case = cases.lid_cavity(16, 100.0)
    R = ref.RefMesh((16, 16, 1), hi=(1.0, 1.0, 0.1), two_d=True)
    d = os.path.join(HERE, "restart_cav")
    shutil.rmtree(d, ignore_errors=True)
    R.flow_run(case, 4, reproducible=True, write_restart=d)
    U, p, phi, _, _, _ = R.flow_run(case, 2, reproducible=True, read_restart=d)
    out.update(cav_U=U, cav_p=p, cav_phi=phi)
    # advective outlet: restart::read gives a fresh condition (markRestarted, IncompressibleFlow.cpp:41-47)
    m, case, U0 = cases.channel_advective(ddt_scheme=2)
    R = ref.RefMesh((40, 10, 1), hi=(4.0, 1.0, 0.1), two_d=True)
    d = os.path.join(HERE, "restart_adv")
    shutil.rmtree(d, ignore_errors=True)
    R.flow_run(case, 3, dt=0.02, U=U0, reproducible=True, write_restart=d)
    U, p, phi, _, _, _ = R.flow_run(case, 2, dt=0.02, U=U0, reproducible=True, read_restart=d)
    out.update(adv_U=U, adv_p=p, adv_phi=phi)
    np.savez_compressed(os.path.join(HERE, "flow_restart_cases.npz"), **out)
    for name in ("restart_chan", "restart_cav", "restart_adv"):
        print(name, sorted(os.listdir(os.path.join(HERE, name))))


if __name__ == "__main__":
    main()
