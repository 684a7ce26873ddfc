"""Restart snapshots (vlm_flow_write_restart / vlm_flow_read_restart) against the reference's own
restart::write / restart::read (io/Restart.cpp), fixtures from tests/golden/make_restart_golden.py:

* the device flow, run as the reference ran before writing, writes the same directory byte for byte
  (binary arrays and state.txt);
* continuing from the reference's directory, the device flow reproduces the reference's continuation
  bit for bit;
* write -> read -> continue equals the uninterrupted run; a directory of another mesh is refused.
All in CFD_REPRODUCIBLE mode: the graded LES channel with mean-velocity forcing (transient, two old
time levels, nu_t), the steady lid cavity, and the channel with an advective outlet (whose
condition restarts without its history, as the reference's markRestarted gives it)."""
import os

import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")
CHAN = (8, 12, 6)


@pytest.fixture(scope="module")
def gold():
    z = np.load(os.path.join(HERE, "flow_restart_cases.npz"))
    return {k: z[k] for k in z.files}


def channel_flow():
    m, case, model, U0, dt = cases.channel(CHAN, les=True, van_driest=False)
    case["reproducible"] = True
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_model(model)
    fl.set_state(U0, None)
    return fl, dt


def cavity_flow():
    m, case = cases.lid_cavity(16, 100.0)
    case["reproducible"] = True
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_state(None, None)
    return fl, 1.0


def advective_flow():
    m, case, U0 = cases.channel_advective(ddt_scheme=2)
    case["reproducible"] = True
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_state(U0, None)
    return fl, 0.02


FLOWS = {"chan": (channel_flow, 3), "cav": (cavity_flow, 4), "adv": (advective_flow, 3)}


def same_files(a, b):
    names = sorted(os.listdir(b))
    assert sorted(os.listdir(a)) == names
    for n in names:
        with open(os.path.join(a, n), "rb") as fa, open(os.path.join(b, n), "rb") as fb:
            assert fa.read() == fb.read(), n


@pytest.mark.parametrize("case", ["chan", "cav", "adv"])
def test_write_matches_reference_bytes(tmp_path, case):
    make, steps = FLOWS[case]
    fl, dt = make()
    for _ in range(steps):
        fl.step(dt)
    fl.write_restart(tmp_path / "r")
    fl.close()
    same_files(tmp_path / "r", os.path.join(HERE, f"restart_{case}"))


@pytest.mark.parametrize("case", ["chan", "cav", "adv"])
def test_continue_from_reference_restart(gold, case):
    make, _ = FLOWS[case]
    fl, dt = make()
    assert fl.read_restart(os.path.join(HERE, f"restart_{case}"))
    for _ in range(2):
        fl.step(dt)
    U, p, phi = fl.state()
    nut, gp = fl.model_state()
    fl.close()
    assert np.array_equal(U, gold[f"{case}_U"])
    assert np.array_equal(p, gold[f"{case}_p"])
    assert np.array_equal(phi, gold[f"{case}_phi"])
    if case == "chan":
        assert gp == float(gold["chan_gradP"])
        assert np.array_equal(nut, gold["chan_nut"])


def test_round_trip_equals_uninterrupted_run(tmp_path):
    fl, dt = channel_flow()
    for _ in range(5):
        fl.step(dt)
    ref = fl.state()
    fl.close()
    fl, dt = channel_flow()
    for _ in range(3):
        fl.step(dt)
    fl.write_restart(tmp_path / "r")
    fl.close()
    fl, dt = channel_flow()
    assert fl.read_restart(tmp_path / "r")
    for _ in range(2):
        fl.step(dt)
    got = fl.state()
    fl.close()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_missing_and_mismatched_restart(tmp_path):
    fl, _ = cavity_flow()
    assert not fl.read_restart(tmp_path / "nothing")
    with pytest.raises(vb.VlmError) as e:
        fl.read_restart(os.path.join(HERE, "restart_chan"))
    assert e.value.name == "BAD_ARG"
    fl.close()
