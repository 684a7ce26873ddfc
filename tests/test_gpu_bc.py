"""Symmetry (slip) planes for U and p in the device incompressible step (SymmetryBC,
BoundaryCondition.h:194-205, VolField.h:156-191: u_b = u - (n.u) n, per-component implicit normal part,
fixesFlux) against the reference's own IncompressibleFlow::step in CFD_REPRODUCIBLE mode (fixtures
tests/golden/flow_bc_cases.npz, made by make_bc_golden.py): fields and residual histories bit for bit,
on sheared meshes whose slip walls lean (normals off the axes)."""
import os

import numpy as np
import pytest

import voluma_b200 as vb
from voluma_b200 import cases

GOLD = os.path.join(os.path.dirname(__file__), "golden", "flow_bc_cases.npz")


def transient(case):
    return dict(case, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0)


CASES = {
    "slip2d": ((16, 16, 1), 0.3, dict, 6, 1.0),
    "slip2d_flat": ((16, 16, 1), 0.0, dict, 4, 1.0),
    "slip3d": ((8, 8, 6), 0.3, transient, 3, 0.05),
}


@pytest.fixture(scope="module")
def gold():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


def slip_faces(m):
    names = list(m["patch_names"])
    idx = []
    for q, nm in enumerate(names):
        if nm in ("xMin", "xMax", "zMin", "zMax"):
            s = int(m["patch_start"][q])
            idx.extend(range(s, s + int(m["patch_size"][q])))
    return np.array(idx, np.int64)


def test_golden_slip_walls_carry_no_flux(gold):
    # the reference's own fields: the flux through every slip face is zero to rounding
    for tag, (n, shear, _, _, _) in CASES.items():
        m, _, _ = cases.slip_cavity(n, shear)
        phi = gold[f"{tag}_phi"]
        f = slip_faces(m)
        assert f.size > 0
        assert np.abs(phi[f]).max() < 1e-15 * max(1.0, np.abs(phi).max())


def test_slip_case_types():
    m, case, pts = cases.slip_cavity((8, 8, 6), 0.3)
    assert not m["skewed"]
    names = list(m["patch_names"])
    assert [int(case["u_type"][names.index(k)]) for k in ("xMin", "zMax", "yMin", "yMax")] == [2, 2, 1, 1]
    assert [int(case["p_type"][names.index(k)]) for k in ("xMax", "zMin", "yMin")] == [2, 2, 0]


@pytest.mark.gpu
@pytest.mark.parametrize("tag", sorted(CASES))
def test_slip_cavity_bitwise(gold, tag):
    n, shear, tf, steps, dt = CASES[tag]
    m, case, _ = cases.slip_cavity(n, shear)
    case = dict(tf(case), reproducible=True)
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_state(None, None)
    hist = []
    for _ in range(steps):
        i = fl.step(dt)
        hist.append([i["UInitialResidual"], i["pInitialResidual"], i["continuityError"]])
    U, p, phi = fl.state()
    fl.close()
    assert np.array_equal(np.array(hist), gold[f"{tag}_hist"][:, :3])
    assert np.array_equal(U, gold[f"{tag}_U"])
    assert np.array_equal(p, gold[f"{tag}_p"])
    assert np.array_equal(phi, gold[f"{tag}_phi"])


@pytest.mark.gpu
def test_slip_cavity_default_mode_close(gold):
    # default (fast) mode against the reference's default mode: the device's parallel DILU and GAMG
    # smoothers change the iterates within the solver tolerances (U relTol 0.1, p relTol 0.05 per
    # outer iteration; measured 1.1e-3 of max |U| after 6 iterations)
    n, shear, tf, steps, dt = CASES["slip2d"]
    m, case, _ = cases.slip_cavity(n, shear)
    fl = vb.Flow(vb.Mesh.from_arrays(m), case)
    fl.set_state(None, None)
    for _ in range(steps):
        fl.step(dt)
    U, p, phi = fl.state()
    fl.close()
    ref = gold["slip2d_default_U"]
    assert np.abs(U - ref).max() < 5e-3 * np.abs(ref).max()
    assert np.abs(phi[slip_faces(m)]).max() < 1e-15


INLET = {
    "inlet": (0.0, dict, 6, 1.0),
    "inlet_backflow": (0.5, dict, 6, 1.0),
    "inlet_transient": (0.5, lambda c: dict(c, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0), 3,
                        0.02),
}


def test_inlet_case_layout():
    m, case, U0 = cases.channel_inlet((40, 10, 1), backflow=0.5)
    names = list(m["patch_names"])
    assert int(case["u_type"][names.index("xMax")]) == 3 and int(case["p_type"][names.index("xMax")]) == 1
    nI = m["n_internal_faces"]
    q = names.index("xMin")
    f = np.arange(m["patch_start"][q], m["patch_start"][q] + m["patch_size"][q]) - nI
    assert case["u_face"][f, 0].min() > 0 and np.abs(case["u_face"][f, 1:]).max() == 0
    assert (U0[:, 0] < 0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("tag", sorted(INLET))
def test_inlet_outlet_channel_bitwise(gold, tag):
    # fixedValue inlet given face by face (vlm_flow_set_boundary_values) and an inletOutlet outlet whose
    # inflow faces (backflow) switch to the inlet value
    backflow, tf, steps, dt = INLET[tag]
    m, case, U0 = cases.channel_inlet((40, 10, 1), backflow=backflow)
    fl = vb.Flow(vb.Mesh.from_arrays(m), dict(tf(case), reproducible=True))
    fl.set_state(U0, None)
    hist = []
    for _ in range(steps):
        i = fl.step(dt)
        hist.append([i["UInitialResidual"], i["pInitialResidual"], i["continuityError"]])
    U, p, phi = fl.state()
    fl.close()
    assert np.array_equal(np.array(hist), gold[f"{tag}_hist"][:, :3])
    assert np.array_equal(U, gold[f"{tag}_U"])
    assert np.array_equal(p, gold[f"{tag}_p"])
    assert np.array_equal(phi, gold[f"{tag}_phi"])


@pytest.mark.gpu
def test_flow_rejects_unknown_boundary_types():
    m, case, _ = cases.channel_inlet((8, 4, 1))
    bad = dict(case, u_type=np.full(len(case["u_type"]), 7, np.int32))
    with pytest.raises(vb.VlmError):
        vb.Flow(vb.Mesh.from_arrays(m), bad)
    bad = dict(case, p_type=np.full(len(case["p_type"]), 3, np.int32))
    with pytest.raises(vb.VlmError):
        vb.Flow(vb.Mesh.from_arrays(m), bad)
    # freestreamPressure takes its direction from a freestream velocity on the same patch
    bad = dict(case, p_type=np.full(len(case["p_type"]), 4, np.int32))
    with pytest.raises(vb.VlmError):
        vb.Flow(vb.Mesh.from_arrays(m), bad)


def run_case(m, case, U0, steps, dt):
    fl = vb.Flow(vb.Mesh.from_arrays(m), dict(case, reproducible=True))
    fl.set_state(U0, None)
    hist = []
    for _ in range(steps):
        i = fl.step(dt)
        hist.append([i["UInitialResidual"], i["pInitialResidual"], i["continuityError"]])
    U, p, phi = fl.state()
    fl.close()
    return U, p, phi, np.array(hist)


@pytest.mark.gpu
def test_freestream_box_bitwise(gold):
    # freestream U / freestreamPressure p on every side, fractional value fractions on the oblique sides
    m, case, U0 = cases.freestream_box()
    U, p, phi, hist = run_case(m, case, U0, 4, 0.02)
    assert np.array_equal(hist, gold["freestream_hist"][:, :3])
    for k, v in (("U", U), ("p", p), ("phi", phi)):
        assert np.array_equal(v, gold[f"freestream_{k}"]), k


@pytest.mark.gpu
@pytest.mark.parametrize("patch,tag", [("xMin", "fluxp"), ("xMax", "fluxpo")])
def test_fixed_flux_pressure_channel_bitwise(gold, patch, tag):
    m, case, U0 = cases.channel_flux_pressure(patch=patch)
    U, p, phi, hist = run_case(m, case, U0, 6, 1.0)
    assert np.array_equal(hist, gold[f"{tag}_hist"][:, :3])
    for k, v in (("U", U), ("p", p), ("phi", phi)):
        assert np.array_equal(v, gold[f"{tag}_{k}"]), k


def test_golden_outlet_flux_pressure_differs():
    z = np.load(GOLD)
    assert not np.array_equal(z["fluxpo_p"], z["inlet_p"])


@pytest.mark.gpu
def test_total_pressure_inlet_bitwise(gold):
    # totalPressure p (values from the inflow faces' velocity at each step start) with a
    # pressureInletOutletVelocity inlet, slip walls and an inletOutlet outlet
    m, case, U0 = cases.channel_total_pressure()
    U, p, phi, hist = run_case(m, case, U0, 8, 1.0)
    assert np.array_equal(hist, gold["totalp_hist"][:, :3])
    for k, v in (("U", U), ("p", p), ("phi", phi)):
        assert np.array_equal(v, gold[f"totalp_{k}"]), k


@pytest.mark.gpu
def test_fixed_gradient_channel_bitwise(gold):
    m, case, U0 = cases.channel_gradient()
    U, p, phi, hist = run_case(m, case, U0, 6, 1.0)
    assert np.array_equal(hist, gold["gradient_hist"][:, :3])
    for k, v in (("U", U), ("p", p), ("phi", phi)):
        assert np.array_equal(v, gold[f"gradient_{k}"]), k


@pytest.mark.gpu
@pytest.mark.parametrize("tag,kw,transient,steps,dt", [
    ("robin", {}, False, 6, 1.0),
    ("robin_walls", {"wall_ab": (2.0, 0.05)}, False, 6, 1.0),
    ("robin_gradient", {"u_ab": (0.0, 1.0), "u_c": (0.02, 0.0, 0.0), "p_ab": (0.0, 1.0), "p_c": 0.3}, False, 6, 1.0),
    ("robin_transient", {}, True, 3, 0.02),
])
def test_robin_channel_bitwise(gold, tag, kw, transient, steps, dt):
    """Robin a phi + b dphi/dn = c (RobinBC, BoundaryCondition.h:166-192) for U and p at the channel
    outlet, on the walls as a partial-slip U condition, and as a pure-gradient condition (a = 0, which
    then fixes neither the value nor the flux): the reference's fields and residual history bit for
    bit in reproducible mode."""
    m, case, U0 = cases.channel_robin(**kw)
    if transient:
        case = dict(case, steady=False, ddt_scheme=1, n_corr=2, alpha_u=1.0, alpha_p=1.0)
    U, p, phi, hist = run_case(m, case, U0, steps, dt)
    assert np.array_equal(hist, gold[f"{tag}_hist"][:, :3])
    for k, v in (("U", U), ("p", p), ("phi", phi)):
        assert np.array_equal(v, gold[f"{tag}_{k}"]), k


@pytest.mark.gpu
def test_robin_needs_its_coefficients():
    m, case, U0 = cases.channel_robin()
    mesh = vb.Mesh.from_arrays(m)
    for bad in (dict(case, u_robin=None), dict(case, p_robin=None),
                dict(case, u_robin=np.zeros_like(case["u_robin"]))):
        with pytest.raises(vb.VlmError) as e:
            vb.Flow(mesh, bad)
        assert e.value.name == "BAD_ARG"


# tag, steps, dt, channel_advective arguments, steady (the cases of flow_bc_cases.npz)
ADVECTIVE = [
    ("adv_euler", 4, 0.02, dict(ddt_scheme=1), False),
    ("adv_backward", 5, 0.02, dict(ddt_scheme=2), False),
    ("adv_far", 5, 0.02, dict(ddt_scheme=2, far_field=(0.5, (0.8, 0.05, 0.0))), False),
    ("adv_steady", 3, 1.0, dict(ddt_scheme=0), True),
]


@pytest.mark.gpu
@pytest.mark.parametrize("tag,steps,dt,kw,steady", ADVECTIVE)
def test_advective_outlet_bitwise(gold, tag, steps, dt, kw, steady):
    """Advective U outlet (AdvectiveBC, BoundaryCondition.h:389-414; VolField.h:235-264): the
    condition's own boundary history, shifted at each new time index, Euler and backward
    coefficients (backward from the third level on), the far-field relaxation, and the steady zero
    gradient; the later steps replay the captured step graph.  The reference's fields and residual
    history bit for bit."""
    m, case, U0 = cases.channel_advective(**kw)
    if steady:
        case = dict(case, steady=True, n_corr=1, alpha_u=0.7, alpha_p=0.3)
    U, p, phi, hist = run_case(m, case, U0, steps, dt)
    assert np.array_equal(hist, gold[f"{tag}_hist"][:, :3])
    for k, v in (("U", U), ("p", p), ("phi", phi)):
        assert np.array_equal(v, gold[f"{tag}_{k}"]), k


def test_golden_advective_cases_differ():
    # the far field and the time scheme change the outlet's fields
    z = np.load(GOLD)
    assert not np.array_equal(z["adv_far_U"], z["adv_backward_U"])
    assert not np.array_equal(z["adv_euler_U"], z["inlet_transient_U"])
    names_ok = [k for k in z.files if k.startswith("adv_")]
    assert len(names_ok) == 16


@pytest.mark.gpu
def test_advective_far_field_checked():
    m, case, U0 = cases.channel_advective(far_field=(-1.0, (1.0, 0.0, 0.0)))
    with pytest.raises(vb.VlmError) as e:
        vb.Flow(vb.Mesh.from_arrays(m), case)
    assert e.value.name == "BAD_ARG"
