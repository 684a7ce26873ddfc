"""Synthetic workloads of the pressure-equation path (host side, numpy).

* tgv_pressure_system(n): the 3D Taylor-Green pressure equation on the periodic [0,2pi]^3 box
  with an n^3 uniform mesh, as the PIMPLE corrector assembles it (laplacian(rAUf = dt) minus the
  divergence of a predicted flux, setReference(0)).
* poisson_batch(...): uneven batch of pressure Poisson systems on graded, jittered unit boxes
  (Neumann walls + one reference cell; right-hand side = divergence of a random Fourier velocity
  field with |k| <= 4 and N(0,1)/|k|^2 amplitudes), as projectDivergenceFree solves them.
"""
from __future__ import annotations

import math

import numpy as np

from . import mesh as vm

DT = 2e-3


def fourier_velocity(X, seed, n_modes=16, kmax=4):
    """Sum of n_modes random Fourier modes (|k| <= kmax, amplitude N(0,1)/|k|^2) at points X."""
    rng = np.random.default_rng(seed)
    u = np.zeros((len(X), 3))
    for _ in range(n_modes):
        while True:
            k = rng.integers(-kmax, kmax + 1, size=3)
            if k.any() and (k * k).sum() <= kmax * kmax:
                break
        kk = float(np.sqrt((k * k).sum()))
        a = rng.standard_normal(3) / kk ** 2
        ph = rng.uniform(0, 2 * np.pi)
        u += np.outer(np.cos(2 * np.pi * (X @ k) + ph), a)
    return u


def face_flux(m, u_face):
    Sf = m["Sf"]
    return u_face[:, 0] * Sf[:, 0] + u_face[:, 1] * Sf[:, 1] + u_face[:, 2] * Sf[:, 2]


def div_per_volume(m, F):
    """fvc::div (Fvc.h:294-304) restated for input preparation."""
    nI = m["n_internal_faces"]
    r = np.zeros(m["n_cells"])
    np.add.at(r, np.stack([m["owner"][:nI], m["neighbour"]], 1).ravel(), np.stack([F[:nI], -F[:nI]], 1).ravel())
    np.add.at(r, m["owner"][nI:], F[nI:])
    return r / m["V"]


def tgv_velocity(C, seed=1234, n_modes=16, amp=0.1):
    x, y, z = C[:, 0], C[:, 1], C[:, 2]
    u = np.stack([np.sin(x) * np.cos(y) * np.cos(z), -np.cos(x) * np.sin(y) * np.cos(z), np.zeros_like(x)], 1)
    rng = np.random.default_rng(seed)
    for _ in range(n_modes):
        k = rng.integers(-4, 5, size=3)
        if not k.any():
            k[0] = 1
        kk = float(np.sqrt((k * k).sum()))
        a = rng.standard_normal(3) / kk ** 2
        ph = rng.uniform(0, 2 * np.pi)
        u += amp * np.outer(np.cos(C @ k + ph), a)
    return u


def tgv_pressure_system(n=128, m=None):
    """(mesh, diag, upper, b) of the TGV pressure equation on an n^3 periodic box."""
    m = m or vm.box_mesh((n, n, n), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    nC, nI = m["n_cells"], m["n_internal_faces"]
    own, nei = m["owner"][:nI], m["neighbour"]
    upper = DT * m["magSf"][:nI] * m["ndc"][:nI]
    diag = np.zeros(nC)
    np.subtract.at(diag, np.stack([own, nei], 1).ravel(), np.repeat(upper, 2))
    u = tgv_velocity(m["C"])
    w = m["w"][:nI, None]
    uf = w * u[own] + (1.0 - w) * u[nei]
    Sf = m["Sf"][:nI]
    phi = uf[:, 0] * Sf[:, 0] + uf[:, 1] * Sf[:, 1] + uf[:, 2] * Sf[:, 2]
    div = np.zeros(nC)
    np.add.at(div, np.stack([own, nei], 1).ravel(), np.stack([phi, -phi], 1).ravel())
    b = (div / m["V"]) * m["V"]
    diag[0] += diag[0]
    return m, diag, upper, b


def graded_jittered_box(n, ratio, jitter, seed):
    """Unit box n^3 with tanh grading (centre/wall cell-size ratio `ratio`, beta = acosh(sqrt(ratio)))
    in every direction and interior vertices jittered by U(+-jitter*h)."""
    beta = math.acosh(math.sqrt(ratio)) if ratio > 1.0 + 1e-12 else 0.0
    pts = vm.box_points((n, n, n), beta=(beta, beta, beta))
    if jitter > 0:
        pts = vm.jitter_interior(pts, (n, n, n), jitter, seed)
    return vm.box_mesh((n, n, n), points=pts)


def poisson_batch_params(n_systems=256, n_min=16, n_max=96, seed=20261203, jitter=0.2, ratio_max=8.0):
    """The seeded draws of poisson_batch, one dict per system (n, ratio, jitter, mesh seed, field seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_systems):
        n = int(rng.integers(n_min, n_max + 1))
        ratio = float(rng.uniform(1.0, ratio_max))
        mesh_seed = int(rng.integers(1 << 30))
        field_seed = int(rng.integers(1 << 30))
        out.append(dict(n=n, ratio=ratio, jitter=jitter, mesh_seed=mesh_seed, field_seed=field_seed))
    return out


def poisson_system(q):
    """(mesh, div_phi) of one poisson_batch_params entry."""
    m = graded_jittered_box(q["n"], q["ratio"], q["jitter"], q["mesh_seed"])
    u_f = fourier_velocity(m["Cf"], q["field_seed"])
    return m, div_per_volume(m, face_flux(m, u_f))


def poisson_batch(n_systems=256, n_min=16, n_max=96, seed=20261203, jitter=0.2, ratio_max=8.0):
    """List of (mesh, div_phi) pairs: the pressure Poisson systems of projectDivergenceFree on
    graded, jittered boxes of uneven sizes."""
    return [poisson_system(q) for q in poisson_batch_params(n_systems, n_min, n_max, seed, jitter, ratio_max)]


def batch_face_array(meshes, per_mesh):
    """Concatenates per-mesh face arrays into the batch layout: every mesh's internal faces, then
    every mesh's boundary faces."""
    ints = [a[: m["n_internal_faces"]] for m, a in zip(meshes, per_mesh)]
    bnds = [a[m["n_internal_faces"]:] for m, a in zip(meshes, per_mesh)]
    return np.concatenate(ints + bnds)


def split_batch_faces(meshes, F):
    nI = [m["n_internal_faces"] for m in meshes]
    nB = [m["n_faces"] - m["n_internal_faces"] for m in meshes]
    ib = np.cumsum([0] + nI)
    bb = sum(nI) + np.cumsum([0] + nB)
    return [np.concatenate([F[ib[i]:ib[i + 1]], F[bb[i]:bb[i + 1]]]) for i in range(len(meshes))]


# ------------------------------------------------------------------ incompressible cases
def _ctl(solver, precond, tol, rel_tol, max_iter):
    return dict(solver=solver, preconditioner=precond, tolerance=tol, relTol=rel_tol, maxIter=max_iter, minIter=0,
                nSweeps=1)


def lid_cavity(n=64, Re=100.0, lid=1.0):
    """The lid-driven cavity of cases/cavity/case.json: generateBox n = (n, n, 1), hi = (1, 1, 0.1), twoD,
    walls on xMin/xMax/yMin/yMax with yMax the moving lid, nu = lid/Re; steady SIMPLE with the fvmFlow
    steady defaults (fvmFlow.cpp:141-178: linearUpwind, alphaU 0.7, alphaP 0.3, nCorr 1,
    U {PBiCGStab, DILU, 1e-10, relTol 0.1}, p {PCG, GAMG, 1e-10, relTol 0.05}).
    Returns (mesh dict, case dict); the case's boundary arrays follow the mesh's patch order."""
    from . import mesh as vm
    m = vm.box_mesh((n, n, 1), hi=(1.0, 1.0, 0.1), two_d=True)
    nP = len(m["patch_start"])
    u_type = np.ones(nP, np.int32)               # noSlip / fixedValue everywhere
    u_value = np.zeros((nP, 3))
    cf_y = [m["Cf"][m["patch_start"][q]:m["patch_start"][q] + m["patch_size"][q], 1] for q in range(nP)]
    lid_patch = int(np.argmax([c.mean() for c in cf_y]))
    u_value[lid_patch] = (lid, 0.0, 0.0)
    case = dict(nu=lid / Re, steady=True, div_scheme=2, ddt_scheme=0, n_outer=1, n_corr=1, n_non_orth_corr=0,
                momentum_predictor=True, alpha_u=0.7, alpha_p=0.3, u_type=u_type, u_value=u_value.ravel(),
                p_type=np.zeros(nP, np.int32), p_value=np.zeros(nP), U=_ctl("PBiCGStab", "DILU", 1e-10, 0.1, 1000),
                p=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000), pFinal=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000),
                p_ref_cell=0, p_ref_value=0.0, lid_patch=lid_patch)
    return m, case


def slip_cavity(n=(16, 16, 1), shear=0.3, Re=100.0, lid=1.0):
    """A lid-driven cavity with slip side walls: the unit box (0.1 deep when nz = 1, two-dimensional)
    sheared by x += shear * y, so that every cell is a parallelogram (non-orthogonal, not skewed) and
    the xMin / xMax walls lean; those walls and, in 3D, zMin / zMax are symmetry planes for U and p
    (SymmetryBC, BoundaryCondition.h:194-205); yMin is a no-slip wall and yMax the lid moving at
    (lid, 0, 0); nu = lid / Re.  Steady SIMPLE with the lid-cavity settings and one non-orthogonal
    corrector.  Returns (mesh, case, points); `points` is the vertex array in generateBox order."""
    from . import mesh as vm
    nx, ny, nz = (int(v) for v in n)
    two_d = nz == 1
    hi = (1.0, 1.0, 0.1 if two_d else 1.0)
    pts = vm.box_points((nx, ny, nz), hi=hi)
    pts[:, 0] += shear * pts[:, 1]
    m = vm.box_mesh((nx, ny, nz), points=pts, two_d=two_d)
    names = list(m["patch_names"])
    nP = len(names)
    slip = ("xMin", "xMax", "zMin", "zMax")
    u_type = np.array([2 if nm in slip else 1 for nm in names], np.int32)
    p_type = np.array([2 if nm in slip else 0 for nm in names], np.int32)
    u_value = np.zeros((nP, 3))
    u_value[names.index("yMax")] = (lid, 0.0, 0.0)
    case = dict(nu=lid / Re, steady=True, div_scheme=2, ddt_scheme=0, n_outer=1, n_corr=1, n_non_orth_corr=1,
                momentum_predictor=True, alpha_u=0.7, alpha_p=0.3, u_type=u_type, u_value=u_value.ravel(),
                p_type=p_type, p_value=np.zeros(nP), U=_ctl("PBiCGStab", "DILU", 1e-10, 0.1, 1000),
                p=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000), pFinal=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000),
                p_ref_cell=0, p_ref_value=0.0)
    return m, case, pts


def skewed_cavity(n=(16, 16, 1), jitter=0.2, seed=20261203, Re=100.0, lid=1.0):
    """The lid-driven cavity on a jittered box: interior vertices moved by U(+-jitter h) (boundary
    vertices stay), so that the mesh is non-orthogonal and skewed (Mesh::skewed: the linear
    interpolation point of a face is off its centre) and the step takes the reference's skew
    corrections.  The unit box is 0.1 deep and two-dimensional when nz = 1; no-slip walls, the yMax
    lid at (lid, 0, 0), nu = lid / Re; the lid-cavity SIMPLE settings with one non-orthogonal
    corrector.  Returns (mesh, case, points); `points` is the vertex array in generateBox order."""
    from . import mesh as vm
    nx, ny, nz = (int(v) for v in n)
    two_d = nz == 1
    hi = (1.0, 1.0, 0.1 if two_d else 1.0)
    pts = vm.jitter_interior(vm.box_points((nx, ny, nz), hi=hi), (nx, ny, nz), jitter, seed)
    m = vm.box_mesh((nx, ny, nz), points=pts, two_d=two_d)
    names = list(m["patch_names"])
    nP = len(names)
    u_value = np.zeros((nP, 3))
    u_value[names.index("yMax")] = (lid, 0.0, 0.0)
    case = dict(nu=lid / Re, steady=True, div_scheme=2, ddt_scheme=0, n_outer=1, n_corr=1, n_non_orth_corr=1,
                momentum_predictor=True, alpha_u=0.7, alpha_p=0.3, u_type=np.ones(nP, np.int32),
                u_value=u_value.ravel(), p_type=np.zeros(nP, np.int32), p_value=np.zeros(nP),
                U=_ctl("PBiCGStab", "DILU", 1e-10, 0.1, 1000), p=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000),
                pFinal=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000), p_ref_cell=0, p_ref_value=0.0)
    return m, case, pts


def channel_inlet(n=(80, 20, 1), ubulk=1.0, nu=0.05, backflow=0.0):
    """The plane channel with an inlet and an outlet of the reference's cases/channelInlet/parabolic.json:
    the 2D box 4 x 1 (0.1 deep), walls yMin / yMax (no slip), the xMin inlet with the parabolic profile
    u = 1.5 ubulk (1 - s^2), s = (y - 0.5) / 0.5, given face by face (u_face) and zeroGradient p, the
    xMax outlet with inletOutlet U (inlet value 0) and fixedValue p = 0; nu 0.05 (Re_h = 20), steady
    SIMPLE with linear divergence.  Initial field U = (ubulk, 0, 0); backflow > 0 reverses the upper
    half of the last tenth of the channel to -backflow, so that the outlet starts with inflow faces.
    Returns (mesh, case, U0)."""
    from . import mesh as vm
    nx, ny, nz = (int(v) for v in n)
    m = vm.box_mesh((nx, ny, nz), hi=(4.0, 1.0, 0.1), two_d=True)
    names = list(m["patch_names"])
    nP = len(names)
    u_type = np.array([{"xMin": 1, "xMax": 3}.get(nm, 1) for nm in names], np.int32)
    p_type = np.array([1 if nm == "xMax" else 0 for nm in names], np.int32)
    nI = m["n_internal_faces"]
    nB = m["n_faces"] - nI
    u_face = np.zeros((nB, 3))
    q = names.index("xMin")
    f = np.arange(m["patch_start"][q], m["patch_start"][q] + m["patch_size"][q])
    s = (m["Cf"][f, 1] - 0.5) / 0.5
    u_face[f - nI, 0] = 1.5 * ubulk * np.maximum(1.0 - s * s, 0.0)
    case = dict(nu=nu, steady=True, div_scheme=1, ddt_scheme=0, n_outer=1, n_corr=1, n_non_orth_corr=0,
                momentum_predictor=True, alpha_u=0.7, alpha_p=0.3, u_type=u_type, u_value=np.zeros(3 * nP),
                p_type=p_type, p_value=np.zeros(nP), u_face=u_face,
                U=_ctl("PBiCGStab", "DILU", 1e-10, 0.1, 1000), p=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000),
                pFinal=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000), p_ref_cell=0, p_ref_value=0.0)
    U0 = np.zeros((m["n_cells"], 3))
    U0[:, 0] = ubulk
    if backflow > 0:
        C = m["C"]
        U0[(C[:, 0] > 3.6) & (C[:, 1] > 0.5), 0] = -backflow
    return m, case, U0


def freestream_box(n=(32, 16, 1), uinf=(1.0, 0.2, 0.0), nu=0.01, vortex=0.5):
    """A vortex carried through a 2D box 2 x 1 (0.1 deep) whose four sides are free-stream boundaries:
    U freestream (FreestreamVelocityBC: inflow faces fixed at uinf, outflow faces zero gradient, with the
    value fraction 1/2 - (uinf.n)/(2|uinf|)) and p freestreamPressure at 0 (fraction 1/2 + (uinf.n) /
    (2|uinf|)); uinf oblique so that the side fractions are fractional.  Transient Euler PISO (nCorr 2),
    linear divergence.  Initial field: uinf plus a Gaussian vortex of peak speed ~vortex at (0.6, 0.5).
    Returns (mesh, case, U0)."""
    from . import mesh as vm
    nx, ny, nz = (int(v) for v in n)
    m = vm.box_mesh((nx, ny, nz), hi=(2.0, 1.0, 0.1), two_d=True)
    nP = len(m["patch_names"])
    u_value = np.tile(np.asarray(uinf, np.float64), nP)
    case = dict(nu=nu, steady=False, div_scheme=1, ddt_scheme=1, n_outer=1, n_corr=2, n_non_orth_corr=0,
                momentum_predictor=True, alpha_u=1.0, alpha_p=1.0, u_type=np.full(nP, 4, np.int32), u_value=u_value,
                p_type=np.full(nP, 4, np.int32), p_value=np.zeros(nP),
                U=_ctl("PBiCGStab", "DILU", 1e-10, 0.0, 1000), p=_ctl("PCG", "GAMG", 1e-10, 0.01, 2000),
                pFinal=_ctl("PCG", "GAMG", 1e-10, 0.0, 2000), p_ref_cell=0, p_ref_value=0.0)
    C = m["C"]
    dx, dy = C[:, 0] - 0.6, C[:, 1] - 0.5
    g = vortex * np.exp(-(dx * dx + dy * dy) / 0.02) / 0.14
    U0 = np.zeros((m["n_cells"], 3))
    U0[:, 0] = uinf[0] - g * dy
    U0[:, 1] = uinf[1] + g * dx
    return m, case, U0


def channel_gradient(n=(40, 10, 1), ubulk=1.0, nu=0.05, dpdn=0.6, dudn=(0.05, 0.0, 0.0)):
    """channel_inlet with fixedGradient conditions (FixedGradientBC): p at the inlet with the normal
    gradient dpdn (the Poiseuille pressure drop -dp/dx = 12 nu ubulk / h^2 = 0.6 seen along the outward
    normal -x) and U at the outlet with the normal gradient dudn.  Returns (mesh, case, U0)."""
    m, case, U0 = channel_inlet(n, ubulk, nu)
    names = list(m["patch_names"])
    qi, qo = names.index("xMin"), names.index("xMax")
    case = dict(case, u_type=case["u_type"].copy(), p_type=case["p_type"].copy(), u_value=case["u_value"].copy(),
                p_value=case["p_value"].copy())
    case["p_type"][qi] = 5
    case["p_value"][qi] = dpdn
    case["u_type"][qo] = 5
    case["u_value"][3 * qo:3 * qo + 3] = dudn
    return m, case, U0


def channel_robin(n=(40, 10, 1), ubulk=1.0, nu=0.05, u_ab=(1.0, 0.4), p_ab=(1.0, 0.25), u_c=(0.9, 0.0, 0.0),
                  p_c=0.05, wall_ab=None):
    """channel_inlet with Robin conditions a phi + b dphi/dn = c (RobinBC, BoundaryCondition.h:166-192):
    U at the outlet ({a, b} = u_ab, c = u_c) and p at the outlet (p_ab, c = p_c); wall_ab: also a Robin
    (partial-slip-like) U condition on the walls with c = 0.  Returns (mesh, case, U0)."""
    m, case, U0 = channel_inlet(n, ubulk, nu)
    names = list(m["patch_names"])
    nP = len(names)
    qo = names.index("xMax")
    case = dict(case, u_type=case["u_type"].copy(), p_type=case["p_type"].copy(), u_value=case["u_value"].copy(),
                p_value=case["p_value"].copy())
    ur = np.zeros(2 * nP)
    pr = np.zeros(2 * nP)
    case["u_type"][qo] = 8
    case["u_value"][3 * qo:3 * qo + 3] = u_c
    ur[2 * qo:2 * qo + 2] = u_ab
    case["p_type"][qo] = 8
    case["p_value"][qo] = p_c
    pr[2 * qo:2 * qo + 2] = p_ab
    if wall_ab is not None:
        for nm in ("yMin", "yMax"):
            q = names.index(nm)
            case["u_type"][q] = 8
            case["u_value"][3 * q:3 * q + 3] = 0.0
            ur[2 * q:2 * q + 2] = wall_ab
    case["u_robin"] = ur
    case["p_robin"] = pr
    return m, case, U0


def channel_advective(n=(40, 10, 1), ubulk=1.0, nu=0.05, ddt_scheme=2, far_field=None):
    """channel_inlet, transient (PISO, nCorr 2, ddt_scheme 1 Euler or 2 backward), with an advective
    U outlet (AdvectiveBC, BoundaryCondition.h:389-414; VolField.h:235-264) and p fixed at 0 there;
    far_field = (lInf, (Ux, Uy, Uz)) adds the relaxation towards that far-field velocity.  Returns
    (mesh, case, U0)."""
    m, case, U0 = channel_inlet(n, ubulk, nu)
    names = list(m["patch_names"])
    nP = len(names)
    qo = names.index("xMax")
    case = dict(case, u_type=case["u_type"].copy(), steady=False, ddt_scheme=ddt_scheme, n_corr=2, alpha_u=1.0,
                alpha_p=1.0)
    case["u_type"][qo] = 9
    if far_field is not None:
        adv = np.zeros(4 * nP)
        adv[4 * qo] = far_field[0]
        adv[4 * qo + 1:4 * qo + 4] = far_field[1]
        case["u_advective"] = adv
    return m, case, U0


def channel_flux_pressure(n=(40, 10, 1), ubulk=1.0, nu=0.05, patch="xMin"):
    """channel_inlet with fixedFluxPressure p on `patch` (FixedFluxPressureBC, whose gradient the
    corrector sets so that the boundary flux is the boundary velocity's).  On the inlet
    (cases/channelInlet/fixedFluxPressure.json) the fixed inlet velocity makes that gradient zero; on
    the outlet, where the velocity is inletOutlet, it is not (and p then needs the reference cell).
    Returns (mesh, case, U0)."""
    m, case, U0 = channel_inlet(n, ubulk, nu)
    q = list(m["patch_names"]).index(patch)
    case = dict(case, p_type=case["p_type"].copy())
    case["p_type"][q] = 6
    return m, case, U0


def channel_total_pressure(n=(40, 10, 1), p0=0.5, nu=0.01):
    """The total-pressure inlet of cases/channelInlet/totalPressure.json: the 2D box 4 x 1 (0.1 deep) with
    slip walls yMin / yMax, the xMin inlet with totalPressure p0 (TotalPressureBC: p0 - |U_b|^2/2 on inflow
    faces) and pressureInletOutletVelocity U, the xMax outlet with inletOutlet U and fixedValue p = 0;
    nu 0.01, steady SIMPLE with linearUpwind, alphaU 0.7, alphaP 0.3, from U = 0 (the exact solution is
    U = (1, 0, 0), p = 0).  Returns (mesh, case, U0)."""
    from . import mesh as vm
    nx, ny, nz = (int(v) for v in n)
    m = vm.box_mesh((nx, ny, nz), hi=(4.0, 1.0, 0.1), two_d=True)
    names = list(m["patch_names"])
    nP = len(names)
    u_type = np.array([{"xMin": 6, "xMax": 3}.get(nm, 2) for nm in names], np.int32)
    p_type = np.array([{"xMin": 7, "xMax": 1}.get(nm, 0) for nm in names], np.int32)
    p_value = np.array([p0 if nm == "xMin" else 0.0 for nm in names])
    case = dict(nu=nu, steady=True, div_scheme=2, ddt_scheme=0, n_outer=1, n_corr=1, n_non_orth_corr=0,
                momentum_predictor=True, alpha_u=0.7, alpha_p=0.3, u_type=u_type, u_value=np.zeros(3 * nP),
                p_type=p_type, p_value=p_value, U=_ctl("PBiCGStab", "DILU", 1e-10, 0.1, 1000),
                p=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000), pFinal=_ctl("PCG", "GAMG", 1e-10, 0.05, 2000),
                p_ref_cell=0, p_ref_value=0.0)
    return m, case, np.zeros((m["n_cells"], 3))


def taylor_green_flow(n=16, nu=1.0 / 1600, u0=1.0):
    """Taylor-Green vortex in the periodic box [0, 2pi]^3 (fvmFlow.cpp:76-89 initial condition
    U = u0 (sin x cos y cos z, -cos x sin y cos z, 0)); transient PIMPLE with the fvmFlow transient
    defaults: backward ddt, linear divergence, nOuter 1, nCorr 2, U {PBiCGStab, DILU, 1e-8},
    p {PCG, GAMG, 1e-8, relTol 0.01}, pFinal {PCG, GAMG, 1e-8}.  Returns (mesh, case, U0)."""
    from . import mesh as vm
    m = vm.box_mesh((n, n, n), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1))
    C = m["C"]
    U0 = u0 * np.stack([np.sin(C[:, 0]) * np.cos(C[:, 1]) * np.cos(C[:, 2]),
                        -np.cos(C[:, 0]) * np.sin(C[:, 1]) * np.cos(C[:, 2]), np.zeros(len(C))], 1)
    nP = max(len(m["patch_start"]), 1)
    case = dict(nu=nu, steady=False, div_scheme=1, ddt_scheme=2, n_outer=1, n_corr=2, n_non_orth_corr=0,
                momentum_predictor=True, alpha_u=1.0, alpha_p=1.0, u_type=np.zeros(nP, np.int32),
                u_value=np.zeros(3 * nP), p_type=np.zeros(nP, np.int32), p_value=np.zeros(nP),
                U=_ctl("PBiCGStab", "DILU", 1e-8, 0.0, 1000), p=_ctl("PCG", "GAMG", 1e-8, 0.01, 2000),
                pFinal=_ctl("PCG", "GAMG", 1e-8, 0.0, 2000), p_ref_cell=0, p_ref_value=0.0)
    return m, case, U0


def channel_beta(ny, y1, height=2.0):
    """tanh grading parameter beta of a two-sided stretched wall-normal direction of ny cells whose
    first cell is y1 high (bisection on tanhStretch, RawMesh.cpp:387-389)."""
    def first(beta):
        t = 2.0 / ny - 1.0
        return 0.5 * height * (1.0 + math.tanh(beta * t) / math.tanh(beta))
    lo, hi = 1e-6, 20.0
    if first(lo) <= y1:
        return 0.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if first(mid) > y1:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def channel(n=(256, 192, 128), Re_b=6875.0, Re_tau=395.0, y_plus1=1.0, ubar=1.0, noise=0.1, seed=20261203,
            les=True, van_driest=True, beta=None):
    """Periodic channel 2pi x 2 x pi (x streamwise and z spanwise periodic, walls at yMin / yMax,
    half-height 1), tanh-graded in y so that the first cell has y+ ~ y_plus1 at Re_tau; nu = ubar / Re_b
    (Re_b 6875 <-> Re_tau ~ 395, the reference's channel395 case); mean-velocity forcing to Ubar =
    (ubar, 0, 0) (fvmFlow.cpp:182-194); Smagorinsky LES with Van Driest damping (LESModels.cpp); the
    fvmFlow transient defaults (backward, linear, nOuter 1, nCorr 2; U {PBiCGStab, DILU, 1e-8},
    p {PCG, GAMG, 1e-8, relTol 0.01}, pFinal relTol 0).  Initial field: the laminar profile
    1.5 ubar (1 - (y - 1)^2) plus a seeded uniform perturbation of +-noise*ubar in every component.
    Returns (mesh, case, model, U0, dt) with dt at a Courant number of ~0.5."""
    from . import mesh as vm
    nx, ny, nz = (int(v) for v in n)
    if beta is None:
        beta = channel_beta(ny, y_plus1 / Re_tau)
    m = vm.box_mesh((nx, ny, nz), hi=(2 * np.pi, 2.0, np.pi), periodic=(True, False, True), beta=(0.0, beta, 0.0))
    nP = len(m["patch_start"])
    walls = np.array([1 if m["patch_names"][q] in ("yMin", "yMax") else 0 for q in range(nP)], np.int32)
    case = dict(nu=ubar / Re_b, steady=False, div_scheme=1, ddt_scheme=2, n_outer=1, n_corr=2, n_non_orth_corr=0,
                momentum_predictor=True, alpha_u=1.0, alpha_p=1.0, u_type=walls.copy(), u_value=np.zeros(3 * nP),
                p_type=np.zeros(nP, np.int32), p_value=np.zeros(nP),
                U=_ctl("PBiCGStab", "DILU", 1e-8, 0.0, 1000), p=_ctl("PCG", "GAMG", 1e-8, 0.01, 2000),
                pFinal=_ctl("PCG", "GAMG", 1e-8, 0.0, 2000), p_ref_cell=0, p_ref_value=0.0)
    model = dict(les="Smagorinsky" if les else "laminar", van_driest=bool(van_driest), wall_patch=walls,
                 forcing="meanVelocity", Ubar=(ubar, 0.0, 0.0))
    y = m["C"][:, 1]
    rng = np.random.default_rng(seed)
    U0 = np.zeros((m["n_cells"], 3))
    U0[:, 0] = 1.5 * ubar * (1.0 - (y - 1.0) ** 2)
    U0 += noise * ubar * rng.uniform(-1.0, 1.0, size=U0.shape)
    dt = 0.5 * (2 * np.pi / nx) / (1.5 * ubar + noise * ubar)
    return m, case, model, U0, dt


def serving_trace(n_requests=32, rate_hz=2.0, seed=20261203, n_range=(32, 256), re_range=(100.0, 1000.0)):
    """Serving stream of steady lid-cavity solves: Poisson arrivals of the given rate (seeded),
    mesh N x N with N uniform in n_range (inclusive), Re uniform in re_range.
    Returns a list of dicts (arrival s, n, Re)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n_requests))
    t -= t[0]
    ns = rng.integers(n_range[0], n_range[1] + 1, n_requests)
    res = rng.uniform(re_range[0], re_range[1], n_requests)
    return [dict(arrival=float(a), n=int(n), Re=float(r)) for a, n, r in zip(t, ns, res)]
