"""ctypes loader for oracle/_ref/libvlmref.so — the UNMODIFIED reference compiled from its
own sources (see oracle/Makefile) plus oracle/ref_driver.cpp.

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libvlmref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference oracle not built: {LIB_PATH} (run make -C oracle REF=<reference tree>)")
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        dp = np.ctypeslib.ndpointer(np.float64, flags="C")
        L.ref_last_error.restype = C.c_char_p
        L.ref_mesh_box.restype = P
        L.ref_mesh_box.argtypes = [P, P, P, P, C.c_int, P, P, P]
        L.ref_mesh_free.argtypes = [P]
        L.ref_mesh_sizes.argtypes = [P, P]
        L.ref_mesh_get.argtypes = [P, C.c_char_p, P]
        L.ref_mesh_ncellfaces.argtypes = [P]
        L.ref_set_reproducible.argtypes = [C.c_int]
        L.ref_amul.argtypes = [P, P, P, P, P, P]
        L.ref_solve_ldu.argtypes = [P, P, P, P, P, P, C.c_char_p, C.c_char_p, C.c_double, C.c_double,
                                    C.c_int, C.c_int, C.c_int, P]
        L.ref_gamg_nlevels.argtypes = [P]
        L.ref_gamg_level.argtypes = [P, C.c_int] + [P] * 11
        L.ref_gamg_meta.argtypes = [P, P, P]
        L.ref_gamg_apply.argtypes = [P, P, P, P, P, P]
        L.ref_laplacian.argtypes = [P, P, P, P, P, C.c_int, C.c_int, P, P, P, P, P, P, P]
        L.ref_grad.argtypes = [P, P, P, P, C.c_int, P]
        L.ref_pressure_solve.argtypes = [P, P, P, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_char_p,
                                         C.c_double, C.c_double, C.c_int, P, P, P]
        L.ref_exact_sum.restype = C.c_double
        L.ref_exact_sum.argtypes = [P, C.c_long]
        L.ref_flow_run.argtypes = [P, C.POINTER(RefFlowSpec), C.c_int, C.c_double, P, P, P, P, C.POINTER(C.c_int)]
        L.ref_flow_run_model.argtypes = [P, C.POINTER(RefFlowSpec), C.POINTER(RefModelSpec), C.c_int, C.c_double,
                                         P, P, P, P, C.POINTER(C.c_int), P, P]
        L.ref_flow_run_restart.argtypes = [P, C.POINTER(RefFlowSpec), C.POINTER(RefModelSpec), C.c_char_p,
                                           C.c_char_p, C.c_int, C.c_double, P, P, P, P, C.POINTER(C.c_int), P, P]
        L.ref_flow_error.restype = C.c_char_p
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().ref_last_error().decode())


class RefSolverCtl(C.Structure):
    _fields_ = [("solver", C.c_char * 32), ("preconditioner", C.c_char * 32), ("tolerance", C.c_double),
                ("relTol", C.c_double), ("maxIter", C.c_int), ("minIter", C.c_int), ("nSweeps", C.c_int)]


class RefFlowSpec(C.Structure):
    _fields_ = [("nu", C.c_double), ("steady", C.c_int), ("divScheme", C.c_int), ("ddtScheme", C.c_int),
                ("nOuter", C.c_int), ("nCorr", C.c_int), ("nNonOrthCorr", C.c_int), ("momentumPredictor", C.c_int),
                ("alphaU", C.c_double), ("alphaP", C.c_double), ("nPatches", C.c_int), ("uType", C.c_void_p),
                ("uValue", C.c_void_p), ("pType", C.c_void_p), ("pValue", C.c_void_p), ("U", RefSolverCtl),
                ("p", RefSolverCtl), ("pFinal", RefSolverCtl), ("pRefCell", C.c_int), ("pRefValue", C.c_double),
                ("reproducible", C.c_int), ("residualTol", C.c_double), ("divK", C.c_double),
                ("uFace", C.c_void_p), ("pFace", C.c_void_p), ("gradScheme", C.c_int),
                ("gradPScheme", C.c_int), ("uRobin", C.c_void_p), ("pRobin", C.c_void_p),
                ("uAdv", C.c_void_p)]


class RefModelSpec(C.Structure):
    _fields_ = [("turbulence", C.c_char_p), ("forcing", C.c_int), ("force", C.c_double * 3),
                ("Ubar", C.c_double * 3), ("relaxation", C.c_double), ("gradP", C.c_double)]


def _model_spec(model):
    """RefModelSpec of a Flow.set_model dict: the turbulence dictionary as the reference's case files
    write it ("model", "vanDriest", "coeffs"; LESModels.cpp:17-60, 274-281) and the forcing."""
    les = model.get("les", "laminar")
    les = {0: "laminar", 1: "Smagorinsky"}.get(les, les)
    turb = None
    if les != "laminar":
        coeffs = {k: model[k] for k in ("Cs", "Aplus", "Cdelta", "kappa") if k in model}
        if "delta_coeff" in model:
            coeffs["deltaCoeff"] = model["delta_coeff"]
        d = {"model": les, "vanDriest": bool(model.get("van_driest", False)), "coeffs": coeffs}
        if "nut_max_ratio" in model:
            d["nutMaxRatio"] = model["nut_max_ratio"]
        turb = json.dumps(d).encode()
    ms = RefModelSpec()
    ms.turbulence = turb
    fo = model.get("forcing", "none")
    ms.forcing = {"none": 0, "constant": 1, "meanVelocity": 2}[fo] if isinstance(fo, str) else int(fo)
    for k, v in enumerate(model.get("force", (0.0, 0.0, 0.0))):
        ms.force[k] = v
    for k, v in enumerate(model.get("Ubar", (0.0, 0.0, 0.0))):
        ms.Ubar[k] = v
    ms.relaxation = model.get("relaxation", 1.0)
    ms.gradP = model.get("grad_p", 0.0)
    return ms, turb


def _solver_ctl(d):
    c = RefSolverCtl()
    c.solver = d["solver"].encode()
    c.preconditioner = d["preconditioner"].encode()
    c.tolerance, c.relTol = d["tolerance"], d["relTol"]
    c.maxIter, c.minIter, c.nSweeps = d["maxIter"], d.get("minIter", 0), d.get("nSweeps", 1)
    return c


class RefMesh:
    """A reference Mesh built by generateBox + Mesh::build (mesh/RawMesh.cpp:391, mesh/Mesh.cpp:476)."""

    def __init__(self, n, lo=(0, 0, 0), hi=(1, 1, 1), periodic=(0, 0, 0), two_d=False, beta=(0, 0, 0),
                 points=None, patch_types=None):
        L = lib()
        n_ = np.asarray(n, np.int32)
        lo_ = np.asarray(lo, np.float64)
        hi_ = np.asarray(hi, np.float64)
        per = np.asarray(periodic, np.int32)
        be = np.asarray(beta, np.float64)
        pts = None if points is None else np.ascontiguousarray(points, np.float64)
        pt = None if patch_types is None else np.asarray(patch_types, np.int32)
        self._h = L.ref_mesh_box(_p(n_), _p(lo_), _p(hi_), _p(per), int(two_d), _p(be), _p(pts), _p(pt))
        if not self._h:
            raise RuntimeError(L.ref_last_error().decode())
        s = np.zeros(8, np.int32)
        L.ref_mesh_sizes(self._h, _p(s))
        (self.n_cells, self.n_internal_faces, self.n_faces, self.n_patches, two, self.empty_dir,
         skew) = [int(v) for v in s[:7]]
        self.two_d = bool(two)
        self.skewed = bool(skew)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.ref_mesh_free(self._h)
            self._h = None

    def get(self, name):
        nC, nI, nF, nP = self.n_cells, self.n_internal_faces, self.n_faces, self.n_patches
        shapes = {"owner": (nF, np.int32), "neighbour": (nI, np.int32), "V": (nC, np.float64),
                  "magSf": (nF, np.float64), "w": (nF, np.float64), "deltaCoeffs": (nF, np.float64),
                  "ndc": (nF, np.float64), "C": ((nC, 3), np.float64), "Sf": ((nF, 3), np.float64),
                  "Cf": ((nF, 3), np.float64), "d": ((nF, 3), np.float64), "corrVecs": ((nF, 3), np.float64),
                  "skewVecs": ((nF, 3), np.float64), "patchStart": (nP, np.int32), "patchSize": (nP, np.int32),
                  "cellFaceOffsets": (nC + 1, np.int32),
                  "cellFaces": (lib().ref_mesh_ncellfaces(self._h), np.int32)}
        shp, dt = shapes[name]
        out = np.zeros(shp, dt)
        _check(lib().ref_mesh_get(self._h, name.encode(), _p(out)))
        return out

    # ------------------------------------------------------------------ incompressible step
    def flow_run(self, case, n_steps, dt=1.0, U=None, p=None, reproducible=False, residual_tol=0.0, model=None,
                 read_restart=None, write_restart=None):
        """n_steps of IncompressibleFlow::step(dt) (solvers/IncompressibleFlow.cpp:138-370) with the case
        settings of `case` (a dict, voluma_b200.cases.lid_cavity layout).  residual_tol > 0 stops at
        convergence like fvmFlow's steady loop.  Returns U (n,3), p, phi, and the per-step history
        [UInitialResidual, pInitialResidual, continuityError, linear iterations] of the steps run.
        `model` (the Flow.set_model dict) adds the reference's turbulence model, built from the equivalent
        "turbulence" case dictionary by TurbulenceModel::create, and the momentum forcing; the run then
        also returns nu_t per cell and the final forcing gradP.  read_restart / write_restart: directories
        the run continues from (restart::read) and ends by writing (restart::write); either implies the
        model form of the return."""
        nC = self.n_cells
        Uc = np.zeros((nC, 3)) if U is None else np.ascontiguousarray(U, np.float64).reshape(nC, 3).copy()
        pc = np.zeros(nC) if p is None else np.ascontiguousarray(p, np.float64).copy()
        phi = np.zeros(self.n_faces)
        hist = np.zeros((n_steps, 4))
        keep = [np.ascontiguousarray(case["u_type"], np.int32), np.ascontiguousarray(case["u_value"], np.float64),
                np.ascontiguousarray(case["p_type"], np.int32), np.ascontiguousarray(case["p_value"], np.float64)]
        sp = RefFlowSpec()
        sp.nu = case["nu"]
        sp.steady, sp.divScheme, sp.ddtScheme = int(case["steady"]), case["div_scheme"], case["ddt_scheme"]
        sp.nOuter, sp.nCorr, sp.nNonOrthCorr = case["n_outer"], case["n_corr"], case["n_non_orth_corr"]
        sp.momentumPredictor = int(case["momentum_predictor"])
        sp.alphaU, sp.alphaP = case["alpha_u"], case["alpha_p"]
        sp.nPatches = self.n_patches
        sp.uType, sp.uValue, sp.pType, sp.pValue = (_p(a) for a in keep)
        sp.U, sp.p, sp.pFinal = (_solver_ctl(case[k]) for k in ("U", "p", "pFinal"))
        sp.pRefCell, sp.pRefValue = case["p_ref_cell"], case["p_ref_value"]
        sp.reproducible = int(reproducible)
        sp.residualTol = residual_tol
        sp.divK = case.get("div_coeff", 1.0)
        sp.gradScheme = int(case.get("grad_scheme", 0))
        sp.gradPScheme = int(case.get("grad_p_scheme", 0))
        if case.get("u_face") is not None:  # face-by-face values (boundary faces in mesh order)
            keep.append(np.ascontiguousarray(case["u_face"], np.float64).reshape(-1))
            sp.uFace = _p(keep[-1])
        if case.get("p_face") is not None:
            keep.append(np.ascontiguousarray(case["p_face"], np.float64).reshape(-1))
            sp.pFace = _p(keep[-1])
        # Robin {a, b} per patch, advective {lInf, fieldInf} per patch
        for key, field in (("u_robin", "uRobin"), ("p_robin", "pRobin"), ("u_advective", "uAdv")):
            if case.get(key) is not None:
                keep.append(np.ascontiguousarray(case[key], np.float64).reshape(-1))
                setattr(sp, field, _p(keep[-1]))
        ran = C.c_int()
        if read_restart is not None or write_restart is not None:
            ms, turb = _model_spec(model or {})
            nut = np.zeros(nC)
            gp = np.zeros(1)
            rd = None if read_restart is None else os.fspath(read_restart).encode()
            wd = None if write_restart is None else os.fspath(write_restart).encode()
            if lib().ref_flow_run_restart(self._h, C.byref(sp), C.byref(ms), rd, wd, n_steps, dt, _p(Uc), _p(pc),
                                          _p(phi), _p(hist), C.byref(ran), _p(nut), _p(gp)) != 0:
                raise RuntimeError(lib().ref_flow_error().decode())
            return Uc, pc, phi, hist[:ran.value], nut, float(gp[0])
        if model is None:
            if lib().ref_flow_run(self._h, C.byref(sp), n_steps, dt, _p(Uc), _p(pc), _p(phi), _p(hist),
                                  C.byref(ran)) != 0:
                raise RuntimeError(lib().ref_flow_error().decode())
            return Uc, pc, phi, hist[:ran.value]
        ms, turb = _model_spec(model)
        nut = np.zeros(nC)
        gp = np.zeros(1)
        if lib().ref_flow_run_model(self._h, C.byref(sp), C.byref(ms), n_steps, dt, _p(Uc), _p(pc), _p(phi), _p(hist),
                                    C.byref(ran), _p(nut), _p(gp)) != 0:
            raise RuntimeError(lib().ref_flow_error().decode())
        return Uc, pc, phi, hist[:ran.value], nut, float(gp[0])

    # ------------------------------------------------------------------ linear algebra
    def amul(self, diag, upper, lower, x):
        y = np.zeros(self.n_cells)
        _check(lib().ref_amul(self._h, _p(np.ascontiguousarray(diag, np.float64)),
                              _p(np.ascontiguousarray(upper, np.float64)),
                              None if lower is None else _p(np.ascontiguousarray(lower, np.float64)),
                              _p(np.ascontiguousarray(x, np.float64)), _p(y)))
        return y

    def solve(self, diag, upper, lower, b, x0, solver="PCG", precond="diagonal", tol=0.0, rel_tol=1e-8,
              max_iter=1000, min_iter=0, n_sweeps=1, reproducible=False):
        """solveLdu (linalg/LinearSolver.cpp:135). Returns (x, perf dict)."""
        L = lib()
        L.ref_set_reproducible(1 if reproducible else 0)
        x = np.ascontiguousarray(x0, np.float64).copy()
        perf = np.zeros(6)
        low = None if lower is None else np.ascontiguousarray(lower, np.float64)
        try:
            _check(L.ref_solve_ldu(self._h, _p(np.ascontiguousarray(diag, np.float64)),
                                   _p(np.ascontiguousarray(upper, np.float64)), _p(low),
                                   _p(np.ascontiguousarray(b, np.float64)), _p(x), solver.encode(),
                                   precond.encode(), tol, rel_tol, max_iter, min_iter, n_sweeps, _p(perf)))
        finally:
            L.ref_set_reproducible(0)
        return x, dict(initialResidual=perf[0], finalResidual=perf[1], residualSum=perf[2],
                       normFactor=perf[3], iterations=int(perf[4]), converged=bool(perf[5]))

    def gamg_levels(self):
        """buildHierarchy (linalg/GAMG.cpp:206) per level: dict of n, l, u, weight, agg, faceMap, faceFlip,
        off, adjCell, adjFace, adjIsL."""
        L = lib()
        out = []
        for lev in range(L.ref_gamg_nlevels(self._h)):
            s = np.zeros(4, np.int32)
            _check(L.ref_gamg_level(self._h, lev, _p(s), *([None] * 10)))
            n, nf, nagg, nnz = [int(v) for v in s]
            d = dict(n=n, l=np.zeros(nf, np.int32), u=np.zeros(nf, np.int32), weight=np.zeros(nf),
                     agg=np.zeros(nagg, np.int32), faceMap=np.zeros(nf if nagg else 0, np.int32),
                     faceFlip=np.zeros(nf if nagg else 0, np.int8), off=np.zeros(n + 1, np.int32),
                     adjCell=np.zeros(nnz, np.int32), adjFace=np.zeros(nnz, np.int32),
                     adjIsL=np.zeros(nnz, np.int8))
            _check(L.ref_gamg_level(self._h, lev, _p(s), _p(d["l"]), _p(d["u"]), _p(d["weight"]), _p(d["agg"]),
                                    _p(d["faceMap"]), _p(d["faceFlip"]), _p(d["off"]), _p(d["adjCell"]),
                                    _p(d["adjFace"]), _p(d["adjIsL"])))
            out.append(d)
        return out

    def gamg_apply(self, diag, upper, lower, r):
        w = np.zeros(self.n_cells)
        _check(lib().ref_gamg_apply(self._h, _p(np.ascontiguousarray(diag, np.float64)),
                                    _p(np.ascontiguousarray(upper, np.float64)),
                                    None if lower is None else _p(np.ascontiguousarray(lower, np.float64)),
                                    _p(np.ascontiguousarray(r, np.float64)), _p(w)))
        return w

    # ------------------------------------------------------------------ discretisation
    def laplacian(self, gamma, psi, bc_type, bc_values=None, non_orth_corr=True, grad_scheme=0):
        nC, nI, nF = self.n_cells, self.n_internal_faces, self.n_faces
        nB = nF - nI
        out = dict(diag=np.zeros(nC), upper=np.zeros(nI), source=np.zeros(nC), internalCoeffs=np.zeros(nB),
                   boundarySource=np.zeros(nB), ffc=np.zeros(nF))
        has = np.zeros(1, np.int32)
        bv = None if bc_values is None else np.ascontiguousarray(bc_values, np.float64)
        _check(lib().ref_laplacian(self._h, _p(np.ascontiguousarray(gamma, np.float64)),
                                   _p(np.ascontiguousarray(psi, np.float64)),
                                   _p(np.ascontiguousarray(bc_type, np.int32)), _p(bv), int(non_orth_corr),
                                   int(grad_scheme), _p(out["diag"]), _p(out["upper"]), _p(out["source"]),
                                   _p(out["internalCoeffs"]), _p(out["boundarySource"]), _p(out["ffc"]),
                                   _p(has)))
        out["hasFfc"] = bool(has[0])
        return out

    def grad(self, psi, bc_type, bc_values=None, scheme=0):
        g = np.zeros((self.n_cells, 3))
        bv = None if bc_values is None else np.ascontiguousarray(bc_values, np.float64)
        _check(lib().ref_grad(self._h, _p(np.ascontiguousarray(psi, np.float64)),
                              _p(np.ascontiguousarray(bc_type, np.int32)), _p(bv), int(scheme), _p(g)))
        return g

    def pressure_solve(self, gamma, div_phi, p0, ref_cell=0, n_non_orth=0, grad_scheme=1, solver="PCG",
                       precond="GAMG", tol=0.0, rel_tol=1e-8, max_iter=1000, reproducible=False):
        """laplacian + (-= divPhi) + setReference + solve, n_non_orth+1 times, with zeroGradient walls
        (IncompressibleFlow.cpp:62-71). Returns (p, flux of the last pass, perf rows)."""
        L = lib()
        p = np.ascontiguousarray(p0, np.float64).copy()
        flux = np.zeros(self.n_faces)
        perf = np.zeros(6 * (n_non_orth + 1))
        L.ref_set_reproducible(1 if reproducible else 0)
        try:
            _check(L.ref_pressure_solve(self._h, _p(np.ascontiguousarray(gamma, np.float64)),
                                        _p(np.ascontiguousarray(div_phi, np.float64)), int(ref_cell),
                                        int(n_non_orth), int(grad_scheme), solver.encode(), precond.encode(),
                                        tol, rel_tol, max_iter, _p(p), _p(flux), _p(perf)))
        finally:
            L.ref_set_reproducible(0)
        return p, flux, perf.reshape(-1, 6)


def exact_sum(v) -> float:
    v = np.ascontiguousarray(v, np.float64)
    return float(lib().ref_exact_sum(_p(v), v.size))


# ---------------------------------------------------------------------- drop-in check
DROPIN_PATH = os.path.join(HERE, "_ref", "libvlmdropin.so")
_dropin = None


def dropin_available() -> bool:
    return os.path.exists(DROPIN_PATH)


def dropin_pressure_solve(n, gamma, div_phi, p0, lo=(0, 0, 0), hi=(1, 1, 1), periodic=(0, 0, 0), points=None,
                          ref_cell=0, n_non_orth=0, grad_scheme=1, solver="PCG", precond="GAMG", tol=0.0,
                          rel_tol=1e-8, max_iter=1000, reproducible=False, smoother="", precision=""):
    """The reference's pressure loop (laplacian, -= divPhi, setReference, FvMatrix::solve) with its
    solveLdu calls redirected to the GPU library (oracle/dropin_driver.cpp).  Returns
    (p, flux, perf rows, number of solveLdu calls that reached the GPU)."""
    global _dropin
    if _dropin is None:
        L = C.CDLL(DROPIN_PATH)
        P = C.c_void_p
        L.dropin_last_error.restype = C.c_char_p
        L.dropin_pressure_solve.argtypes = [P, P, P, P, P, P, P, C.c_int, C.c_int, C.c_int, C.c_char_p, C.c_char_p,
                                            C.c_double, C.c_double, C.c_int, C.c_int, C.c_char_p, C.c_char_p, P, P,
                                            P]
        _dropin = L
    L = _dropin
    before = L.dropin_calls()
    p = np.ascontiguousarray(p0, np.float64).copy()
    nF = len(gamma)
    flux = np.zeros(nF)
    perf = np.zeros(6 * (n_non_orth + 1))
    pts = None if points is None else np.ascontiguousarray(points, np.float64)
    rc = L.dropin_pressure_solve(_p(np.asarray(n, np.int32)), _p(np.asarray(lo, np.float64)),
                                 _p(np.asarray(hi, np.float64)), _p(np.asarray(periodic, np.int32)), _p(pts),
                                 _p(np.ascontiguousarray(gamma, np.float64)),
                                 _p(np.ascontiguousarray(div_phi, np.float64)), int(ref_cell), int(n_non_orth),
                                 int(grad_scheme), solver.encode(), precond.encode(), tol, rel_tol, max_iter,
                                 int(reproducible), smoother.encode(), precision.encode(), _p(p), _p(flux), _p(perf))
    if rc != 0:
        raise RuntimeError(L.dropin_last_error().decode())
    return p, flux, perf.reshape(-1, 6), L.dropin_calls() - before
