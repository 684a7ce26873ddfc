"""ctypes loader for oracle/_build/libvlmoracle.so — the CPU restatement of the reference's
solve path (oracle/vlm_oracle.c).  Test infrastructure only: imported by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, never by the product package."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libvlmoracle.so")
SMOOTHERS = {"gs": 0, "mcgs": 1, "jacobi": 2, "mcgs-jacobi": 3}

_lib = None


class GamgOpts(C.Structure):
    _fields_ = [("smoother", C.c_int), ("omega", C.c_double), ("coarse", C.c_int), ("mergeLevels", C.c_int),
                ("matching", C.c_int)]


def build():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.vo_exact_sum.restype = C.c_double
        L.vo_exact_sum.argtypes = [P, C.c_long]
        L.vo_amul.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P]
        L.vo_hier_build.restype = P
        L.vo_hier_build.argtypes = [C.c_int, C.c_int, P, P, P, P, C.c_int, C.c_int]
        L.vo_hier_build_matching.restype = P
        L.vo_hier_build_matching.argtypes = [C.c_int, C.c_int, P, P, P, P, C.c_int, C.c_int]
        L.vo_hier_free.argtypes = [P]
        L.vo_hier_nlevels.argtypes = [P]
        L.vo_hier_level.argtypes = [P, C.c_int, P, P, P, P, P, P, P]
        L.vo_hier_colour.argtypes = [P, C.c_int, P]
        L.vo_gamg_apply.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P, C.POINTER(GamgOpts)]
        L.vo_solve.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P, C.c_char_p, C.c_char_p, C.c_double,
                               C.c_double, C.c_int, C.c_int, C.c_int, C.POINTER(GamgOpts), P]
        L.vo_solve_ex.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P, C.c_char_p, C.c_char_p, C.c_double,
                                  C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(GamgOpts), P]
        L.vo_precond_apply.argtypes = [C.c_int, C.c_int, P, P, P, P, P, C.c_char_p, P, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _d(a):
    return None if a is None else np.ascontiguousarray(a, np.float64)


def _i(a):
    return np.ascontiguousarray(a, np.int32)


def opts(smoother="gs", omega=1.0, coarse=0, merge=2, matching=False):
    return GamgOpts(SMOOTHERS[smoother] if isinstance(smoother, str) else smoother, omega, coarse, merge,
                    int(matching))


def exact_sum(v) -> float:
    v = _d(v)
    return float(lib().vo_exact_sum(_p(v), v.size))


def amul(m, diag, upper, lower, x):
    nI = len(m["neighbour"])
    y = np.zeros(m["n_cells"])
    lib().vo_amul(m["n_cells"], nI, _p(_i(m["owner"][:nI])), _p(_i(m["neighbour"])), _p(_d(diag)), _p(_d(upper)),
                  _p(_d(lower)), _p(_d(x)), _p(y))
    return y


def hierarchy(m, merge=2, n_coarsest=64, colours=False, matching=False):
    """buildHierarchy restated (matching: the device agglomeration's parallel matching): list of
    dicts n, l, u, weight, agg, faceMap, faceFlip (+colour)."""
    L = lib()
    nI = len(m["neighbour"])
    build = L.vo_hier_build_matching if matching else L.vo_hier_build
    h = build(m["n_cells"], nI, _p(_i(m["owner"][:nI])), _p(_i(m["neighbour"])), _p(_d(m["magSf"])),
              _p(_d(m["ndc"])), merge, n_coarsest)
    out = []
    try:
        for k in range(L.vo_hier_nlevels(h)):
            s = np.zeros(3, np.int32)
            L.vo_hier_level(h, k, _p(s), None, None, None, None, None, None)
            n, nf, na = (int(v) for v in s)
            d = dict(n=n, l=np.zeros(nf, np.int32), u=np.zeros(nf, np.int32), weight=np.zeros(nf),
                     agg=np.zeros(na, np.int32), faceMap=np.zeros(nf if na else 0, np.int32),
                     faceFlip=np.zeros(nf if na else 0, np.int8))
            L.vo_hier_level(h, k, _p(s), _p(d["l"]), _p(d["u"]), _p(d["weight"]), _p(d["agg"]), _p(d["faceMap"]),
                            _p(d["faceFlip"]))
            if colours:
                c = np.zeros(n, np.int32)
                d["ncolours"] = L.vo_hier_colour(h, k, _p(c))
                d["colour"] = c
            out.append(d)
    finally:
        L.vo_hier_free(h)
    return out


def gamg_apply(m, diag, upper, lower, r, smoother="gs", omega=1.0, coarse=0, merge=2):
    nI = len(m["neighbour"])
    w = np.zeros(m["n_cells"])
    o = opts(smoother, omega, coarse, merge)
    st = lib().vo_gamg_apply(m["n_cells"], nI, _p(_i(m["owner"][:nI])), _p(_i(m["neighbour"])), _p(_d(m["magSf"])),
                             _p(_d(m["ndc"])), _p(_d(diag)), _p(_d(upper)), _p(_d(lower)), _p(_d(r)), _p(w),
                             C.byref(o))
    if st:
        raise RuntimeError(f"oracle gamg_apply status {st}")
    return w


def solve(m, diag, upper, lower, b, x0, solver="PCG", precond="diagonal", tol=0.0, rel_tol=1e-8, max_iter=1000,
          min_iter=0, exact=False, smoother="gs", omega=1.0, coarse=0, merge=2, n_sweeps=1, matching=False):
    """solveLdu restated (PCG, PBiCGStab, GaussSeidel, symGaussSeidel, Jacobi). Returns (x, perf dict)."""
    nI = len(m["neighbour"])
    x = np.ascontiguousarray(x0, np.float64).copy()
    perf = np.zeros(6)
    o = opts(smoother, omega, coarse, merge, matching)
    st = lib().vo_solve_ex(m["n_cells"], nI, _p(_i(m["owner"][:nI])), _p(_i(m["neighbour"])), _p(_d(m["magSf"])),
                           _p(_d(m["ndc"])), _p(_d(diag)), _p(_d(upper)), _p(_d(lower)), _p(_d(b)), _p(x),
                           solver.encode(), precond.encode(), tol, rel_tol, max_iter, min_iter, n_sweeps, int(exact),
                           C.byref(o), _p(perf))
    if st:
        raise RuntimeError(f"oracle solve status {st}")
    return x, dict(initialResidual=perf[0], finalResidual=perf[1], residualSum=perf[2], normFactor=perf[3],
                   iterations=int(perf[4]), converged=bool(perf[5]))


def precond_apply(m, diag, upper, lower, r, precond="DILU"):
    """w = M^-1 r for none / diagonal / DIC / DILU (Preconditioner, linalg/LinearSolver.cpp:56-107)."""
    nI = len(m["neighbour"])
    w = np.zeros(m["n_cells"])
    st = lib().vo_precond_apply(m["n_cells"], nI, _p(_i(m["owner"][:nI])), _p(_i(m["neighbour"])), _p(_d(diag)),
                                _p(_d(upper)), _p(_d(lower)), precond.encode(), _p(_d(r)), _p(w))
    if st:
        raise RuntimeError(f"oracle precond_apply status {st}")
    return w
