"""Generates the golden fixtures of tests/golden/ from the reference itself.

Run where the reference sources are present:  make -C oracle REF=<reference tree> && python
tests/golden/make_golden.py.  Every array comes from the unmodified reference compiled from its
own sources (oracle/_ref/libvlmref.so through oracle/ref_driver.cpp): generateBox + Mesh::build
meshes, the LDU pressure matrix of fvm::laplacian(1, p) + setReference(0), and the results of
solveLdu (PCG/diagonal in CFD_REPRODUCIBLE mode and plain, PCG/GAMG, PBiCGStab/diagonal,
PBiCGStab/DILU, PCG/DIC, GaussSeidel, symGaussSeidel, Jacobi),
one GamgPreconditioner::apply, buildHierarchy, amul and ExactSum.  The fixtures are small
(each case < 0.5 MB) so the CPU tests load them in milliseconds.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from voluma_b200 import mesh as vm  # noqa: E402

CASES = {
    "periodic8": dict(n=(8, 8, 8), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1)),
    "walls7x5x3": dict(n=(7, 5, 3)),
    "cavity16": dict(n=(16, 16, 1), hi=(1, 1, 0.1), two_d=True),
    "stretched6x9x5": dict(n=(6, 9, 5), periodic=(1, 0, 1), beta=(0, 2.0, 0)),
    "jitter10x8x6": dict(n=(10, 8, 6), beta=(1.2, 0, 0.7), jitter=(0.2, 3)),
    "periodic24": dict(n=(24, 24, 24), hi=(2 * np.pi,) * 3, periodic=(1, 1, 1)),
}

MESH_KEYS = ["owner", "neighbour", "V", "C", "Sf", "magSf", "Cf", "d", "w", "deltaCoeffs", "ndc", "corrVecs",
             "skewVecs", "patchStart", "patchSize"]


def make(name, spec):
    spec = dict(spec)
    jit = spec.pop("jitter", None)
    pts = None
    if jit:
        pts = vm.jitter_interior(vm.box_points(spec["n"], spec.get("lo", (0, 0, 0)), spec.get("hi", (1, 1, 1)),
                                               spec.get("beta", (0, 0, 0))), spec["n"], *jit)
    R = ref.RefMesh(spec["n"], spec.get("lo", (0, 0, 0)), spec.get("hi", (1, 1, 1)), spec.get("periodic", (0, 0, 0)),
                    spec.get("two_d", False), spec.get("beta", (0, 0, 0)), points=pts)
    out = {k: R.get(k) for k in MESH_KEYS}
    out["sizes"] = np.array([R.n_cells, R.n_internal_faces, R.n_faces, R.n_patches, int(R.two_d), R.empty_dir,
                             int(R.skewed)])
    out["spec_n"] = np.array(spec["n"])
    out["spec_lo"] = np.array(spec.get("lo", (0, 0, 0)), float)
    out["spec_hi"] = np.array(spec.get("hi", (1, 1, 1)), float)
    out["spec_periodic"] = np.array(spec.get("periodic", (0, 0, 0)))
    out["spec_two_d"] = np.array(int(spec.get("two_d", False)))
    out["spec_beta"] = np.array(spec.get("beta", (0, 0, 0)), float)
    if pts is not None:
        out["points"] = pts
    nC, nI = R.n_cells, R.n_internal_faces
    mesh = dict(n_cells=nC, n_internal_faces=nI, n_faces=R.n_faces, owner=out["owner"], neighbour=out["neighbour"],
                magSf=out["magSf"], ndc=out["ndc"])
    diag, upper = vm.poisson_matrix(mesh)
    rng = np.random.default_rng(7)
    b = rng.standard_normal(nC)
    b -= b.mean()
    x0 = 0.01 * rng.standard_normal(nC)
    out.update(diag=diag, upper=upper, b=b, x0=x0)
    xa = rng.standard_normal(nC)
    out["amul_x"] = xa
    out["amul_y"] = R.amul(diag, upper, None, xa)
    lower = upper * (0.75 + 0.5 * rng.random(nI))  # an asymmetric matrix for PBiCGStab
    out["lower_asym"] = lower
    runs = {
        "pcg_diag_repro": (diag, upper, None, "PCG", "diagonal", True),
        "pcg_diag": (diag, upper, None, "PCG", "diagonal", False),
        "pcg_gamg": (diag, upper, None, "PCG", "GAMG", False),
        "bicg_diag_repro": (diag, upper, lower, "PBiCGStab", "diagonal", True),
        "bicg_gamg": (diag, upper, lower, "PBiCGStab", "GAMG", False),
    }
    for key, (d, u, l, solver, prec, repro) in runs.items():
        x, perf = R.solve(d, u, l, b, x0, solver, prec, 0.0, 1e-8, 2000, reproducible=repro)
        out[key + "_x"] = x
        out[key + "_perf"] = np.array([perf["initialResidual"], perf["finalResidual"], perf["residualSum"],
                                       perf["normFactor"], perf["iterations"], perf["converged"]])
    # DIC / DILU and the relaxation solvers (LinearSolver.cpp:56-112, 238-278)
    runs2 = {
        "bicg_dilu": (lower, "PBiCGStab", "DILU", 1e-8, 2000, 1),
        "pcg_dic": (None, "PCG", "DIC", 1e-8, 2000, 1),
        "gs": (None, "GaussSeidel", "none", 1e-3, 300, 2),
        "sgs": (lower, "symGaussSeidel", "none", 1e-3, 300, 1),
        "jac": (None, "Jacobi", "none", 1e-3, 300, 3),
    }
    for key, (l, solver, prec, rtol, mx, nsw) in runs2.items():
        x, perf = R.solve(diag, upper, l, b, x0, solver, prec, 0.0, rtol, mx, n_sweeps=nsw)
        out[key + "_x"] = x
        out[key + "_perf"] = np.array([perf["initialResidual"], perf["finalResidual"], perf["residualSum"],
                                       perf["normFactor"], perf["iterations"], perf["converged"]])
    out["vcycle_w"] = R.gamg_apply(diag, upper, None, b)
    levels = R.gamg_levels()
    out["nlevels"] = np.array(len(levels))
    for k, L in enumerate(levels):
        for f in ("l", "u", "weight", "agg", "faceMap", "faceFlip"):
            out[f"lev{k}_{f}"] = L[f]
    # ---- assembly: fvm::laplacian with its non-orthogonal correction, fvc::grad, pressure loop
    nP = R.n_patches
    gamma = 0.5 + rng.random(R.n_faces)
    psi = rng.standard_normal(nC)
    bct = np.zeros(max(nP, 1), np.int32)
    if nP:
        bct[0] = 1  # fixedValue on the first patch, zeroGradient elsewhere
    bcv = rng.standard_normal(R.n_faces - nI)
    out.update(lap_gamma=gamma, lap_psi=psi, lap_bctype=bct, lap_bcvalues=bcv)
    for gs in (0, 1):
        L = R.laplacian(gamma, psi, bct[:nP] if nP else bct, bcv, non_orth_corr=True, grad_scheme=gs)
        for k2, v2 in L.items():
            out[f"lap{gs}_{k2}"] = np.asarray(v2)
        out[f"grad{gs}"] = R.grad(psi, bct[:nP] if nP else bct, bcv, scheme=gs)
    divphi = rng.standard_normal(nC)
    divphi -= (divphi * out["V"]).sum() / out["V"].sum()
    out["ps_gamma"] = gamma
    out["ps_divphi"] = divphi
    p_r, flux_r, perf_r = R.pressure_solve(gamma, divphi, np.zeros(nC), ref_cell=0, n_non_orth=2, grad_scheme=1,
                                           solver="PCG", precond="diagonal", rel_tol=1e-8, max_iter=3000,
                                           reproducible=True)
    out.update(ps_p=p_r, ps_flux=flux_r, ps_perf=perf_r)
    out["exact_sum_b"] = np.array(ref.exact_sum(b))
    spread = rng.standard_normal(4096) * np.exp(rng.uniform(-40, 40, 4096))
    out["exact_spread"] = spread
    out["exact_spread_sum"] = np.array(ref.exact_sum(spread))
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(name, nC, "cells", len(levels), "levels")


if __name__ == "__main__":
    for name, spec in CASES.items():
        make(name, spec)
