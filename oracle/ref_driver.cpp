// Test-infrastructure driver over the UNMODIFIED Voluma reference sources.
//
// This file is part of the oracle, not of the product: it is linked with the
// reference's own src/fvm/{parallel/Comm,mesh/Mesh,mesh/RawMesh,linalg/LinearSolver,
// linalg/GAMG}.cpp (built by oracle/Makefile into oracle/_ref/) and exposes a
// plain C interface so the tests and the CPU baseline can call the reference's
// public API on the same inputs the CUDA path receives:
//   generateBox + Mesh::build         (mesh/RawMesh.cpp:391, mesh/Mesh.cpp:476)
//   amul / solveLdu                   (linalg/LinearSolver.cpp:121, :135)
//   buildHierarchy / GamgPreconditioner (linalg/GAMG.cpp:206, :263, :445)
//   fvm::laplacian / fvc::grad        (discretization/Fvm.h:141, Fvc.h:209)
//   par::ExactSum                     (parallel/Comm.h:42)
// Nothing here re-implements reference arithmetic; it only marshals arrays.

#include "fvm/discretization/Fvm.h"
#include "fvm/linalg/GAMG.h"
#include "fvm/linalg/LinearSolver.h"
#include "fvm/mesh/Mesh.h"
#include "fvm/mesh/RawMesh.h"
#include "fvm/parallel/Comm.h"

#include <cstring>
#include <exception>
#include <memory>
#include <string>

using namespace cfd;

namespace {
thread_local std::string g_err;

void setErr(const char* what) { g_err = what ? what : "unknown error"; }

template <class F> int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        setErr(e.what());
        return 1;
    }
}
} // namespace

struct RefMesh {
    MeshPtr mesh;
};

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

// Box mesh through generateBox + Mesh::build.  beta[d] > 0 applies tanhStretch(beta[d])
// in direction d.  `points` (optional, 3*(nx+1)*(ny+1)*(nz+1) doubles, point order of
// generateBox) replaces the generated vertex coordinates before Mesh::build, so callers
// can jitter vertices.  patchTypes[6] uses PatchType's order (0 patch, 1 wall, 2 symmetry).
RefMesh* ref_mesh_box(const int* n, const double* lo, const double* hi, const int* periodic, int twoD,
                      const double* beta, const double* points, const int* patchTypes) {
    RefMesh* out = nullptr;
    guarded([&] {
        BoxSpec s;
        for (int d = 0; d < 3; ++d) {
            s.n[d] = n[d];
            s.lo[d] = lo[d];
            s.hi[d] = hi[d];
            s.periodic[d] = periodic[d] != 0;
            if (beta && beta[d] > 0) s.stretch[d] = tanhStretch(beta[d]);
        }
        s.twoD = twoD != 0;
        if (patchTypes)
            for (int k = 0; k < 6; ++k) s.types[k] = PatchType(patchTypes[k]);
        RawMesh raw = generateBox(s);
        if (points)
            for (std::size_t p = 0; p < raw.points.size(); ++p)
                raw.points[p] = Vec3{points[3 * p], points[3 * p + 1], points[3 * p + 2]};
        out = new RefMesh{Mesh::build(&raw)};
    });
    return out;
}

void ref_mesh_free(RefMesh* m) { delete m; }

// sizes: nCells, nInternalFaces, nFaces, nPatches, twoD, emptyDir, skewed
void ref_mesh_sizes(const RefMesh* r, int* out) {
    const Mesh& m = *r->mesh;
    out[0] = m.nCells();
    out[1] = m.nInternalFaces();
    out[2] = m.nFaces();
    out[3] = int(m.patches().size());
    out[4] = m.twoD() ? 1 : 0;
    out[5] = m.emptyDir();
    out[6] = m.skewed() ? 1 : 0;
}

static void copyVec3(const std::vector<Vec3>& v, double* out) {
    for (std::size_t i = 0; i < v.size(); ++i) {
        out[3 * i] = v[i].x;
        out[3 * i + 1] = v[i].y;
        out[3 * i + 2] = v[i].z;
    }
}

// Copies one mesh array out. Names: owner neighbour (int32), V magSf w deltaCoeffs ndc
// (double), C Sf Cf d corrVecs skewVecs (3 doubles each), patchStart patchSize (int32),
// cellFaceOffsets cellFaces (int32).
int ref_mesh_get(const RefMesh* r, const char* what, void* out) {
    return guarded([&] {
        const Mesh& m = *r->mesh;
        const std::string w(what);
        auto cpyI = [&](const std::vector<label>& v) { std::memcpy(out, v.data(), v.size() * sizeof(label)); };
        auto cpyD = [&](const std::vector<scalar>& v) { std::memcpy(out, v.data(), v.size() * sizeof(scalar)); };
        if (w == "owner") cpyI(m.owner());
        else if (w == "neighbour") cpyI(m.neighbour());
        else if (w == "V") cpyD(m.V());
        else if (w == "magSf") cpyD(m.magSf());
        else if (w == "w") cpyD(m.w());
        else if (w == "deltaCoeffs") cpyD(m.deltaCoeffs());
        else if (w == "ndc") cpyD(m.nonOrthDeltaCoeffs());
        else if (w == "C") copyVec3(m.C(), static_cast<double*>(out));
        else if (w == "Sf") copyVec3(m.Sf(), static_cast<double*>(out));
        else if (w == "Cf") copyVec3(m.Cf(), static_cast<double*>(out));
        else if (w == "d") copyVec3(m.d(), static_cast<double*>(out));
        else if (w == "corrVecs") copyVec3(m.corrVecs(), static_cast<double*>(out));
        else if (w == "skewVecs") copyVec3(m.skewVecs(), static_cast<double*>(out));
        else if (w == "patchStart" || w == "patchSize") {
            auto* o = static_cast<int*>(out);
            for (std::size_t p = 0; p < m.patches().size(); ++p)
                o[p] = w == "patchStart" ? m.patches()[p].start : m.patches()[p].size;
        } else if (w == "cellFaceOffsets") cpyI(m.cellFaceOffsets());
        else if (w == "cellFaces") {
            cpyI(m.cellFaces());
        } else throw std::runtime_error("ref_mesh_get: unknown array " + w);
    });
}

int ref_mesh_ncellfaces(const RefMesh* r) { return int(r->mesh->cellFaces().size()); }

void ref_set_reproducible(int on) { par::setReproducible(on != 0); }

int ref_amul(const RefMesh* r, const double* diag, const double* upper, const double* lower, const double* x,
             double* y) {
    return guarded([&] {
        const Mesh& m = *r->mesh;
        const label n = m.nTotalCells();
        std::vector<scalar> d(diag, diag + n), xv(x, x + n), yv(n);
        std::vector<scalar> b(n, 0.0);
        LduSystem s{m, d, upper, lower ? lower : upper, b, lower == nullptr};
        amul(s, xv, yv);
        std::memcpy(y, yv.data(), n * sizeof(double));
    });
}

// perf: initialResidual, finalResidual, residualSum, normFactor, iterations, converged
int ref_solve_ldu(const RefMesh* r, const double* diag, const double* upper, const double* lower, const double* b,
                  double* x, const char* solver, const char* precond, double tol, double relTol, int maxIter,
                  int minIter, int nSweeps, double* perf) {
    return guarded([&] {
        const Mesh& m = *r->mesh;
        const label n = m.nTotalCells();
        std::vector<scalar> d(diag, diag + n), bv(b, b + n), xv(x, x + n);
        LduSystem s{m, d, upper, lower ? lower : upper, bv, lower == nullptr};
        SolverControls c;
        c.solver = solver;
        c.preconditioner = precond;
        c.tolerance = tol;
        c.relTol = relTol;
        c.maxIter = maxIter;
        c.minIter = minIter;
        c.nSweeps = nSweeps;
        const SolverPerformance p = solveLdu(s, xv, c);
        std::memcpy(x, xv.data(), n * sizeof(double));
        perf[0] = p.initialResidual;
        perf[1] = p.finalResidual;
        perf[2] = p.residualSum;
        perf[3] = p.normFactor;
        perf[4] = p.iterations;
        perf[5] = p.converged ? 1.0 : 0.0;
    });
}

int ref_gamg_nlevels(const RefMesh* r) { return int(gamgHierarchy(*r->mesh).levels.size()); }

// sizes: n, nFaces. Any output pointer may be null. agg/faceMap/faceFlip are empty on the
// coarsest level.
int ref_gamg_level(const RefMesh* r, int lev, int* sizes, int* l, int* u, double* weight, int* agg, int* faceMap,
                   signed char* faceFlip, int* off, int* adjCell, int* adjFace, signed char* adjIsL) {
    return guarded([&] {
        const auto& L = gamgHierarchy(*r->mesh).levels.at(lev);
        sizes[0] = L.n;
        sizes[1] = int(L.l.size());
        sizes[2] = int(L.agg.size());
        sizes[3] = int(L.adjCell.size());
        if (l) std::memcpy(l, L.l.data(), L.l.size() * sizeof(int));
        if (u) std::memcpy(u, L.u.data(), L.u.size() * sizeof(int));
        if (weight) std::memcpy(weight, L.weight.data(), L.weight.size() * sizeof(double));
        if (agg) std::memcpy(agg, L.agg.data(), L.agg.size() * sizeof(int));
        if (faceMap) std::memcpy(faceMap, L.faceMap.data(), L.faceMap.size() * sizeof(int));
        if (faceFlip)
            for (std::size_t k = 0; k < L.faceFlip.size(); ++k) faceFlip[k] = L.faceFlip[k];
        if (off) std::memcpy(off, L.off.data(), L.off.size() * sizeof(int));
        if (adjCell) std::memcpy(adjCell, L.adjCell.data(), L.adjCell.size() * sizeof(int));
        if (adjFace) std::memcpy(adjFace, L.adjFace.data(), L.adjFace.size() * sizeof(int));
        if (adjIsL)
            for (std::size_t k = 0; k < L.adjIsL.size(); ++k) adjIsL[k] = L.adjIsL[k];
    });
}

// Level-0 face map of the hierarchy: meshFace[k], ownerIsL[k] for k < nFaces(level 0).
int ref_gamg_meta(const RefMesh* r, int* meshFace, signed char* ownerIsL) {
    return guarded([&] {
        const auto& H = gamgHierarchy(*r->mesh);
        std::memcpy(meshFace, H.meshFace.data(), H.meshFace.size() * sizeof(int));
        for (std::size_t k = 0; k < H.ownerIsL.size(); ++k) ownerIsL[k] = H.ownerIsL[k];
    });
}

// One GAMG V-cycle w = M^-1 r with the reference's Gauss-Seidel smoother and LU coarse solve.
int ref_gamg_apply(const RefMesh* r, const double* diag, const double* upper, const double* lower, const double* rv,
                   double* w) {
    return guarded([&] {
        const Mesh& m = *r->mesh;
        const label n = m.nTotalCells();
        std::vector<scalar> d(diag, diag + n), b(n, 0.0), rr(rv, rv + n), ww(n, 0.0);
        LduSystem s{m, d, upper, lower ? lower : upper, b, lower == nullptr};
        GamgPreconditioner P(s);
        P.apply(rr, ww);
        std::memcpy(w, ww.data(), n * sizeof(double));
    });
}

// Boundary conditions for a scalar field: bcType[p] = 0 zeroGradient, 1 fixedValue (values
// from bcValues at the patch's boundary-face slots, indexed f - nInternalFaces).
static void setScalarBCs(const Mesh& m, VolField<scalar>& f, const int* bcType, const double* bcValues) {
    const label nI = m.nInternalFaces();
    for (std::size_t p = 0; p < m.patches().size(); ++p) {
        const Patch& pt = m.patches()[p];
        if (bcType[p] == 1) {
            auto& bc = f.set<FixedValueBC<scalar>>(pt.name, 0.0);
            for (label i = 0; i < pt.size; ++i) bc.values()[i] = bcValues ? bcValues[pt.start - nI + i] : 0.0;
        } else {
            f.set<ZeroGradientBC<scalar>>(pt.name);
        }
    }
    f.correctBoundaryConditions();
}

// fvm::laplacian(gamma, psi, nonOrthCorr) for a scalar field. gradScheme: 0 Gauss linear,
// 1 leastSquares (the mesh default the non-orthogonal correction uses).
// Outputs: diag[nCells], upper[nInternal], source[nCells], internalCoeffs[nBoundary],
// boundarySource[nBoundary], ffc[nFaces] (zeros when no correction); *hasFfc.
int ref_laplacian(const RefMesh* r, const double* gamma, const double* psi, const int* bcType,
                  const double* bcValues, int nonOrthCorr, int gradScheme, double* diag, double* upper,
                  double* source, double* internalCoeffs, double* boundarySource, double* ffc, int* hasFfc) {
    return guarded([&] {
        Mesh& m = *r->mesh;
        m.setGradScheme(gradScheme == 1 ? GradScheme::LeastSquares : GradScheme::GaussLinear);
        VolField<scalar> f(r->mesh, "p");
        for (label c = 0; c < m.nCells(); ++c) f[c] = psi[c];
        setScalarBCs(m, f, bcType, bcValues);
        std::vector<scalar> g(gamma, gamma + m.nFaces());
        FvMatrix<scalar> M = fvm::laplacian(g, f, nonOrthCorr != 0);
        const label nC = m.nCells(), nI = m.nInternalFaces(), nB = m.nBoundaryFaces();
        std::memcpy(diag, M.diag().data(), nC * sizeof(double));
        std::memcpy(upper, M.upper().data(), nI * sizeof(double));
        std::memcpy(source, M.source().data(), nC * sizeof(double));
        std::memcpy(internalCoeffs, M.internalCoeffs().data(), nB * sizeof(double));
        std::memcpy(boundarySource, M.boundarySource().data(), nB * sizeof(double));
        *hasFfc = M.hasFaceFluxCorrection() ? 1 : 0;
        if (M.hasFaceFluxCorrection())
            std::memcpy(ffc, M.faceFluxCorrection().data(), m.nFaces() * sizeof(double));
        else
            std::memset(ffc, 0, m.nFaces() * sizeof(double));
    });
}

// fvc::grad of a scalar field. scheme: 0 Gauss linear, 1 leastSquares. out: 3*nCells.
int ref_grad(const RefMesh* r, const double* psi, const int* bcType, const double* bcValues, int scheme, double* out) {
    return guarded([&] {
        Mesh& m = *r->mesh;
        VolField<scalar> f(r->mesh, "p");
        for (label c = 0; c < m.nCells(); ++c) f[c] = psi[c];
        setScalarBCs(m, f, bcType, bcValues);
        const auto g = fvc::grad(f, scheme == 1 ? GradScheme::LeastSquares : GradScheme::GaussLinear);
        for (label c = 0; c < m.nCells(); ++c) {
            out[3 * c] = g[c].x;
            out[3 * c + 1] = g[c].y;
            out[3 * c + 2] = g[c].z;
        }
    });
}

// Full pressure-equation assembly + solve as in projectDivergenceFree / the PISO corrector
// (solvers/IncompressibleFlow.cpp:62-71, :322-341): for no in 0..nNonOrth:
//   eqn = laplacian(gamma, p) ; eqn -= divPhi ; setReference(refCell, 0) ; eqn.solve(ctrl)
// p (nCells, in/out), divPhi per unit volume (nCells), flux out (nFaces) = eqn.flux() of the
// last pass. perfOut: 6 doubles per pass.
int ref_pressure_solve(const RefMesh* r, const double* gamma, const double* divPhi, int refCell, int nNonOrth,
                       int gradScheme, const char* solver, const char* precond, double tol, double relTol,
                       int maxIter, double* p, double* flux, double* perfOut) {
    return guarded([&] {
        Mesh& m = *r->mesh;
        m.setGradScheme(gradScheme == 1 ? GradScheme::LeastSquares : GradScheme::GaussLinear);
        VolField<scalar> f(r->mesh, "p");
        for (label c = 0; c < m.nCells(); ++c) f[c] = p[c];
        std::vector<int> zg(m.patches().size(), 0);
        setScalarBCs(m, f, zg.data(), nullptr);
        std::vector<scalar> g(gamma, gamma + m.nFaces()), dv(divPhi, divPhi + m.nCells());
        SolverControls c;
        c.solver = solver;
        c.preconditioner = precond;
        c.tolerance = tol;
        c.relTol = relTol;
        c.maxIter = maxIter;
        for (int no = 0; no <= nNonOrth; ++no) {
            FvMatrix<scalar> eqn = fvm::laplacian(g, f, true);
            eqn -= dv;
            if (refCell >= 0) eqn.setReference(refCell, 0.0);
            const auto perf = eqn.solve(c);
            perfOut[6 * no + 0] = perf[0].initialResidual;
            perfOut[6 * no + 1] = perf[0].finalResidual;
            perfOut[6 * no + 2] = perf[0].residualSum;
            perfOut[6 * no + 3] = perf[0].normFactor;
            perfOut[6 * no + 4] = perf[0].iterations;
            perfOut[6 * no + 5] = perf[0].converged ? 1.0 : 0.0;
            if (no == nNonOrth && flux) {
                const auto F = eqn.flux();
                std::memcpy(flux, F.data(), F.size() * sizeof(double));
            }
        }
        for (label c2 = 0; c2 < m.nCells(); ++c2) p[c2] = f[c2];
    });
}

double ref_exact_sum(const double* v, long n) {
    par::ExactSum s;
    for (long i = 0; i < n; ++i) s.add(v[i]);
    return s.value();
}

} // extern "C"
