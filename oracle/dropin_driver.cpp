// Drop-in check (test infrastructure): the reference's UNMODIFIED FvMatrix / fvm::laplacian code
// with its call to cfd::solveLdu redirected, at link time (ld --wrap), to the GPU solver through
// include/voluma_b200_ldu.hpp.  Built by oracle/Makefile into oracle/_ref/libvlmdropin.so from
// the reference sources + this file + voluma_b200/_lib/libvoluma_b200.so.
//
// dropin_pressure_solve runs the reference's projectDivergenceFree-style pressure loop
// (solvers/IncompressibleFlow.cpp:62-71: laplacian, -= divPhi, setReference, FvMatrix::solve)
// entirely in reference code; only the linear solve runs on the device.
#include "fvm/discretization/Fvm.h"
#include "fvm/linalg/LinearSolver.h"
#include "fvm/mesh/Mesh.h"
#include "fvm/mesh/RawMesh.h"
#include "fvm/parallel/Comm.h"
#include "voluma_b200_ldu.hpp"

#include <cstring>
#include <string>

using namespace cfd;

namespace {
thread_local std::string g_err;
thread_local std::string g_smoother, g_precision;
thread_local int g_calls = 0;
}  // namespace

// Every call the reference makes to solveLdu lands here.
extern "C" SolverPerformance __wrap__ZN3cfd8solveLduERKNS_9LduSystemERSt6vectorIdSaIdEERKNS_14SolverControlsE(
    const LduSystem& s, std::vector<scalar>& x, const SolverControls& c) {
    ++g_calls;
    return vlm_dropin::solveLdu<SolverPerformance>(s, x, c, par::reproducible(), g_smoother, g_precision);
}

extern "C" {

const char* dropin_last_error() { return g_err.c_str(); }
int dropin_calls() { return g_calls; }

// Same inputs as ref_pressure_solve in ref_driver.cpp; perfOut: 6 doubles per pass.
int dropin_pressure_solve(const int* n, const double* lo, const double* hi, const int* periodic, const double* points,
                          const double* gamma, const double* divPhi, int refCell, int nNonOrth, int gradScheme,
                          const char* solver, const char* precond, double tol, double relTol, int maxIter,
                          int reproducible, const char* smoother, const char* precision, double* p, double* flux,
                          double* perfOut) {
    try {
        g_smoother = smoother ? smoother : "";
        g_precision = precision ? precision : "";
        BoxSpec spec;
        for (int d = 0; d < 3; ++d) {
            spec.n[d] = n[d];
            spec.lo[d] = lo[d];
            spec.hi[d] = hi[d];
            spec.periodic[d] = periodic[d] != 0;
        }
        RawMesh raw = generateBox(spec);
        if (points)
            for (std::size_t q = 0; q < raw.points.size(); ++q)
                raw.points[q] = Vec3{points[3 * q], points[3 * q + 1], points[3 * q + 2]};
        MeshPtr mesh = Mesh::build(&raw);
        mesh->setGradScheme(gradScheme == 1 ? GradScheme::LeastSquares : GradScheme::GaussLinear);
        VolField<scalar> f(mesh, "p");
        for (label c = 0; c < mesh->nCells(); ++c) f[c] = p[c];
        for (const Patch& pt : mesh->patches()) f.set<ZeroGradientBC<scalar>>(pt.name);
        f.correctBoundaryConditions();
        std::vector<scalar> g(gamma, gamma + mesh->nFaces()), dv(divPhi, divPhi + mesh->nCells());
        SolverControls ctrl;
        ctrl.solver = solver;
        ctrl.preconditioner = precond;
        ctrl.tolerance = tol;
        ctrl.relTol = relTol;
        ctrl.maxIter = maxIter;
        par::setReproducible(reproducible != 0);
        for (int no = 0; no <= nNonOrth; ++no) {
            FvMatrix<scalar> eqn = fvm::laplacian(g, f, true);
            eqn -= dv;
            if (refCell >= 0) eqn.setReference(refCell, 0.0);
            const auto perf = eqn.solve(ctrl);
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
        par::setReproducible(false);
        for (label c = 0; c < mesh->nCells(); ++c) p[c] = f[c];
        return 0;
    } catch (const std::exception& e) {
        par::setReproducible(false);
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
