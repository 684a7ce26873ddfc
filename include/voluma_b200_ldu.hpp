// voluma_b200_ldu.hpp — header-only C++ drop-in for the reference's linear-solver seam.
//
// Replaces   SolverPerformance cfd::solveLdu(const LduSystem&, std::vector<scalar>& x,
//                                            const SolverControls&)   (src/fvm/linalg/LinearSolver.h:42)
// with the same contract on one GPU, through the C ABI of voluma_b200.h.  It is written against
// the reference's public member names only (templates, no reference header included here):
//   LduSystem   {mesh, diag, upper, lower, b, symmetric}            (LinearSolver.h:33-40)
//   Mesh        nCells(), nTotalCells(), nInternalFaces(), owner(), neighbour(), magSf(),
//               nonOrthDeltaCoeffs(), cached<T>(key, build)         (src/fvm/mesh/Mesh.h:54-122)
//   SolverControls / SolverPerformance fields                        (LinearSolver.h:15-31)
// The device copy of a mesh (addressing + GAMG hierarchy) is cached on the Mesh itself, like
// the reference caches its own GAMG hierarchy (GAMG.cpp:204), and released with it.
// Errors are rethrown as std::runtime_error with the library's message, as the reference does
// for unknown solvers / preconditioners, PCG on an asymmetric matrix and a singular coarsest
// GAMG matrix (LinearSolver.cpp:76,177,280; GAMG.cpp:336).
#pragma once

#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "voluma_b200.h"

namespace vlm_dropin {

// One context per host thread (the reference solver is single-threaded per rank).
inline vlm_ctx* context() {
    struct Holder {
        vlm_ctx* ctx = nullptr;
        Holder() {
            if (vlm_ctx_create(0, &ctx) != VLM_OK) throw std::runtime_error(vlm_last_error(nullptr));
        }
        ~Holder() { vlm_ctx_destroy(ctx); }
    };
    thread_local Holder h;
    return h.ctx;
}

// Device mesh owned by the reference Mesh's cache.
struct DeviceMesh {
    vlm_mesh* mesh = nullptr;
    DeviceMesh() = default;
    DeviceMesh(const DeviceMesh&) = delete;
    DeviceMesh& operator=(const DeviceMesh&) = delete;
    DeviceMesh(DeviceMesh&& o) noexcept : mesh(o.mesh) { o.mesh = nullptr; }
    ~DeviceMesh() { vlm_mesh_release(mesh); }
};

template <class Mesh>
vlm_mesh* deviceMesh(const Mesh& m) {
    const DeviceMesh& dm = m.template cached<DeviceMesh>("voluma_b200", [&] {
        if (m.nTotalCells() != m.nCells())
            throw std::runtime_error("voluma_b200: halo (MPI-decomposed) meshes are not supported on the device");
        vlm_mesh_desc d;
        std::memset(&d, 0, sizeof d);
        d.n_cells = m.nCells();
        d.n_internal_faces = m.nInternalFaces();
        d.n_faces = int32_t(m.owner().size());
        d.owner = m.owner().data();
        d.neighbour = m.neighbour().data();
        d.magSf = m.magSf().data();
        d.ndc = m.nonOrthDeltaCoeffs().data();
        DeviceMesh out;
        if (vlm_mesh_register(context(), &d, 0, &out.mesh) != VLM_OK)
            throw std::runtime_error(vlm_last_error(context()));
        return out;
    });
    return dm.mesh;
}

inline void copyName(char* dst, size_t n, const std::string& s) {
    std::memset(dst, 0, n);
    std::strncpy(dst, s.c_str(), n - 1);
}

// solveLdu on the GPU.  `reproducible` carries par::reproducible() (CFD_REPRODUCIBLE): the
// device then applies the same preconditioner / smoother swap and exact sums.  `smoother` and
// `precision` are the additive dictionary keys ("" = defaults).
template <class Perf, class LduSystem, class Controls>
Perf solveLdu(const LduSystem& s, std::vector<double>& x, const Controls& c, bool reproducible = false,
              const std::string& smoother = "", const std::string& precision = "") {
    vlm_mesh* mesh = deviceMesh(s.mesh);
    vlm_solver_ctrl ctrl;
    std::memset(&ctrl, 0, sizeof ctrl);
    copyName(ctrl.solver, sizeof ctrl.solver, c.solver);
    copyName(ctrl.preconditioner, sizeof ctrl.preconditioner, c.preconditioner);
    copyName(ctrl.smoother, sizeof ctrl.smoother, smoother);
    copyName(ctrl.precision, sizeof ctrl.precision, precision);
    ctrl.tolerance = c.tolerance;
    ctrl.relTol = c.relTol;
    ctrl.maxIter = c.maxIter;
    ctrl.minIter = c.minIter;
    ctrl.nSweeps = c.nSweeps;
    ctrl.reproducible = reproducible ? 1 : 0;
    vlm_solver_perf p;
    const vlm_status st = vlm_ldu_solve(context(), mesh, s.diag.data(), s.upper, s.symmetric ? nullptr : s.lower,
                                        s.b.data(), x.data(), &ctrl, &p);
    if (st != VLM_OK) throw std::runtime_error(vlm_last_error(context()));
    Perf out;
    out.solver = c.solver;
    out.initialResidual = p.initialResidual;
    out.finalResidual = p.finalResidual;
    out.residualSum = p.residualSum;
    out.normFactor = p.normFactor;
    out.iterations = p.iterations;
    out.converged = p.converged != 0;
    return out;
}

}  // namespace vlm_dropin
