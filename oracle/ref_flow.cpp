// Test-infrastructure driver: the reference's own incompressible step (solvers/IncompressibleFlow.cpp,
// IncompressibleFlow::step) on a mesh built by ref_driver.cpp, with boundary conditions set through
// the reference's public VolField API the way CaseSetup.cpp:300-430 sets them (fixedValue/noSlip,
// zeroGradient) and the controls fvmFlow.cpp:141-178 derives from a case file.  It only marshals
// arrays and settings; every number comes from the unmodified reference.

#include "fvm/solvers/IncompressibleFlow.h"
#include "fvm/core/Json.h"
#include "fvm/io/Restart.h"
#include "fvm/models/TurbulenceModel.h"
#include "fvm/parallel/Comm.h"

#include <cstring>
#include <exception>
#include <iomanip>
#include <memory>
#include <sstream>
#include <string>

using namespace cfd;

struct RefMesh {
    MeshPtr mesh;
};

extern "C" {

// One linear-solver dictionary (SolverControls, LinearSolver.h:15-23).
struct RefSolverCtl {
    char solver[32];
    char preconditioner[32];
    double tolerance, relTol;
    int maxIter, minIter, nSweeps;
};

// Case settings: scheme codes follow Schemes.h (div: 0 upwind, 1 linear, 2 linearUpwind, 3 LUST,
// 4 limitedLinear divK, 5 vanLeer, 6 MUSCL, 7 minmod;
// ddt: 0 steadyState, 1 Euler, 2 backward); per patch (mesh patch order) U/p boundary type
// 0 zeroGradient, 1 fixedValue with the given value, 2 symmetry, 3 inletOutlet with the given inlet
// value (InletOutletBC on the flow's BCContext), 4 freestream (U: the free-stream velocity; p:
// freestreamPressure with the p value and the U free-stream velocity of the patch), 5 fixedGradient
// (the value is the gradient), 6 pressureInletOutletVelocity (U, the value is the tangential velocity)
// and fixedFluxPressure (p), 7 totalPressure (p, the value is p0), 8 Robin a phi + b dphi/dn = value
// with {a, b} per patch in uRobin / pRobin; uFace / pFace override the values face by face.
struct RefFlowSpec {
    double nu;
    int steady, divScheme, ddtScheme, nOuter, nCorr, nNonOrthCorr, momentumPredictor;
    double alphaU, alphaP;
    int nPatches;
    const int* uType;
    const double* uValue;  // 3 per patch
    const int* pType;
    const double* pValue;  // 1 per patch
    RefSolverCtl U, p, pFinal;
    int pRefCell;
    double pRefValue;
    int reproducible;
    double residualTol;  // > 0: stop once U and p residuals are below it (from step 2, fvmFlow.cpp:611-625)
    double divK;         // limitedLinear's k
    const double* uFace; // optional, 3 per boundary face: values of the fixedValue / inletOutlet U faces
    const double* pFace; // optional, 1 per boundary face: values of the fixedValue p faces
    int gradScheme;      // IncompressibleFlow::gradScheme and the mesh default: 0 Gauss, 1 leastSquares
    int gradPScheme;     // IncompressibleFlow::gradPScheme: 0 Gauss, 1 leastSquares, 2 GaussSkew
    const double* uRobin;  // optional, {a, b} per patch: Robin U patches
    const double* pRobin;  // optional, {a, b} per patch: Robin p patches
    const double* uAdv;    // optional, {lInf, fieldInf x, y, z} per patch: advective U patches
};

// Turbulence model and momentum forcing, as fvmFlow.cpp:182-194, 234 sets them from a case file:
// `turbulence` is the case's "turbulence" dictionary as JSON text (NULL: laminar); forcing 0 none,
// 1 constant (force), 2 meanVelocity (Ubar, relaxation; gradP is the initial driving gradient).
struct RefModelSpec {
    const char* turbulence;
    int forcing;
    double force[3], Ubar[3];
    double relaxation, gradP;
};

int ref_flow_run(const RefMesh* r, const RefFlowSpec* spec, int nSteps, double dt, double* U, double* p,
                 double* phi, double* hist, int* stepsRun);
// ref_flow_run_model that first continues from a restart directory (restart::read, when readDir is
// not NULL) and ends by writing one (restart::write, when writeDir is not NULL).
int ref_flow_run_restart(const RefMesh* r, const RefFlowSpec* spec, const RefModelSpec* model, const char* readDir,
                         const char* writeDir, int nSteps, double dt, double* U, double* p, double* phi, double* hist,
                         int* stepsRun, double* nut, double* gradP);
// ref_flow_run with a turbulence model / forcing; also returns nu_t per cell and the final gradP.
int ref_flow_run_model(const RefMesh* r, const RefFlowSpec* spec, const RefModelSpec* model, int nSteps, double dt,
                       double* U, double* p, double* phi, double* hist, int* stepsRun, double* nut, double* gradP);
const char* ref_flow_error();
}

namespace {
thread_local std::string g_flowErr;

SolverControls toCtl(const RefSolverCtl& c) {
    SolverControls s;
    s.solver = c.solver;
    s.preconditioner = c.preconditioner;
    s.tolerance = c.tolerance;
    s.relTol = c.relTol;
    s.maxIter = c.maxIter;
    s.minIter = c.minIter;
    s.nSweeps = c.nSweeps;
    return s;
}
}  // namespace

const char* ref_flow_error() { return g_flowErr.c_str(); }

namespace {
// Runs nSteps of IncompressibleFlow::step(dt) from the given U (3 per cell) and p (per cell).
// Outputs U, p, phi (nFaces) and per step hist[4*k..]: UInitialResidual, pInitialResidual,
// continuityError, total linear-solver iterations.
int runFlow(const RefMesh* r, const RefFlowSpec* sp, const RefModelSpec* model, int nSteps, double dt, double* U,
            double* p, double* phi, double* hist, int* stepsRun, double* nut, double* gradP,
            const char* readDir = nullptr, const char* writeDir = nullptr) {
    try {
        par::setReproducible(sp->reproducible != 0);
        const Mesh& m = *r->mesh;
        IncompressibleFlow flow(r->mesh, sp->nu);
        // gradient schemes as fvmFlow sets them (fvmFlow.cpp:151-154); the mesh default follows gradScheme
        flow.gradScheme = sp->gradScheme == 1 ? GradScheme::LeastSquares : GradScheme::GaussLinear;
        r->mesh->setGradScheme(flow.gradScheme);
        flow.gradPScheme = sp->gradPScheme == 1   ? GradScheme::LeastSquares
                           : sp->gradPScheme == 2 ? GradScheme::GaussSkew
                                                  : GradScheme::GaussLinear;
        PimpleControls& c = flow.controls;
        c.steady = sp->steady != 0;
        c.nOuter = sp->nOuter;
        c.nCorr = sp->nCorr;
        c.nNonOrthCorr = sp->nNonOrthCorr;
        c.momentumPredictor = sp->momentumPredictor != 0;
        c.alphaU = sp->alphaU;
        c.alphaP = sp->alphaP;
        c.UControls = toCtl(sp->U);
        c.pControls = toCtl(sp->p);
        c.pFinalControls = toCtl(sp->pFinal);
        c.pRefCell = sp->pRefCell;
        c.pRefValue = sp->pRefValue;
        static const char* div[8] = {"upwind", "linear",  "linearUpwind", "LUST",
                                     "limitedLinear", "vanLeer", "MUSCL", "minmod"};
        if (sp->divScheme < 0 || sp->divScheme > 7) throw std::runtime_error("unknown divergence scheme code");
        std::string scheme = div[sp->divScheme];
        if (sp->divScheme == 4) {
            std::ostringstream os;
            os << std::setprecision(17) << scheme << ' ' << sp->divK;
            scheme = os.str();
        }
        flow.divScheme = ConvectionScheme::parse(scheme);
        flow.ddtScheme = sp->ddtScheme == 0 ? DdtScheme::Steady : sp->ddtScheme == 1 ? DdtScheme::Euler
                                                                                      : DdtScheme::Backward;
        if (sp->nPatches != int(m.patches().size())) throw std::runtime_error("patch count mismatch");
        const label nI = m.nInternalFaces();
        for (int q = 0; q < sp->nPatches; ++q) {
            const std::string name = m.patches()[q].name;
            if (m.patches()[q].type == PatchType::Empty || m.patches()[q].type == PatchType::Cyclic) continue;
            const label start = m.patches()[q].start, size = m.patches()[q].size;
            const Vec3 uv{sp->uValue[3 * q], sp->uValue[3 * q + 1], sp->uValue[3 * q + 2]};
            auto uFace = [&](label i) {
                const double* v = sp->uFace + 3 * (start - nI + i);
                return Vec3{v[0], v[1], v[2]};
            };
            if (sp->uType[q] == 1) {
                auto& bc = flow.U().set<FixedValueBC<Vec3>>(name, uv);
                if (sp->uFace)
                    for (label i = 0; i < size; ++i) bc.values()[i] = uFace(i);
            } else if (sp->uType[q] == 2) {
                flow.U().set<SymmetryBC<Vec3>>(name);
            } else if (sp->uType[q] == 3) {
                auto& bc = flow.U().set<InletOutletBC<Vec3>>(name, &flow.context(), uv);
                if (sp->uFace)
                    for (label i = 0; i < size; ++i) bc.refValue()[i] = uFace(i);
            } else if (sp->uType[q] == 4) {
                flow.U().set<FreestreamVelocityBC>(name, uv);
            } else if (sp->uType[q] == 5) {
                flow.U().set<FixedGradientBC<Vec3>>(name, uv);
            } else if (sp->uType[q] == 6) {
                flow.U().set<PressureInletOutletVelocityBC>(name, &flow.context(), uv);
            } else if (sp->uType[q] == 8) {
                flow.U().set<RobinBC<Vec3>>(name, sp->uRobin[2 * q], sp->uRobin[2 * q + 1], uv);
            } else if (sp->uType[q] == 9) {
                const double* a = sp->uAdv ? sp->uAdv + 4 * q : nullptr;
                const bool inf = a && a[0] > 0;
                flow.U().set<AdvectiveBC<Vec3>>(name, &flow.context(), inf, inf ? Vec3{a[1], a[2], a[3]} : Vec3{},
                                                inf ? a[0] : 0.0);
            } else {
                flow.U().zeroGradient(name);
            }
            if (sp->pType[q] == 1) {
                auto& bc = flow.p().set<FixedValueBC<scalar>>(name, sp->pValue[q]);
                if (sp->pFace)
                    for (label i = 0; i < size; ++i) bc.values()[i] = sp->pFace[start - nI + i];
            } else if (sp->pType[q] == 2) {
                flow.p().set<SymmetryBC<scalar>>(name);
            } else if (sp->pType[q] == 3) {
                flow.p().set<InletOutletBC<scalar>>(name, &flow.context(), sp->pValue[q]);
            } else if (sp->pType[q] == 4) {
                flow.p().set<FreestreamPressureBC>(name, &flow.context(), sp->pValue[q], &uv);
            } else if (sp->pType[q] == 5) {
                flow.p().set<FixedGradientBC<scalar>>(name, sp->pValue[q]);
            } else if (sp->pType[q] == 6) {
                flow.p().set<FixedFluxPressureBC>(name);
            } else if (sp->pType[q] == 7) {
                const double p0 = sp->pValue[q];
                flow.p().set<TotalPressureBC>(name, &flow.context(), [p0](scalar) { return p0; });
            } else if (sp->pType[q] == 8) {
                flow.p().set<RobinBC<scalar>>(name, sp->pRobin[2 * q], sp->pRobin[2 * q + 1], sp->pValue[q]);
            } else {
                flow.p().zeroGradient(name);
            }
        }
        // the turbulence model keeps references to its dictionaries: they live as long as the run
        const Json empty = Json::parse("{}");
        const Json turb = Json::parse(model && model->turbulence ? model->turbulence : "{}");
        std::unique_ptr<TurbulenceModel> tm;
        if (model && model->turbulence) tm = TurbulenceModel::create(flow, turb, empty, empty);
        if (model && model->forcing == 1) {
            flow.forcing.mode = MomentumForcing::Mode::Constant;
            flow.forcing.force = Vec3{model->force[0], model->force[1], model->force[2]};
        } else if (model && model->forcing == 2) {
            flow.forcing.mode = MomentumForcing::Mode::MeanVelocity;
            flow.forcing.Ubar = Vec3{model->Ubar[0], model->Ubar[1], model->Ubar[2]};
            flow.forcing.relaxation = model->relaxation;
            flow.forcing.gradP = model->gradP;
        }
        const label nC = m.nCells();
        for (label k = 0; k < nC; ++k) {
            flow.U()[k] = Vec3{U[3 * k], U[3 * k + 1], U[3 * k + 2]};
            flow.p()[k] = p[k];
        }
        if (readDir && !restart::read(readDir, flow)) throw std::runtime_error("no restart state in " + std::string(readDir));
        int s = 0;
        for (s = 0; s < nSteps; ++s) {
            const StepInfo info = flow.step(dt);
            double its = 0;
            for (const auto& pf : info.perf) its += pf.iterations;
            if (hist) {
                hist[4 * s] = info.UInitialResidual;
                hist[4 * s + 1] = info.pInitialResidual;
                hist[4 * s + 2] = info.continuityError;
                hist[4 * s + 3] = its;
            }
            if (sp->residualTol > 0 && s > 0 && info.UInitialResidual < sp->residualTol &&
                info.pInitialResidual < sp->residualTol) {
                ++s;
                break;
            }
        }
        if (stepsRun) *stepsRun = s;
        if (writeDir) restart::write(writeDir, flow);
        for (label k = 0; k < nC; ++k) {
            U[3 * k] = flow.U()[k].x;
            U[3 * k + 1] = flow.U()[k].y;
            U[3 * k + 2] = flow.U()[k].z;
            p[k] = flow.p()[k];
        }
        if (phi)
            for (label f = 0; f < m.nFaces(); ++f) phi[f] = flow.phi()[f];
        if (nut)
            for (label k = 0; k < nC; ++k) nut[k] = flow.nut().empty() ? 0.0 : flow.nut()[k];
        if (gradP) *gradP = flow.forcing.gradP;
        par::setReproducible(false);
        return 0;
    } catch (const std::exception& e) {
        g_flowErr = e.what();
        par::setReproducible(false);
        return 1;
    }
}
}  // namespace

int ref_flow_run(const RefMesh* r, const RefFlowSpec* sp, int nSteps, double dt, double* U, double* p, double* phi,
                 double* hist, int* stepsRun) {
    return runFlow(r, sp, nullptr, nSteps, dt, U, p, phi, hist, stepsRun, nullptr, nullptr);
}

int ref_flow_run_model(const RefMesh* r, const RefFlowSpec* sp, const RefModelSpec* model, int nSteps, double dt,
                       double* U, double* p, double* phi, double* hist, int* stepsRun, double* nut, double* gradP) {
    return runFlow(r, sp, model, nSteps, dt, U, p, phi, hist, stepsRun, nut, gradP);
}

int ref_flow_run_restart(const RefMesh* r, const RefFlowSpec* sp, const RefModelSpec* model, const char* readDir,
                         const char* writeDir, int nSteps, double dt, double* U, double* p, double* phi, double* hist,
                         int* stepsRun, double* nut, double* gradP) {
    return runFlow(r, sp, model, nSteps, dt, U, p, phi, hist, stepsRun, nut, gradP, readDir, writeDir);
}
