// Device-resident incompressible step: IncompressibleFlow::step (solvers/IncompressibleFlow.cpp:138-370)
// for laminar flow on a mesh whose geometry is registered on the device.
//
// One step: momentum assembly (fvm::ddt + fvm::div(phi, U) - fvm::laplacian(nu, U), Fvm.h:18-182),
// implicit under-relaxation (FvMatrix::relax, FvMatrix.h:111-131), the momentum predictor (one
// PBiCGStab/DILU solve per solved component), then nCorr pressure corrections: A, H, HbyA, rAUf and
// the face flux phiHbyA (Rhie-Chow, IncompressibleFlow.cpp:244-292), the pressure equation with its
// non-orthogonal correctors (GAMG-PCG), phi = phiHbyA - flux, the explicit pressure relaxation
// (steady) and U = HbyA - rAU grad p.  Every array stays on the device; the host reads only the
// solver performance records and the step's residual figures.
//
// Every kernel restates one loop of the reference with its accumulation order (per cell: its faces
// in ascending face order; per boundary face: the order of the patch), so in CFD_REPRODUCIBLE mode
// (exact sums, diagonal preconditioning) a step reproduces the reference's fields bit for bit.
//
// Supported: steady SIMPLE and transient PIMPLE (Euler, backward), divergence schemes upwind /
// linear / linearUpwind / LUST / limitedLinear / vanLeer / MUSCL / minmod, Gauss linear gradients,
// fixedValue (uniform or face by face), zeroGradient, symmetry, freestream / freestreamPressure and
// fixedGradient boundary conditions for U and p, inletOutlet and pressureInletOutletVelocity for U,
// fixedFluxPressure and totalPressure for p, empty (2D) directions and
// cyclic (internal) faces, skewed meshes (the skew corrections of linear / LUST div, rAUf, the
// Rhie-Chow flux and the initial flux), the LES Smagorinsky model with Van Driest damping and
// constant / mean-velocity momentum forcing (flow_les.cu), Gauss or leastSquares mesh-default gradients
// and Gauss / leastSquares / GaussSkew pressure gradients.  Not supported: other turbulence models,
// wall models, buoyancy body forces, ddtPhiCoeff.
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "assembly.h"
#include "solver.h"
#include "voluma_b200.h"

namespace vlm {

class DeviceFlow {
public:
    // uType/pType: per patch 0 zeroGradient, 1 fixedValue; uValue 3 per patch, pValue 1 per patch.
    DeviceFlow(DeviceBatch& batch, DeviceGeom& geom, const vlm_flow_ctrl& ctrl, const int32_t* uType,
               const double* uValue, const int32_t* pType, const double* pValue, cudaStream_t stream);
    ~DeviceFlow();
    DeviceFlow(const DeviceFlow&) = delete;
    DeviceFlow& operator=(const DeviceFlow&) = delete;

    // IncompressibleFlow::initialize (IncompressibleFlow.cpp:32-40) from host fields (U: 3 per cell)
    void setState(const double* U, const double* p);
    // Per boundary face (index f - nInternal) values of the fixedValue / inletOutlet U faces (3 each,
    // AoS) and of the fixedValue p faces; NULL keeps the current values.
    void setBoundaryValues(const double* uFace, const double* pFace);
    // IncompressibleFlow::step(dt)
    vlm_step_info step(double dt);
    // fields to host (any pointer may be null)
    void getState(double* U, double* p, double* phi);
    // kernels run by this flow so far (its own, the geometry's and the solves', graph nodes included)
    int64_t launches() const { return total_; }
    // turbulence model and momentum forcing (flow_les.cu); before the first step
    void setModel(const vlm_flow_model& model);
    void modelState(double* nut, double* gradP);
    // restart::write / restart::read (io/Restart.cpp): the flow's state in the reference's restart
    // directory format; readRestart returns false when the directory has no state.txt
    void writeRestart(const std::string& dir);
    bool readRestart(const std::string& dir);

private:
    void boundaryU();
    void ioFractions();
    void totalPressure(bool noFlux);
    void boundaryP();
    void gradU();
    void assembleMomentum(double aU, bool haveGradU);
    // TurbulenceModel::correct for the LES model: wall shear, filter width, nu_t, face nu_eff
    void lesCorrect();
    // the explicit momentum sources after fvm::laplacian: div(nu_eff dev2(T(grad U))) and the forcing
    void explicitSources();
    // IncompressibleFlow::applyForcingCorrection (mean-velocity forcing)
    void forcingCorrection(double aU);
    void solveMomentum(vlm_step_info& info, bool first);
    void correctPressure(bool finalCorr, bool first, vlm_step_info& info);
    void stepWork(bool copyOld, bool copyOldOld);

    // captured steps: one graph per (steady, dt, dt0, old-time copies) configuration
    struct StepKey {
        bool steady;
        double dt, dt0;
        bool copyOld, copyOldOld;
        bool advShift, advShiftOldOld;
        double advC, advC0, advC00;
        bool operator==(const StepKey& o) const {
            return steady == o.steady && dt == o.dt && dt0 == o.dt0 && copyOld == o.copyOld &&
                   copyOldOld == o.copyOldOld && advShift == o.advShift && advShiftOldOld == o.advShiftOldOld &&
                   advC == o.advC && advC0 == o.advC0 && advC00 == o.advC00;
        }
    };
    struct StepGraph {
        StepKey key{};
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        int64_t ownLaunches = 0;
        int nSolves = 0, pSolve = -1;
        std::vector<int> uSolves;
        std::vector<DeviceBatch::LaunchCount> solveLaunches;
        std::vector<int> solveGroup;
        StepGraph() = default;
        StepGraph(const StepGraph&) = delete;
        StepGraph& operator=(const StepGraph&) = delete;
        ~StepGraph();
    };
    StepGraph* stepGraph(bool copyOld, bool copyOldOld);
    std::vector<std::unique_ptr<StepGraph>> stepGraphs_;
    bool graphOn_ = true;
    int64_t stepsRun_ = 0;
    void* pinned_ = nullptr;  // per-step read-back: continuity error, solver records, status words

    DeviceBatch& batch_;
    DeviceGeom& G_;
    vlm_flow_ctrl ctrl_;
    cudaStream_t s_;
    int nC_, nI_, nF_, nB_;
    bool needRef_ = false;
    std::vector<int32_t> uTypeHost_, pTypeHost_, pTypeAsm_;
    bool hasFluxPressure_ = false, hasTotalPressure_ = false;
    std::vector<int> solved_;
    DBuf<int32_t> uType_;
    DBuf<double> uValueB_, pValueB_;  // per boundary face: U values (SoA) / inlet values, p values
    DBuf<double> wIO_;                // mixed U value fraction per boundary face: inletOutlet (phi < 0 at
                                      // step start), freestream (constant)
    DBuf<double> pFrac_;              // freestreamPressure value fraction per boundary face
    DBuf<double> pTotal_;             // totalPressure p0 per boundary face
    DBuf<int32_t> uLsFix_, pLsFix_;   // per patch: the condition fixes the value (least-squares gradients)
    DBuf<int32_t> pType_;
    DBuf<int32_t> uFixesFlux_;        // per patch: the U condition fixes the flux (fixedValue, symmetry, Robin a != 0)
    std::vector<double> uRobinH_, pRobinH_;  // per patch {a, b} of Robin conditions (0 elsewhere)
    DBuf<double> uRobin_, pRobin_;
    // advective outflow (type 9): the condition keeps its own history of boundary values, advanced
    // when the time index changes (AdvectiveBC::update, VolField.h:235-264)
    bool hasAdvective_ = false;
    DBuf<double> advOld_, advOldOld_;  // boundary values at the old / old-old time levels (3 x nB)
    DBuf<double> uAdv_;                // per patch {lInf, fieldInf x, y, z}; lInf 0: no far field
    int advN_ = 0, advLastTI_ = -1;    // levels held (0..2) and the time index of the last shift
    struct AdvStep {
        bool on = false, shift = false, shiftOldOld = false, fromZero = false, noFlux = false;
        double c = 0, c0 = 0, c00 = 0;
    } adv_;
    // one update of the condition's state on the host (ddt: 0 steady, 1 Euler, 2 backward); the
    // launch that applies it is advectiveApply
    void advectiveAdvance(int ddt, bool fromZero, bool noFlux);
    void advectiveApply();
    bool hasInletOutlet_ = false;
    // fields (vectors SoA: component k at [k * n])
    DBuf<double> U_, Ub_, p_, pB_, phi_, U0_, U00_, phiOld_, phiOldOld_;
    // momentum matrix: UEqn (diag, upper, lower, source, internalCoeffs, boundarySource)
    DBuf<double> diag_, upper_, lower_, src_, ic_, bs_;
    // face terms of the operators and their per-cell sums
    DBuf<double> loDiv_, upDiv_, lapUp_, cDiv_, ffc_;
    // momentum predictor and pressure correction
    DBuf<double> gU_, gP_, msrc_, rAU_, HbyA_, rAUf_, phiHbyA_, divPhi_, pPrev_, fd_, fb_;
    DBuf<double> pdiag_, pupper_, psrc_, pic_, pbs_, pffc_, pflux_;
    DBuf<double> cont_;  // continuity error (max, as ordered bits)
    // skewed meshes: div skew correction, least-squares gradients of rAU / HbyA, HbyA boundary values
    DBuf<double> cSkew_, gR_, gH_, hB_;
    // solver records of the step's solves, read once at the end of the step
    DBuf<SysState> solveState_;
    DBuf<int> solveStatus_;
    int nSolves_ = 0;
    std::vector<int> uSolves_;  // record indices of the first outer pass's momentum solves
    int pSolve_ = -1;           // record index of the monitored pressure solve
    int solveSlot(bool momentum, bool monitoredP, int group = 1);
    std::vector<int> solveGroup_;  // per record: systems of the solve that wrote it (0: a later system's)
    // momentum components solved together: one batch of the mesh once per solved component
    bool componentBatch();
    std::unique_ptr<DeviceBatch> uBatch_;
    bool uBatchTried_ = false;
    DBuf<double> fdU_, fbU_, upU_, loU_, xU_;
    std::vector<DeviceBatch::LaunchCount> solveLaunches_;  // per record, set after its solve
    int64_t launches_ = 0, total_ = 0;
    // time state (Schemes.h TimeState) and the pressure-residual normalisation of the step
    double time_ = 0, dt_ = 1, dt0_ = -1;
    int timeIndex_ = 0, nOld_ = 0;
    double pNormRef_ = 0;
    int pNormSteps_ = 0;
    bool initialized_ = false;

    // turbulence model and forcing (flow_les.cu)
    bool les_ = false, vanDriest_ = false, exactSums_ = false;
    int forcing_ = 0, nWall_ = 0;
    double CsCs_ = 0, kOverC_ = 0, Aplus_ = 26, nutMax_ = 0;
    double force_[3] = {0, 0, 0}, Ubar_[3] = {0, 0, 0}, dir_[3] = {0, 0, 0};
    double magUbar_ = 0, relax_ = 1, totalVolume_ = 0;
    DBuf<int32_t> wallFace_, wallCell_, nearest_, wallB_;
    DBuf<double> wallN_, wallY_, uTau_, delta0_, yWall_, nut_, nuEffC_, nuF_, devF_;
    DBuf<double> forceState_;          // gradP, dU, rAUave
    DBuf<double> forcePart_;           // per-CTA partial sums (plain)
    DBuf<long long> forceBins_;        // per-CTA partial sums (exact)
    DBuf<unsigned long long> forceCount_;
};

}  // namespace vlm
