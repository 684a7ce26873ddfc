// Device-resident batch of LDU systems with GAMG hierarchies, and the solve drivers.
#pragma once

#include <map>
#include <tuple>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "devtypes.h"
#include "plan.h"

namespace vlm {

struct ChunkList {
    int off = 0, n = 0;
};

struct DevLevel {
    bool blockGS = false;
    int nrows = 0, nfaces = 0, nActiveRows = 0, nSteps = 0, nent = 0, maxColours = 0;
    ChunkList blocks;
    DBuf<int8_t> rowColour;
    DBuf<int32_t> slPtr, rlen, col, src;
    DBuf<Chunk> chunks;
    std::vector<Chunk> hostChunks;  // host copy of `chunks`
    ChunkList active, all;
    ChunkList headActive, headIn;  // coarse-tail mode: rows above each system's tail / restricted into
    std::vector<ChunkList> headFwd, headRev;  // coarse-tail mode: colour steps of the systems above the tail
    std::vector<ChunkList> fwd, rev;
    DBuf<int32_t> agg, childPtr, child, intraPtr, intraFace, cfacePtr, cfaceSrc;
    ChunkList coarse;  // CoarseDev entries whose coarsest level is this one
    // level 0 of box meshes (box.h): the face of each row's +x/+y/+z neighbour, and the
    // per-direction coefficients materialised from it per solve
    bool box = false;
    DBuf<int32_t> boxFace;
    DBuf<double> bcoef;
    DBuf<float> bcoef32;
    // numeric, per solve
    DBuf<double> diag, val, up, lo;
    DBuf<float> diag32, val32;
    // V-cycle vectors
    DBuf<double> r, x, t, x2;
    DBuf<float> r32, x32, t32, x232;
    Sell sell() const { return Sell{slPtr.get(), rlen.get(), col.get()}; }
    const Chunk* ch(const ChunkList& l) const { return chunks.get() + l.off; }
};

enum class SolverKind { PCG, PBiCGStab, Jacobi, GaussSeidel, SymGaussSeidel };
enum class PrecondKind { None, Diagonal, GAMG, DIC, DILU };
// MCGS: level-0 multicolour GS (block-hybrid GS where it needs many colours) + block-hybrid GS on
// coarser levels; MCGSJacobi: the same level 0 + Jacobi on coarser levels; Jacobi: every level.
enum class SmootherKind { MCGS, MCGSJacobi, Jacobi };
// FP64; FP64 Krylov recurrence with an FP32 GAMG V-cycle; FP32 inner PCG in FP64 defect correction
enum class Precision { FP64, MixedPrecond, MixedDC };

struct SolveKey {
    SolverKind solver;
    PrecondKind precond;
    SmootherKind smoother;
    Precision prec;
    bool exact;
    int nSweeps;  // relaxation solvers: sweeps per residual evaluation (0 for Krylov solvers)
    bool box;     // level 0 runs the box kernels (box mesh, symmetric matrix)
    bool operator<(const SolveKey& o) const {
        return std::tie(solver, precond, smoother, prec, exact, nSweeps, box) <
               std::tie(o.solver, o.precond, o.smoother, o.prec, o.exact, o.nSweeps, o.box);
    }
};

struct DiluDev;  // device copy of the DIC/DILU / Gauss-Seidel level schedule (solver.cu)

struct GraphExec {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int64_t preK = 0, bodyK = 0, innerK = 0;  // kernels per captured segment
    ~GraphExec();
};

// A batch of systems resident on one device (a single-system mesh is a batch of one).
class DeviceBatch {
public:
    // deviceAgglomeration: the GAMG hierarchy from the device's parallel matching (aggl.h) instead
    // of the host's sequential pass
    DeviceBatch(const std::vector<SysTopo>& systems, int mergeLevels, cudaStream_t stream,
                bool deviceAgglomeration = false);
    ~DeviceBatch();

    const BatchPlan& plan() const { return plan_; }
    int nLevels() const { return int(L_.size()); }
    const DevLevel& level(int k) const { return L_[k]; }
    int64_t userCells() const { return plan_.userCells; }
    int64_t userFaces() const { return plan_.userFaces; }

    // Coefficients: device pointers to user-layout (concatenated, input order) arrays.
    // lower == upper for symmetric systems.
    void setupMatrix(const double* diag, const double* upper, const double* lower, bool gamg, bool mixed);

    // Full solve on device pointers (user layout). perfOut: one per input system (input order).
    void solve(const double* diag, const double* upper, const double* lower, const double* b, double* x,
               const vlm_solver_ctrl& ctrl, std::vector<vlm_solver_perf>& perfOut);

    // The next solve() only enqueues its work: its final solver state (one SysState per system) and
    // its status words (coarsest-matrix status, level-schedule barrier status) are copied, on the
    // stream, to these device locations, and solve() returns without waiting or filling perfOut.
    void deferNextSolve(SysState* stateOut, int* statusOut) {
        deferState_ = stateOut;
        deferStatus_ = statusOut;
    }
    // Clears a level-schedule barrier error left by a deferred solve.
    void clearLevelError();
    // Launch counts of the last deferred solve: kernels launched directly, and (graph mode) the
    // kernel nodes of the loop's entry and of one loop pass; launches = eager + pre + its * body.
    struct LaunchCount {
        int64_t eager = 0, pre = 0, body = 0;
    };
    LaunchCount lastDeferred() const { return lastDeferred_; }

    // y = A x (user layout device pointers)
    void amul(const double* diag, const double* upper, const double* lower, const double* x, double* y);

    // One V-cycle w = M^-1 r (user layout device pointers)
    void gamgApply(const double* diag, const double* upper, const double* lower, const double* r, double* w,
                   SmootherKind sm);

    // w = M^-1 r for the preconditioner named in ctrl (user layout device pointers)
    void precondApply(const double* diag, const double* upper, const double* lower, const double* r, double* w,
                      const vlm_solver_ctrl& ctrl);

    cudaStream_t stream() const { return stream_; }
    // While the caller captures the batch's stream into its own graph, solve() adds its iteration loop
    // to that graph (a conditional WHILE node whose body is captured on a side stream) instead of
    // launching the solve's graph.  Only valid after every solve key has run once outside a capture.
    void beginEmbedding();
    void endEmbedding();
    // Whether solves can be embedded in a captured graph (graph mode, no cooperative launches).
    bool embeddable() const;
    // Whether a solve with these controls keeps every system's level-scheduled sweeps (DIC / DILU /
    // Gauss-Seidel) in one CTA each (builds the level schedule on first use); true without them.
    bool levelScheduleInSharedMemory(const vlm_solver_ctrl& ctrl);
    const std::vector<SysTopo>& topology() const { return topo_; }
    int mergeLevels() const { return mergeLevels_; }
    size_t deviceBytes() const;
    // Coarse-tail configuration (tuning): cluster size 1/2/4/8, level row limit, whole-V-cycle row
    // limit (0 keeps a value); re-plans the batch's launches, same results.
    void setTail(int cluster, int64_t maxRows, int64_t fullRows);
    void setFusion(int64_t pre, int64_t restrict, int64_t post);
    // The next solve() reads b and x only after `ev` (their upload on another stream), so the
    // upload overlaps the matrix set-up.
    void inputsAfter(cudaEvent_t ev) { inputsReady_ = ev; }
    void streamConfig(int32_t* ty, int32_t* stages, int32_t* ctas) const {
        *ty = stream64_.grid > 0 ? stream64_.TY : 0;
        *stages = stream64_.grid > 0 ? stream64_.S : 0;
        *ctas = stream64_.grid;
    }
    void fusionConfig(int64_t* pre, int64_t* restrict, int64_t* post) const {
        *pre = fusePre_;
        *restrict = fuseRestrict_;
        *post = fusePost_;
    }
    void tailConfig(int* cluster, int64_t* maxRows, int64_t* fullRows) const {
        *cluster = tailCl_;
        *maxRows = tailMaxRows_;
        *fullRows = tailFullRows_;
    }
    int64_t launches() const { return launches_; }
    void countLaunches(int64_t n) { launches_ += n; }  // kernels of deferred solves, counted by the caller
    // Times `reps` back-to-back launches of one level-0 kernel on the current matrix (after a
    // solve); returns ms per launch and the algorithmic bytes one launch moves.
    double profileKernel(const std::string& name, int reps, double* bytesPerLaunch);
    // fused two-colour level-0 sweep (k_box_sweep4): ticket counters and per-piece done stamps.
    // Off by default: at 128^3 one fused launch measured 33 us per sweep against 17 us for the two
    // colour launches (each CTA serialises ticket, dependency wait and fence per piece)
    bool sweepFused_ = false;
    int sweepGrid_ = 0;
    DBuf<SweepSync> sweepSync_;
    DBuf<unsigned> sweepDone_;
    template <class T>
    bool recordFusedSweep(const ChunkList& la, const ChunkList& lb, const T* r, T* x, bool pre, int sweep,
                          const int32_t* agg, const T* xc);
    void checkSweepError();
    // streamed level-0 kernels (boxstream.cuh): launch shape per element size, planned once
    struct StreamShape {
        int TY = 0, S = 0, threads = 0, grid = 0;  // grid 0: the kernels do not apply
        size_t smem = 0;
    };
    StreamShape stream64_, stream32_;
    bool streamAllowed_ = true;
    cudaEvent_t inputsReady_ = nullptr;
    template <class T> void planStream(const BoxRows& R);
    template <class T> const StreamShape* streamShape(const BoxRows& R) const;
    // live timing of the level-0 sweeps: solves run eagerly with CUDA events around every level-0
    // sweep (setSweepTiming); the stream's own order, so each sweep meets the cache state the solve
    // leaves it
    bool timeSweeps_ = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> sweepEvents_;
    double sweepMs_ = 0.0;
    int64_t sweepCount_ = 0;
    void collectSweepTimes();

public:
    void setSweepTiming(bool on);
    void sweepTiming(double* msTotal, int64_t* count) const {
        *msTotal = sweepMs_;
        *count = sweepCount_;
    }

private:
    DBuf<int4> flush_;       // profileKernel's L2-evicting read buffer (allocated on first use)
    DBuf<int> flushSink_;


private:
    template <class T> void recordVcycle(const T* r0, T* x0, SmootherKind sm, int flag, bool allowTail = true);
    template <class T> void recordSmooth(int k, const T* r, T* x, SmootherKind sm, bool pre, int flag, bool head);
    template <class T> void recordTail(const T* r0, T* x0, int flag, bool jacobi0);
    template <class T> void buildTailTable(DBuf<TailLevel<T>>& out);
    void planTail();
    void buildChunkLists();
    void ensureDilu();
    void recordDiluApply(const double* r, double* w);
    void diluFactor(const double* upper, const double* lower);
    void checkLevelError();
    void recordRelaxIter(const SolveKey& key);
    template <bool EXACT> void recordRelaxIterT(const SolveKey& key);
    void recordPrecond(PrecondKind pk, SmootherKind sm, const double* r, double* w, bool f32);
    void recordIter(const SolveKey& key);
    void runEager(const SolveKey& key, int maxIter);
    void recordPcgIter(PrecondKind pk, SmootherKind sm, bool f32);
    void recordInnerPcgIter(PrecondKind pk, SmootherKind sm);
    void recordBicgIter(PrecondKind pk, SmootherKind sm, bool f32);
    template <bool EXACT> void recordPcgIterT(PrecondKind pk, SmootherKind sm, bool f32);
    template <bool EXACT> void recordBicgIterT(PrecondKind pk, SmootherKind sm, bool f32);
    void recordSetCond(cudaGraphConditionalHandle h, int flag);
    void embedSolve(const SolveKey& key);
    GraphExec& graphFor(const SolveKey& key);
    void buildGraph(const SolveKey& key, GraphExec& g);
    void ensureVectors(bool mixed, bool bicg);
    RedCtx red() const;
    BoxRows boxRows(const DevLevel& D, const ChunkList& l, int* grid) const;

    BatchPlan plan_;
    std::vector<DevLevel> L_;
    cudaStream_t stream_;
    DBuf<CoarseDev> coarse_;
    DBuf<double> lu_, inv_;
    DBuf<int32_t> perm0_, sysCells_, slotBegin_, slotEnd_, counters_, status_;
    DBuf<BoxSys> boxes_;     // per batch position, when level 0 has the box layout
    bool boxOn_ = false;     // the current solve's matrix uses the box kernels on level 0
    DBuf<DD> partials_;
    DBuf<long long> xbins_;  // exact-sum partials (reproducible mode)
    bool exact_ = false;
    DBuf<SysState> st_;
    DBuf<DevCtrl> dctrl_;
    DBuf<int> anyActive_;
    // Krylov vectors, level-0 solver order
    DBuf<double> x_, b_, r_, w_, p_, Ap_, rD_, r0_, y_, Ay_, s_, z_, t_;
    DBuf<float> e32_, r32_, w32_, p32_, Ap32_, rD32_;
    DBuf<float> dL32_;  // defect correction: FP32 diagonal of the inner operator (reference row's refC removed)
    void recordRefSetup();   // reference row, inner diagonal, inner right-hand side (mixed-dc)
    void recordMixedTail();  // outer correction, FP64 defect, next inner right-hand side (mixed-dc)
    std::map<SolveKey, std::unique_ptr<GraphExec>> graphs_;
    std::vector<SysState> hostState_;
    double jacobiOmega_ = 1.0;
    // coarse tail: levels tailFirst_[b].. of system b run in one CTA (Jacobi coarse levels)
    bool tailOn_ = false;
    int tailMaxFirst_ = 0;      // head levels: k < tailMaxFirst_
    std::vector<int> tailFirst_;
    DBuf<TailSys> tailSys_;
    // shared-memory tail (k_vcycle_tail_smem): used when every tail system's levels fit
    bool tailSmem_ = false, tailSmemAllowed_ = true;
    DBuf<TailImg> tailImg_;
    DBuf<int32_t> tailCodes_;            // value-image gather codes (k_tail_values)
    DBuf<uint16_t> tailStr_;             // structure images
    DBuf<double> tailVal64_;
    DBuf<float> tailVal32_;
    size_t tailSmem64_ = 0, tailSmem32_ = 0;  // dynamic shared memory per CTA
    void planTailSmem(const std::vector<TailSys>& ts);
    int tailCl_ = 1;                     // CTAs of the cluster that runs one system's tail (the tuner may widen it)
    int64_t tailMaxRows_ = 0;            // levels of at most this many rows go to the tail (0: scaled default)
    int64_t tailFullRows_ = 0;           // systems of at most this many level-0 rows: whole V-cycle there
    // fused coarse-level launches on levels of at most this many rows (all systems): both Jacobi
    // pre-sweeps in one pass, residual with restriction, prolongation inside the first post-sweep.
    // Off by default: at 128^3 each fusion measured slower than its separate launches (inside the
    // captured graph a launch costs less than the longer dependent-load chain of the fused kernel).
    int64_t fusePre_ = 0, fuseRestrict_ = 0, fusePost_ = 0;
    bool fusedLevel(int k, int64_t limit) const { return int64_t(L_[k].nrows) <= limit; }
    std::vector<SysTopo> topo_;          // host topology (owned by the caller for the batch's lifetime)
    int mergeLevels_ = 2;
    std::unique_ptr<DiluDev> dilu_;      // built on the first DIC/DILU/Gauss-Seidel solve
    SysState* deferState_ = nullptr;     // deferNextSolve targets (one-shot)
    LaunchCount lastDeferred_;
    int* deferStatus_ = nullptr;
    const double* curUpper_ = nullptr;   // face coefficients of the current solve (device, user layout)
    const double* curLower_ = nullptr;
    DBuf<TailLevel<double>> tail64_;
    DBuf<TailLevel<float>> tail32_;
    int64_t launches_ = 0;
    bool useGraphs_ = true;
    bool embedding_ = false;
    cudaStream_t side_ = nullptr;        // captures loop bodies while stream_ is being captured

    friend struct StreamSwap;
};

// The level-scheduled kernels' bounded group barrier run on its own: G co-resident CTAs pass
// `rounds` barriers, CTA `absent` (if in range) never arrives.  Returns the status word the barrier
// left (0 or VLM_ERR_TIMEOUT); passed[b] = barriers CTA b got through before any wait gave up.
int groupBarrierCheck(cudaStream_t s, int G, long long spinLimit, int absent, int rounds, int* passed);

// Exact (order-independent) sum of n device doubles, ordered on stream s.
double exactSumOnDevice(cudaStream_t s, const double* v, int64_t n);

SolverKind parseSolver(const char* s);
PrecondKind parsePrecond(const char* s);
SmootherKind parseSmoother(const char* s);

}  // namespace vlm
