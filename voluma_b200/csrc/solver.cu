// Solve drivers of the device-resident LDU batch: per-solve setup (coefficient
// materialisation, Galerkin coarsening, coarsest LU), the GAMG V-cycle, PCG / PBiCGStab
// and the FP64-defect-correction mixed-precision PCG.  Each solve's iteration loop is one
// CUDA graph launch: a conditional WHILE node whose body is one iteration and whose
// predicate is set on the device from the per-system convergence flags.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <functional>
#include <set>
#include <utility>

#include "boxkernels.cuh"
#include "boxstream.cuh"
#include "dilu.cuh"
#include "krylov.cuh"
#include "aggl.h"
#include "solver.h"
#include "tailplan.h"

namespace vlm {

// Device copy of the level schedule (dilu.h) and the per-solve DIC/DILU arrays.
struct DiluDev {
    DBuf<int32_t> loPtr, loCol, loFace, upPtr, upCol, upFace, levPtr, levRows;
    DBuf<DiluSys> sys;
    DBuf<double> loAul, loAlu, upAlu, rD;
    DBuf<DiluBar> bars;
    DBuf<int> err;
    int G = 1, groups = 0, nFaces = 0;
    // streamed shared-memory sweeps (dilu.h DiluLevel): used when smem > 0
    DBuf<DiluLevel> lev;
    DBuf<int32_t> slotRow, sLoCol, sLoFace, sUpCol, sUpFace;
    DBuf<double> prod, coefLo, coefUp, rDs;
    int W = 0, M = 0, nLoS = 0, nUpS = 0;
    size_t smem = 0;   // > 0: shared-memory sweeps with this many bytes per CTA
    int threads = 0;   // their CTA size: the widest level rounded up to whole warps (cheap barriers)
};


GraphExec::~GraphExec() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
}

static bool eq(const char* a, const char* b) { return std::strcmp(a, b) == 0; }

SolverKind parseSolver(const char* s) {
    if (eq(s, "PCG")) return SolverKind::PCG;
    if (eq(s, "PBiCGStab")) return SolverKind::PBiCGStab;
    if (eq(s, "Jacobi")) return SolverKind::Jacobi;
    if (eq(s, "GaussSeidel")) return SolverKind::GaussSeidel;
    if (eq(s, "symGaussSeidel")) return SolverKind::SymGaussSeidel;
    throw Error(VLM_ERR_UNSUPPORTED, std::string("unknown linear solver ") + s);
}

SmootherKind parseSmoother(const char* s) {
    if (s[0] == 0 || eq(s, "mcgs-jacobi")) return SmootherKind::MCGSJacobi;  // default: fastest measured
    if (eq(s, "mcgs")) return SmootherKind::MCGS;
    if (eq(s, "jacobi")) return SmootherKind::Jacobi;
    throw Error(VLM_ERR_BAD_ARG, std::string("unknown smoother ") + s);
}

PrecondKind parsePrecond(const char* s) {
    if (eq(s, "none")) return PrecondKind::None;
    if (eq(s, "diagonal")) return PrecondKind::Diagonal;
    if (eq(s, "GAMG")) return PrecondKind::GAMG;
    if (eq(s, "DIC")) return PrecondKind::DIC;
    if (eq(s, "DILU")) return PrecondKind::DILU;
    throw Error(VLM_ERR_UNSUPPORTED, std::string("unknown preconditioner ") + s);
}

namespace {

inline int nblk(int n, int t = 256) { return (n + t - 1) / t; }

// Coarsest matrices up to this order are factorised in shared memory (2 n^2 doubles).
constexpr int kCoarseSharedN = 80;

// Kernels enqueued (or captured) by this thread; solve() turns captured counts into executed ones.
thread_local int64_t tl_launches = 0;

// Launch helper: skips empty grids (a zero-block launch is an error) and counts the launch.
// Programmatic dependent launch for the solver kernels (VLM_PDL=0 turns it off): each kernel loads
// its fixed inputs while its predecessor drains (pdl_launch / pdl_wait).
thread_local bool tl_capturing = false;

bool pdlEnabled() {
    static const bool on = [] {
        const char* v = std::getenv("VLM_PDL");
        return !(v && v[0] == '0');
    }();
    // inside captured solve graphs too (programmatic edges between consecutive kernel nodes), unless
    // VLM_PDL_GRAPH=0
    static const bool inGraphs = [] {
        const char* v = std::getenv("VLM_PDL_GRAPH");
        return !(v && v[0] == '0');
    }();
    return on && (inGraphs || !tl_capturing);
}

template <class... Exp, class... Act>
void launchKS(void (*kernel)(Exp...), int grid, int block, size_t smem, cudaStream_t s, Act&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdlEnabled() ? 1 : 0;
    VLM_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Act>(args)...));
}

template <class... Exp, class... Act>
void launchK(void (*kernel)(Exp...), int grid, int block, cudaStream_t s, Act&&... args) {
    launchKS(kernel, grid, block, 0, s, std::forward<Act>(args)...);
}

#define VLM_LAUNCH(kernel, grid, block, stream, ...)                    \
    do {                                                                \
        if ((grid) > 0) {                                               \
            launchK(kernel, (grid), (block), (stream), __VA_ARGS__);    \
            ++tl_launches;                                              \
        }                                                               \
    } while (0)

// VLM_LAUNCH with dynamic shared memory
#define VLM_LAUNCH_SMEM(kernel, grid, block, smem, stream, ...)                 \
    do {                                                                        \
        if ((grid) > 0) {                                                       \
            launchKS(kernel, (grid), (block), (smem), (stream), __VA_ARGS__);   \
            ++tl_launches;                                                      \
        }                                                                       \
    } while (0)

template <class T> struct LV;
template <> struct LV<double> {
    static double* r(DevLevel& L) { return L.r.get(); }
    static double* x(DevLevel& L) { return L.x.get(); }
    static double* t(DevLevel& L) { return L.t.get(); }
    static double* x2(DevLevel& L) { return L.x2.get(); }
    static const double* val(const DevLevel& L) { return L.val.get(); }
    static const double* diag(const DevLevel& L) { return L.diag.get(); }
    static const double* bcoef(const DevLevel& L) { return L.bcoef.get(); }
};
template <> struct LV<float> {
    static float* r(DevLevel& L) { return L.r32.get(); }
    static float* x(DevLevel& L) { return L.x32.get(); }
    static float* t(DevLevel& L) { return L.t32.get(); }
    static float* x2(DevLevel& L) { return L.x232.get(); }
    static const float* val(const DevLevel& L) { return L.val32.get(); }
    static const float* diag(const DevLevel& L) { return L.diag32.get(); }
    static const float* bcoef(const DevLevel& L) { return L.bcoef32.get(); }
};

__global__ void k_set_cond(cudaGraphConditionalHandle h, int nsys, const SysState* st, int flag) {
    int a = 0;
    for (int i = threadIdx.x; i < nsys; i += blockDim.x) a |= sys_idle(st[i], flag) ? 0 : 1;
    a = __syncthreads_or(a);
    if (threadIdx.x == 0) cudaGraphSetConditional(h, a ? 1u : 0u);
}

__global__ void k_set_ctrl(DevCtrl* out, DevCtrl v) {
    pdl_entry();
    *out = v;
}

std::vector<cudaGraphNode_t> nodesOf(cudaGraph_t g) {
    size_t n = 0;
    VLM_CUDA(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> v(n);
    if (n) VLM_CUDA(cudaGraphGetNodes(g, v.data(), &n));
    return v;
}

}  // namespace

// ====================================================================== construction
DeviceBatch::DeviceBatch(const std::vector<SysTopo>& systems, int mergeLevels, cudaStream_t stream,
                         bool deviceAgglomeration)
    : stream_(stream), topo_(systems), mergeLevels_(mergeLevels) {
    // VLM_BOX=0 keeps box meshes on the general (SELL) level-0 layout
    const char* bv = std::getenv("VLM_BOX");
    std::function<Hierarchy(const SysTopo&)> hier;
    if (deviceAgglomeration)
        hier = [&](const SysTopo& t) {
            return buildHierarchyDevice(stream, t.nCells, t.nInternal, t.own, t.nei, t.magSf, t.ndc, mergeLevels);
        };
    plan_ = buildPlan(systems, mergeLevels, !(bv && bv[0] == '0'), hier);
    const char* gv = std::getenv("VLM_GRAPH");
    useGraphs_ = !(gv && gv[0] == '0');

    const int nL = int(plan_.levels.size());
    L_.resize(nL);
    const char* om = std::getenv("VLM_JACOBI_OMEGA");
    if (om) jacobiOmega_ = std::atof(om);
    // coarse descriptors grouped by level
    std::vector<CoarseDev> cds;
    for (int k = 0; k < nL; ++k) {
        L_[k].coarse.off = int(cds.size());
        for (const auto& c : plan_.coarse)
            if (c.level == k) cds.push_back(CoarseDev{c.rowStart, c.n, c.invOffset, c.sys});
        L_[k].coarse.n = int(cds.size()) - L_[k].coarse.off;
    }
    coarse_.upload(cds, stream_);
    if (const char* cl = std::getenv("VLM_TAIL_CLUSTER")) tailCl_ = std::atoi(cl);
    if (const char* mr = std::getenv("VLM_TAIL_ROWS")) tailMaxRows_ = std::atoll(mr);
    if (const char* fr = std::getenv("VLM_TAIL_FULL_ROWS")) tailFullRows_ = std::atoll(fr);
    // VLM_BOX_FUSED=1: a box level-0 sweep as one fused launch instead of the two colour launches
    if (const char* f = std::getenv("VLM_BOX_FUSED")) sweepFused_ = f[0] == '1';
    // VLM_BOX_STREAM=0: level 0 of box systems without the plane-streamed kernels
    if (const char* f = std::getenv("VLM_BOX_STREAM")) streamAllowed_ = f[0] != '0';
    // VLM_TAIL_SMEM=0: the coarse tail reads its operands from global memory
    if (const char* f = std::getenv("VLM_TAIL_SMEM")) tailSmemAllowed_ = f[0] != '0';
    if (const char* f = std::getenv("VLM_FUSE_PRE")) fusePre_ = std::atoll(f);
    if (const char* f = std::getenv("VLM_FUSE_RESTRICT")) fuseRestrict_ = std::atoll(f);
    if (const char* f = std::getenv("VLM_FUSE_POST")) fusePost_ = std::atoll(f);
    planTail();
    buildChunkLists();
    for (int k = 0; k < nL; ++k) {
        LevelPlan& P = plan_.levels[k];
        DevLevel& D = L_[k];
        D.blockGS = P.blockGS;
        if (P.blockGS && P.rowColour.size() != size_t(P.nrows))
            throw Error(VLM_ERR_BAD_ARG, "internal: block colour layout mismatch");
        D.nrows = P.nrows;
        D.nfaces = P.nfaces;
        D.nActiveRows = P.nActiveRows;
        D.nSteps = P.nSteps;
        D.maxColours = P.maxColours;
        D.nent = P.slPtr.back();
        D.slPtr.upload(P.slPtr, stream_);
        D.rlen.upload(P.rlen, stream_);
        D.col.upload(P.col, stream_);
        D.src.upload(P.src, stream_);
        if (P.blockGS) D.rowColour.upload(P.rowColour, stream_);
        if (P.box) {
            D.box = true;
            D.boxFace.upload(P.boxFace, stream_);
            D.bcoef.resize(P.boxFace.size());
            boxes_.upload(P.boxes, stream_);
            std::vector<int32_t>().swap(P.boxFace);
        }
        if (k + 1 < nL) {
            D.agg.upload(P.agg, stream_);
            D.childPtr.upload(P.childPtr, stream_);
            D.child.upload(P.child, stream_);
            D.intraPtr.upload(P.intraPtr, stream_);
            D.intraFace.upload(P.intraFace, stream_);
            D.cfacePtr.upload(P.cfacePtr, stream_);
            D.cfaceSrc.upload(P.cfaceSrc, stream_);
        }
        D.diag.resize(size_t(D.nrows));
        D.val.resize(size_t(std::max(D.nent, 1)));
        if (k > 0) {
            D.up.resize(size_t(std::max(D.nfaces, 1)));
            D.lo.resize(size_t(std::max(D.nfaces, 1)));
            D.r.resize(size_t(D.nrows));
            D.x.resize(size_t(D.nrows));
        }
        D.t.resize(size_t(D.nrows));
        D.x2.resize(size_t(D.nrows));
        D.t.zero(stream_);
        D.x2.zero(stream_);
        if (k > 0) {
            D.r.zero(stream_);
            D.x.zero(stream_);
        }
        // host-side plan data no longer needed on the device path; the column indices of levels a
        // shared-memory tail may take (below level 0, every system under 16-bit local indices) stay
        // for re-planning the tail (setTail)
        bool tailLevel = k > 0;
        for (size_t b = 0; tailLevel && b + 1 < P.sysRow.size(); ++b)
            if (P.sysRow[b + 1] - P.sysRow[b] >= 0xffff) tailLevel = false;
        if (!tailLevel) std::vector<int32_t>().swap(P.col);
        std::vector<int32_t>().swap(P.src);
    }
    lu_.resize(size_t(std::max(plan_.invTotal, 1)));
    inv_.resize(size_t(std::max(plan_.invTotal, 1)));
    perm0_.upload(plan_.perm0, stream_);
    sysCells_.upload(plan_.sysCells, stream_);
    slotBegin_.upload(plan_.sysSlotBegin, stream_);
    slotEnd_.upload(plan_.sysSlotEnd, stream_);
    counters_.resize(size_t(plan_.nsys));
    counters_.zero(stream_);
    status_.resize(1);
    status_.zero(stream_);
    partials_.resize(size_t(plan_.nSlots) * 3);  // up to three sums per reduction (k_inner_dot_wr)
    st_.resize(size_t(plan_.nsys));
    st_.zero(stream_);
    dctrl_.resize(1);
    anyActive_.resize(1);
    const int n0 = L_[0].nrows;
    for (DBuf<double>* v : {&x_, &b_, &r_, &w_, &p_, &Ap_}) {
        v->resize(n0);
        v->zero(stream_);
    }
    hostState_.resize(size_t(plan_.nsys));
    if (tailOn_) buildTailTable<double>(tail64_);
    // launch shapes of the plane-streamed level-0 kernels, planned before any stream capture
    if (L_[0].box && plan_.nsys == 1) {
        int g = 0;
        const BoxRows R = boxRows(L_[0], L_[0].all, &g);
        planStream<double>(R);
    }
    VLM_CUDA(cudaStreamSynchronize(stream_));
}

// Row chunk lists of every level (uploaded): all rows, smoothing rows, colour steps, blocks and,
// with the coarse tail on, the rows still handled by per-level launches.
void DeviceBatch::buildChunkLists() {
    for (int k = 0; k < int(L_.size()); ++k) {
        const LevelPlan& P = plan_.levels[k];
        DevLevel& D = L_[k];
        D.headFwd.clear();
        D.headRev.clear();
        D.fwd.clear();
        D.rev.clear();
        std::vector<Chunk> all;
        auto add = [&](const std::vector<Chunk>& v) {
            ChunkList l{int(all.size()), int(v.size())};
            all.insert(all.end(), v.begin(), v.end());
            return l;
        };
        D.active = add(P.active);
        D.all = add(P.all);
        if (tailOn_) {
            // coarse-tail mode: rows still smoothed by per-level launches, and the rows the last
            // of those restrictions writes (systems whose tail starts at or below this level)
            std::vector<Chunk> head, in;
            for (const Chunk& c : P.active)
                if (tailFirst_[c.sys] > k) head.push_back(c);
            for (const Chunk& c : P.all)
                if (k > 0 && tailFirst_[c.sys] >= k) in.push_back(c);
            D.headActive = add(head);
            D.headIn = add(in);
            for (int t = 0; t < P.nSteps; ++t) {
                std::vector<Chunk> hf, hr;
                for (const Chunk& c : P.fwd[t])
                    if (tailFirst_[c.sys] > k) hf.push_back(c);
                for (const Chunk& c : P.rev[t])
                    if (tailFirst_[c.sys] > k) hr.push_back(c);
                D.headFwd.push_back(add(hf));
                D.headRev.push_back(add(hr));
            }
        }
        for (int t = 0; t < P.nSteps; ++t) D.fwd.push_back(add(P.fwd[t]));
        for (int t = 0; t < P.nSteps; ++t) D.rev.push_back(add(P.rev[t]));
        D.blocks = add(P.blocks);
        D.chunks.upload(all, stream_);
        D.hostChunks = all;
    }
}

// Re-plans the coarse tail (cluster size, level row limit, whole-V-cycle row limit; 0 keeps the
// current value) on a registered batch: chunk lists, tail tables, and the recorded graphs.
// Row limits of the fused coarse-level launches (negative keeps a value); the recorded graphs go.
void DeviceBatch::setFusion(int64_t pre, int64_t restrict, int64_t post) {
    VLM_CUDA(cudaStreamSynchronize(stream_));
    if (pre >= 0) fusePre_ = pre;
    if (restrict >= 0) fuseRestrict_ = restrict;
    if (post >= 0) fusePost_ = post;
    graphs_.clear();
}

void DeviceBatch::setTail(int cluster, int64_t maxRows, int64_t fullRows) {
    if (cluster != 0) tailCl_ = cluster;
    if (maxRows != 0) tailMaxRows_ = maxRows;
    if (fullRows != 0) tailFullRows_ = fullRows;
    VLM_CUDA(cudaStreamSynchronize(stream_));
    graphs_.clear();
    tailOn_ = false;
    planTail();
    buildChunkLists();
    if (tailOn_) {
        buildTailTable<double>(tail64_);
        if (e32_.size() == size_t(L_[0].nrows)) buildTailTable<float>(tail32_);
    }
    VLM_CUDA(cudaStreamSynchronize(stream_));
}

DeviceBatch::~DeviceBatch() {
    graphs_.clear();
    if (side_) cudaStreamDestroy(side_);
}

// Temporarily points the batch's recording stream elsewhere (every record function launches on
// stream_): used to capture graph bodies on the side stream while stream_ is being captured.
struct StreamSwap {
    DeviceBatch* b;
    cudaStream_t old;
    StreamSwap(DeviceBatch* batch, cudaStream_t s) : b(batch), old(batch->stream_) { b->stream_ = s; }
    ~StreamSwap() { b->stream_ = old; }
};

void DeviceBatch::beginEmbedding() {
    if (!side_) VLM_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
    embedding_ = true;
    tl_capturing = true;
}

void DeviceBatch::endEmbedding() {
    embedding_ = false;
    tl_capturing = false;
}

bool DeviceBatch::embeddable() const { return useGraphs_ && !(dilu_ && dilu_->G > 1); }

bool DeviceBatch::levelScheduleInSharedMemory(const vlm_solver_ctrl& ctrl) {
    PrecondKind pk = parsePrecond(ctrl.preconditioner);
    SolverKind sk = parseSolver(ctrl.solver);
    if (ctrl.reproducible) {
        if (pk != PrecondKind::None) pk = PrecondKind::Diagonal;
        if (sk == SolverKind::GaussSeidel || sk == SolverKind::SymGaussSeidel) sk = SolverKind::Jacobi;
    }
    const bool levels = pk == PrecondKind::DIC || pk == PrecondKind::DILU || sk == SolverKind::GaussSeidel ||
                        sk == SolverKind::SymGaussSeidel;
    if (!levels) return true;
    ensureDilu();
    return dilu_->smem > 0;
}

template <class T>
void DeviceBatch::buildTailTable(DBuf<TailLevel<T>>& out) {
    const int nL = int(L_.size());
    std::vector<TailLevel<T>> tab(static_cast<size_t>(nL));
    for (int k = 0; k < nL; ++k) {
        DevLevel& D = L_[k];
        TailLevel<T>& t = tab[k];
        t.S = D.sell();
        t.val = LV<T>::val(D);
        t.diag = LV<T>::diag(D);
        t.r = k > 0 ? LV<T>::r(D) : nullptr;
        t.x = k > 0 ? LV<T>::x(D) : nullptr;
        t.x2 = LV<T>::x2(D);
        t.agg = D.agg.get();
        t.cptr = D.childPtr.get();
        t.child = D.child.get();
    }
    out.upload(tab, stream_);
    VLM_CUDA(cudaStreamSynchronize(stream_));  // the host table is a local
}

size_t DeviceBatch::deviceBytes() const {
    size_t b = 0;
    for (const auto& D : L_)
        b += D.slPtr.bytes() + D.rlen.bytes() + D.col.bytes() + D.src.bytes() + D.chunks.bytes() + D.agg.bytes() +
             D.childPtr.bytes() + D.child.bytes() + D.intraPtr.bytes() + D.intraFace.bytes() + D.cfacePtr.bytes() +
             D.cfaceSrc.bytes() + D.diag.bytes() + D.val.bytes() + D.up.bytes() + D.lo.bytes() + D.diag32.bytes() +
             D.val32.bytes() + D.r.bytes() + D.x.bytes() + D.t.bytes() + D.x2.bytes() + D.r32.bytes() +
             D.x32.bytes() + D.t32.bytes() + D.x232.bytes();
    b += lu_.bytes() + inv_.bytes() + perm0_.bytes() + partials_.bytes();
    b += x_.bytes() + b_.bytes() + r_.bytes() + w_.bytes() + p_.bytes() + Ap_.bytes() + rD_.bytes() + r0_.bytes() +
         y_.bytes() + Ay_.bytes() + s_.bytes() + z_.bytes() + t_.bytes();
    b += e32_.bytes() + r32_.bytes() + w32_.bytes() + p32_.bytes() + Ap32_.bytes() + rD32_.bytes();
    return b;
}

void DeviceBatch::ensureVectors(bool mixed, bool bicg) {
    const size_t n0 = size_t(L_[0].nrows);
    if (bicg && r0_.size() != n0) {
        r0_.resize(n0);
        y_.resize(n0);
        Ay_.resize(n0);
        s_.resize(n0);
        z_.resize(n0);
        t_.resize(n0);
    }
    if (mixed && e32_.size() != n0) {
        e32_.resize(n0);
        r32_.resize(n0);
        w32_.resize(n0);
        p32_.resize(n0);
        Ap32_.resize(n0);
        e32_.zero(stream_);
        r32_.zero(stream_);
        w32_.zero(stream_);
        p32_.zero(stream_);
        Ap32_.zero(stream_);
        for (size_t k = 0; k < L_.size(); ++k) {
            DevLevel& D = L_[k];
            D.diag32.resize(size_t(D.nrows));
            D.val32.resize(size_t(std::max(D.nent, 1)));
            if (k > 0) {
                D.r32.resize(size_t(D.nrows));
                D.x32.resize(size_t(D.nrows));
                D.r32.zero(stream_);
                D.x32.zero(stream_);
            }
            D.t32.resize(size_t(D.nrows));
            D.x232.resize(size_t(D.nrows));
            D.t32.zero(stream_);
            D.x232.zero(stream_);
            if (D.box) D.bcoef32.resize(D.bcoef.size());
        }
        if (tailOn_) buildTailTable<float>(tail32_);
    }
}

// The rows of a box-kernel launch: the range form for a batch of one system (its chunks are
// consecutive), else the chunk list.  *grid: CTAs of the launch.
BoxRows DeviceBatch::boxRows(const DevLevel& D, const ChunkList& l, int* grid) const {
    BoxRows R = {};
    if (plan_.nsys == 1 && l.n > 0) {
        const Chunk& a = D.hostChunks[size_t(l.off)];
        const Chunk& z = D.hostChunks[size_t(l.off + l.n - 1)];
        R.ch = nullptr;
        R.one = plan_.levels[0].boxes[0];
        R.begin = a.start;
        R.end = z.start + z.count;
        *grid = (R.end - R.begin + kRowsPerCta - 1) / kRowsPerCta;
    } else {
        R.ch = D.ch(l);
        R.boxes = boxes_.get();
        *grid = l.n;
    }
    return R;
}

// Launch shape of the streamed level-0 kernels (boxstream.cuh) for this batch's box system in
// elements of T, planned at registration (streamShape: null where they do not apply and the
// four-slot kernels run; VLM_BOX_STREAM=0 at registration: never).  They need a batch of one
// system in the range form, H % 4 == 0 (16-byte rows), colour
// groups and coefficient arrays on 16-byte boundaries, at least 3 planes, and a pencil height TY
// (8, 4 or 2 x-rows) dividing ny with 2 * TY * H / N consumer threads (N slots of one colour, 16
// bytes, each) a whole number of warps, at most 256.  The ring takes as many plane stages (3..8)
// as the opt-in shared memory holds; the grid is one wave.
template <class T>
void DeviceBatch::planStream(const BoxRows& R) {
    StreamShape& sh = sizeof(T) == 8 ? stream64_ : stream32_;
    sh = StreamShape{};
    if (!streamAllowed_ || R.ch != nullptr || plan_.nsys != 1) return;
    const BoxSys& B = R.one;
    if (B.H % 4 != 0 || B.nz < 3 || B.base0 % 4 != 0 || B.base1 % 4 != 0 || L_[0].nrows % 4 != 0) return;
    auto kernel = k_box_pcg_spmv_stream<T, kFlagDone>;
    int dev = 0, optin = 0, perSm = 0, sms = 0;
    VLM_CUDA(cudaGetDevice(&dev));
    VLM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    VLM_CUDA(cudaDeviceGetAttribute(&perSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    VLM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaFuncAttributes fa = {};
    VLM_CUDA(cudaFuncGetAttributes(&fa, kernel));
    // the most resident warps per SM over pencil heights and CTAs per SM, with at least 4 stages
    // (two read, two in flight); VLM_STREAM_TY / VLM_STREAM_CTAS pin a choice
    const int pinTY = std::getenv("VLM_STREAM_TY") ? std::atoi(std::getenv("VLM_STREAM_TY")) : 0;
    const int pinCtas = std::getenv("VLM_STREAM_CTAS") ? std::atoi(std::getenv("VLM_STREAM_CTAS")) : 0;
    int TY = 0, S = 0, bestWarps = 0;
    for (int t : {8, 4, 2}) {
        const int consumers = 2 * t * B.H / SG<T>::N;
        if (B.ny % t != 0 || consumers % 32 != 0 || consumers > kStreamMaxThreads - 32) continue;
        if (pinTY && t != pinTY) continue;
        const size_t stage = size_t(stream_stage_elems(B.H, t)) * sizeof(T);
        for (int c = 1; c <= 3; ++c) {
            if (pinCtas && c != pinCtas) continue;
            const size_t budget = std::min<size_t>(size_t(optin), size_t(perSm) / c - 1024);
            if (budget < fa.sharedSizeBytes + 128 + 4 * stage) continue;
            const int s = int(std::min<size_t>(8, (budget - fa.sharedSizeBytes - 128) / stage));
            const int warps = c * (consumers / 32 + 1);
            if (warps > bestWarps || (warps == bestWarps && s > S)) {
                bestWarps = warps;
                TY = t;
                S = s;
            }
        }
    }
    if (TY == 0) return;
    const size_t smem = 128 + size_t(S) * size_t(stream_stage_elems(B.H, TY)) * sizeof(T);
    // the attribute belongs to the kernel, not to this mesh: allow the most any mesh's launch asks
    VLM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin - int(fa.sharedSizeBytes)));
    int per = 0;
    const int threads = 32 + 2 * TY * B.H / SG<T>::N;  // the producer warp and the consumers
    VLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem));
    if (per < 1) return;
    const int W = (B.ny / TY) * B.nz;
    const int slots = plan_.sysSlotEnd[0] - plan_.sysSlotBegin[0];
    if (sweepSync_.size() == 0) {
        sweepSync_.resize(1);
        sweepSync_.zero(stream_);
    }
    sh.TY = TY;
    sh.S = S;
    sh.threads = threads;
    sh.smem = smem;
    sh.grid = std::min({sms * per, W, slots});
}

template <class T>
const DeviceBatch::StreamShape* DeviceBatch::streamShape(const BoxRows& R) const {
    const StreamShape& sh = sizeof(T) == 8 ? stream64_ : stream32_;
    return sh.grid > 0 && R.ch == nullptr ? &sh : nullptr;
}

RedCtx DeviceBatch::red() const {
    return RedCtx{partials_.get(), xbins_.get(), counters_.get(), slotBegin_.get(), slotEnd_.get()};
}

// ====================================================================== per-solve setup
void DeviceBatch::setupMatrix(const double* diag, const double* upper, const double* lower, bool gamg, bool mixed) {
    cudaStream_t s = stream_;
    curUpper_ = upper;
    curLower_ = lower;
    DevLevel& D0 = L_[0];
    VLM_LAUNCH(k_gather_diag0<double>, nblk(D0.nrows), 256, s, D0.nrows, perm0_.get(), diag, D0.diag.get());
    if (mixed) VLM_LAUNCH(k_gather_diag0<float>, nblk(D0.nrows), 256, s, D0.nrows, perm0_.get(), diag, D0.diag32.get());
    VLM_LAUNCH(k_materialize, nblk(D0.nent), 256, s, D0.nent, D0.src.get(), upper, lower, D0.val.get(),
               mixed ? D0.val32.get() : nullptr);
    // the box kernels take each face coefficient once: symmetric matrices only
    boxOn_ = D0.box && lower == upper;
    if (boxOn_) {
        const int n3 = int(D0.bcoef.size());
        VLM_LAUNCH(k_box_coef, nblk(n3), 256, s, n3, D0.boxFace.get(), upper, D0.bcoef.get(),
                   mixed ? D0.bcoef32.get() : nullptr);
    }
    if (!gamg) return;
    const int nL = int(L_.size());
    for (int k = 0; k + 1 < nL; ++k) {
        DevLevel& F = L_[k];
        DevLevel& C = L_[k + 1];
        const double* up = k == 0 ? upper : F.up.get();
        const double* lo = k == 0 ? lower : F.lo.get();
        VLM_LAUNCH(k_galerkin_diag, nblk(C.nrows), 256, s, C.nrows, F.childPtr.get(), F.child.get(), F.intraPtr.get(),
                   F.intraFace.get(), F.diag.get(), up, lo, C.diag.get(), mixed ? C.diag32.get() : nullptr);
        VLM_LAUNCH(k_galerkin_faces, nblk(C.nfaces), 256, s, C.nfaces, F.cfacePtr.get(), F.cfaceSrc.get(), up, lo,
                   C.up.get(), C.lo.get());
        VLM_LAUNCH(k_materialize, nblk(C.nent), 256, s, C.nent, C.src.get(), C.up.get(), C.lo.get(), C.val.get(),
                   mixed ? C.val32.get() : nullptr);
    }
    VLM_CUDA(cudaMemsetAsync(status_.get(), 0, sizeof(int), s));
    for (int k = 0; k < nL; ++k) {
        DevLevel& D = L_[k];
        if (D.coarse.n == 0) continue;
        int nmax = 0;
        for (const auto& c : plan_.coarse)
            if (c.level == k) nmax = std::max(nmax, c.n);
        const int smemN = nmax <= kCoarseSharedN ? nmax : 0;
        const size_t smem = size_t(2) * smemN * smemN * sizeof(double);
        // the opt-in limit is per function and shared by every mesh: raised once to the ceiling
        static const bool raised = [] {
            VLM_CUDA(cudaFuncSetAttribute(k_coarse_factor, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(size_t(2) * kCoarseSharedN * kCoarseSharedN * sizeof(double))));
            return true;
        }();
        (void)raised;
        k_coarse_factor<<<D.coarse.n, 512, smem, s>>>(coarse_.get() + D.coarse.off, D.sell(), D.val.get(),
                                                     D.diag.get(), lu_.get(), inv_.get(), status_.get(), smemN);
        VLM_CUDA(cudaGetLastError());
        ++tl_launches;
    }
    if (tailOn_ && tailSmem_) {
        // the shared-memory tail's value images of this solve's coarse levels
        const int nv = int(tailCodes_.size());
        VLM_LAUNCH(k_tail_values<double>, nblk(nv), 256, s, nv, tailCodes_.get(), tail64_.get(), tailVal64_.get());
        if (mixed && tail32_.size() != 0)
            VLM_LAUNCH(k_tail_values<float>, nblk(nv), 256, s, nv, tailCodes_.get(), tail32_.get(), tailVal32_.get());
    }
}

// ====================================================================== V-cycle
template <class T>
void DeviceBatch::recordSmooth(int k, const T* r, T* x, SmootherKind sm, bool pre, int flag, bool head) {
    DevLevel& D = L_[k];
    cudaStream_t s = stream_;
    const Sell S = D.sell();
    const T* val = LV<T>::val(D);
    const T* diag = LV<T>::diag(D);
    const SysState* st = st_.get();
    T* x2 = LV<T>::x2(D);
    const int32_t* agg = D.agg.get();
    const T* xc = k + 1 < int(L_.size()) ? LV<T>::x(L_[k + 1]) : nullptr;
    const bool jacobiHere = sm == SmootherKind::Jacobi || (sm == SmootherKind::MCGSJacobi && k > 0);
    if (jacobiHere) {
        // Jacobi; pre: from zero, post: after the ascent's prolongation pass
        const T om = T(jacobiOmega_);
        const ChunkList& rows = head ? D.headActive : D.active;
        if (pre && fusedLevel(k, fusePre_)) {
            // both sweeps from zero in one pass
            VLM_LAUNCH((k_smooth_jacobi<T, 3>), rows.n, kRowsPerCta, s, D.ch(rows), S, val, diag, r,
                       (const T*)nullptr, x, om, agg, xc, st, flag);
        } else if (!pre && fusedLevel(k, fusePost_)) {
            // the coarse-grid correction inside the first sweep (no k_prolong pass)
            VLM_LAUNCH((k_smooth_jacobi<T, 2>), rows.n, kRowsPerCta, s, D.ch(rows), S, val, diag, r, x, x2,
                       om, agg, xc, st, flag);
            VLM_LAUNCH((k_smooth_jacobi<T, 0>), rows.n, kRowsPerCta, s, D.ch(rows), S, val, diag, r, x2, x,
                       om, agg, xc, st, flag);
        } else if (pre) {
            VLM_LAUNCH((k_smooth_jacobi<T, 1>), rows.n, kRowsPerCta, s, D.ch(rows), S, val, diag, r,
                       (const T*)nullptr, x2, om, agg, xc, st, flag);
            VLM_LAUNCH((k_smooth_jacobi<T, 0>), rows.n, kRowsPerCta, s, D.ch(rows), S, val, diag, r, x2, x,
                       om, agg, xc, st, flag);
        } else {
            // the correction x += xc[agg] as its own coalesced pass (the ascent launches k_prolong), then
            // plain sweeps: the same values as a first sweep that adds xc[agg[j]] to every neighbour it
            // reads, which pays two more dependent loads per entry and measured slower
            VLM_LAUNCH((k_smooth_jacobi<T, 0>), rows.n, kRowsPerCta, s, D.ch(rows), S, val, diag, r, x, x2,
                       om, agg, xc, st, flag);
            VLM_LAUNCH((k_smooth_jacobi<T, 0>), rows.n, kRowsPerCta, s, D.ch(rows), S, val, diag, r, x2, x,
                       om, agg, xc, st, flag);
        }
    } else if (D.blockGS) {
        // block-hybrid GS; pre: from zero, post: prolongation fused into the first sweep
        const int8_t* rc = D.rowColour.get();
        if (pre) {
            VLM_LAUNCH((k_smooth_bgs<T, 1, true>), D.blocks.n, kBlockRows, s, D.ch(D.blocks), S, val, diag, r, x, x2,
                       rc, agg, xc, st, flag);
            VLM_LAUNCH((k_smooth_bgs<T, 0, true>), D.blocks.n, kBlockRows, s, D.ch(D.blocks), S, val, diag, r, x2, x,
                       rc, agg, xc, st, flag);
        } else {
            VLM_LAUNCH((k_smooth_bgs<T, 2, false>), D.blocks.n, kBlockRows, s, D.ch(D.blocks), S, val, diag, r, x,
                       x2, rc, agg, xc, st, flag);
            VLM_LAUNCH((k_smooth_bgs<T, 0, false>), D.blocks.n, kBlockRows, s, D.ch(D.blocks), S, val, diag, r, x2,
                       x, rc, agg, xc, st, flag);
        }
    } else {
        // global multicolour GS: forward colours pre-smoothing, reversed colours post-smoothing.
        // Two colours: the pre-smoothing's first colour sees only zeros (x = r/D, no zeroing
        // needed) and the post-smoothing's first colour applies the prolongation to the
        // neighbours it reads (no separate prolongation).
        const bool two = D.nSteps == 2;
        const ChunkList& rows = head ? D.headActive : D.active;
        if (pre && !two) VLM_LAUNCH(k_zero_rows<T>, rows.n, kRowsPerCta, s, D.ch(rows), x, st, flag);
        const bool boxK = k == 0 && boxOn_;
        const T* bc = LV<T>::bcoef(D);
        // live sweep timing (eager solves only): an event pair around each level-0 sweep
        cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
        if (timeSweeps_ && k == 0) VLM_CUDA(cudaStreamIsCapturing(s, &cap));
        const bool timed = timeSweeps_ && k == 0 && cap == cudaStreamCaptureStatusNone;
        cudaEvent_t te0 = nullptr;
        auto sweepEnd = [&] {
            if (!timed) return;
            cudaEvent_t te1 = nullptr;
            VLM_CUDA(cudaEventCreate(&te1));
            VLM_CUDA(cudaEventRecord(te1, s));
            sweepEvents_.push_back({te0, te1});
        };
        for (int sweep = 0; sweep < 2; ++sweep) {
            if (timed) {
                VLM_CUDA(cudaEventCreate(&te0));
                VLM_CUDA(cudaEventRecord(te0, s));
            }
            if (boxK && two) {
                const ChunkList& la = head ? (pre ? D.headFwd[0] : D.headRev[0]) : (pre ? D.fwd[0] : D.rev[0]);
                const ChunkList& lb = head ? (pre ? D.headFwd[1] : D.headRev[1]) : (pre ? D.fwd[1] : D.rev[1]);
                if (recordFusedSweep<T>(la, lb, r, x, pre, sweep, agg, xc)) {
                    sweepEnd();
                    continue;
                }
            }
            for (int t = 0; t < D.nSteps; ++t) {
                const ChunkList& l = head ? (pre ? D.headFwd[t] : D.headRev[t]) : (pre ? D.fwd[t] : D.rev[t]);
                if (boxK) {
                    int g = 0;
                    const BoxRows R = boxRows(D, l, &g);
                    if (R.ch == nullptr && R.one.H % 4 == 0) {
                        // four slots per thread
                        const int g4 = (R.end - R.begin + 4 * kRowsPerCta - 1) / (4 * kRowsPerCta);
                        if (two && sweep == 0 && t == 0 && pre)
                            VLM_LAUNCH((k_box_gs4<T, 1>), g4, kRowsPerCta, s, R, bc, D.nrows, diag, r, x, agg, xc);
                        else if (two && sweep == 0 && t == 0)
                            VLM_LAUNCH((k_box_gs4<T, 2>), g4, kRowsPerCta, s, R, bc, D.nrows, diag, r, x, agg, xc);
                        else
                            VLM_LAUNCH((k_box_gs4<T, 0>), g4, kRowsPerCta, s, R, bc, D.nrows, diag, r, x, agg, xc);
                        continue;
                    }
                    if (two && sweep == 0 && t == 0 && pre)
                        VLM_LAUNCH((k_box_gs<T, 1>), g, kRowsPerCta, s, R, bc, D.nrows, diag, r, x, agg, xc, st, flag);
                    else if (two && sweep == 0 && t == 0)
                        VLM_LAUNCH((k_box_gs<T, 2>), g, kRowsPerCta, s, R, bc, D.nrows, diag, r, x, agg, xc, st, flag);
                    else
                        VLM_LAUNCH((k_box_gs<T, 0>), g, kRowsPerCta, s, R, bc, D.nrows, diag, r, x, agg, xc, st, flag);
                    continue;
                }
                if (two && sweep == 0 && t == 0 && pre)
                    VLM_LAUNCH((k_smooth_gs<T, 1>), l.n, kRowsPerCta, s, D.ch(l), S, val, diag, r, x, agg, xc, st,
                               flag);
                else if (two && sweep == 0 && t == 0)
                    VLM_LAUNCH((k_smooth_gs<T, 2>), l.n, kRowsPerCta, s, D.ch(l), S, val, diag, r, x, agg, xc, st,
                               flag);
                else
                    VLM_LAUNCH((k_smooth_gs<T, 0>), l.n, kRowsPerCta, s, D.ch(l), S, val, diag, r, x, agg, xc, st,
                               flag);
            }
            sweepEnd();
        }
    }
}

void DeviceBatch::setSweepTiming(bool on) {
    VLM_CUDA(cudaStreamSynchronize(stream_));
    collectSweepTimes();
    timeSweeps_ = on;
    sweepMs_ = 0.0;
    sweepCount_ = 0;
}

// Adds the recorded level-0 sweep times (the stream has been synchronised) and frees the events.
void DeviceBatch::collectSweepTimes() {
    for (auto& e : sweepEvents_) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess) {
            sweepMs_ += ms;
            ++sweepCount_;
        }
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    sweepEvents_.clear();
}

// One red-black sweep of a single box system's level 0 as one launch (k_box_sweep4): forward colours
// for pre-smoothing, reversed for post-smoothing; the first sweep starts from zero (pre) or carries
// the coarse-grid correction (post).  False when the layout does not qualify (the caller then
// launches the two colour steps).
template <class T>
bool DeviceBatch::recordFusedSweep(const ChunkList& la, const ChunkList& lb, const T* r, T* x, bool pre, int sweep,
                                   const int32_t* agg, const T* xc) {
    DevLevel& D = L_[0];
    if (!sweepFused_ || plan_.nsys != 1 || D.nSteps != 2 || la.n == 0 || lb.n == 0) return false;
    int g = 0;
    const BoxRows RA = boxRows(D, la, &g);
    const BoxRows RB = boxRows(D, lb, &g);
    if (RA.ch != nullptr || RB.ch != nullptr || RA.one.H % 4 != 0) return false;
    const int nA = (RA.end - RA.begin + kSweepPiece - 1) / kSweepPiece;
    const int nB = (RB.end - RB.begin + kSweepPiece - 1) / kSweepPiece;
    if (sweepDone_.size() == 0) {
        int dev = 0, sms = 0, per = 0;
        VLM_CUDA(cudaGetDevice(&dev));
        VLM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        VLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_box_sweep4<T, 0>, kRowsPerCta, 0));
        sweepGrid_ = sms * std::max(1, per);
        if (sweepSync_.size() == 0) {
            sweepSync_.resize(1);
            sweepSync_.zero(stream_);
        }
        sweepDone_.resize(size_t(std::max(nA, nB)));
        sweepDone_.zero(stream_);
    }
    if (sweepDone_.size() < size_t(std::max(nA, nB))) return false;
    const int grid = std::min(sweepGrid_, nA + nB);
    const T* bc = LV<T>::bcoef(D);
    cudaStream_t s = stream_;
    const int mode = sweep == 0 ? (pre ? 1 : 2) : 0;
    if (mode == 1)
        VLM_LAUNCH((k_box_sweep4<T, 1>), grid, kRowsPerCta, s, RA.one, RA.begin, RA.end, RB.begin, RB.end, bc, D.nrows,
                   LV<T>::diag(D), r, x, agg, xc, sweepSync_.get(), sweepDone_.get());
    else if (mode == 2)
        VLM_LAUNCH((k_box_sweep4<T, 2>), grid, kRowsPerCta, s, RA.one, RA.begin, RA.end, RB.begin, RB.end, bc, D.nrows,
                   LV<T>::diag(D), r, x, agg, xc, sweepSync_.get(), sweepDone_.get());
    else
        VLM_LAUNCH((k_box_sweep4<T, 0>), grid, kRowsPerCta, s, RA.one, RA.begin, RA.end, RB.begin, RB.end, bc, D.nrows,
                   LV<T>::diag(D), r, x, agg, xc, sweepSync_.get(), sweepDone_.get());
    return true;
}

// A wait of the fused sweep (bit 0) or of a streamed kernel (bit 1) that gave up leaves a non-zero
// error word.
void DeviceBatch::checkSweepError() {
    if (sweepSync_.size() == 0) return;
    SweepSync h = {};
    VLM_CUDA(cudaMemcpy(&h, sweepSync_.get(), sizeof h, cudaMemcpyDeviceToHost));
    if (h.err != 0) {
        VLM_CUDA(cudaMemsetAsync(&sweepSync_.get()->err, 0, sizeof(unsigned), stream_));
        VLM_CUDA(cudaStreamSynchronize(stream_));
        throw Error(VLM_ERR_TIMEOUT, (h.err & 1u) ? "fused level-0 sweep: a wait for another CTA's piece gave up"
                                                  : "streamed level-0 kernel: a plane stage never arrived");
    }
}

// GamgPreconditioner::vcycle (GAMG.cpp:403-443) for every system of the batch at once:
// descend (2 pre-sweeps, residual, restriction) through the levels on which at least one
// system still smooths, solve every system's coarsest level, then ascend (prolongation,
// 2 post-sweeps).
template <class T>
void DeviceBatch::recordVcycle(const T* r0, T* x0, SmootherKind sm, int flag, bool allowTail) {
    cudaStream_t s = stream_;
    const int nL = int(L_.size());
    const SysState* st = st_.get();
    auto rr = [&](int k) -> const T* { return k == 0 ? r0 : LV<T>::r(L_[k]); };
    auto xx = [&](int k) -> T* { return k == 0 ? x0 : LV<T>::x(L_[k]); };
    // Jacobi coarse levels: each system's levels from tailFirst_ down run in one cluster launch
    const bool tail = allowTail && tailOn_ && sm != SmootherKind::MCGS;
    const int headEnd = tail ? tailMaxFirst_ : nL - 1;
    for (int k = 0; k < headEnd; ++k) {
        DevLevel& D = L_[k];
        DevLevel& N = L_[k + 1];
        const ChunkList& rows = tail ? D.headActive : D.active;
        const ChunkList& next = tail ? N.headIn : N.all;
        recordSmooth<T>(k, rr(k), xx(k), sm, true, flag, tail);
        if (k == 0 && boxOn_) {
            int g = 0;
            const BoxRows R = boxRows(D, rows, &g);
            if (R.ch == nullptr && R.one.H % 4 == 0)
                VLM_LAUNCH(k_box_residual4<T>, (R.end - R.begin + 4 * kRowsPerCta - 1) / (4 * kRowsPerCta),
                           kRowsPerCta, s, R, LV<T>::bcoef(D), D.nrows, LV<T>::diag(D), rr(k), (const T*)xx(k),
                           LV<T>::t(D));
            else
                VLM_LAUNCH(k_box_residual<T>, g, kRowsPerCta, s, R, LV<T>::bcoef(D), D.nrows, LV<T>::diag(D), rr(k),
                           (const T*)xx(k), LV<T>::t(D), st, flag);
        } else if (fusedLevel(k, fuseRestrict_)) {
            VLM_LAUNCH(k_residual_restrict<T>, next.n, kRowsPerCta, s, N.ch(next), D.sell(), LV<T>::val(D),
                       LV<T>::diag(D), rr(k), (const T*)xx(k), D.childPtr.get(), D.child.get(), LV<T>::r(N), st, flag);
            continue;
        } else
            VLM_LAUNCH(k_residual<T>, rows.n, kRowsPerCta, s, D.ch(rows), D.sell(), LV<T>::val(D), LV<T>::diag(D),
                       rr(k), xx(k), LV<T>::t(D), st, flag);
        VLM_LAUNCH(k_restrict<T>, next.n, kRowsPerCta, s, N.ch(next), D.childPtr.get(), D.child.get(), LV<T>::t(D),
                   LV<T>::r(N), st, flag);
    }
    if (tail) {
        recordTail<T>(r0, x0, flag, sm == SmootherKind::Jacobi);
    } else {
        for (int k = 0; k < nL; ++k) {
            DevLevel& D = L_[k];
            VLM_LAUNCH(k_coarse_apply<T>, D.coarse.n, 128, s, coarse_.get() + D.coarse.off, inv_.get(), rr(k), xx(k),
                       st, flag);
        }
    }
    for (int k = headEnd - 1; k >= 0; --k) {
        DevLevel& D = L_[k];
        const bool jacobiHere = sm == SmootherKind::Jacobi || (sm == SmootherKind::MCGSJacobi && k > 0);
        // block GS and two-colour GS fuse the prolongation into their first sweep (for two colours
        // the separate pass measured no faster); Jacobi (on any level layout) and multicolour GS
        // with more colours sweep after this pass (active chunks are at most kRowsPerCta rows, one
        // per k_prolong thread)
        const bool fusedProlong = jacobiHere && fusedLevel(k, fusePost_);
        if (!fusedProlong && (jacobiHere || (!D.blockGS && D.nSteps != 2))) {
            const ChunkList& rows = tail ? D.headActive : D.active;
            VLM_LAUNCH(k_prolong<T>, rows.n, kRowsPerCta, s, D.ch(rows), D.agg.get(), xx(k + 1), xx(k), st, flag);
        }
        recordSmooth<T>(k, rr(k), xx(k), sm, false, flag, tail);
    }
}

template <class T>
void DeviceBatch::recordTail(const T* r0, T* x0, int flag, bool jacobi0) {
    const TailLevel<T>* tab = std::is_same<T, float>::value ? (const TailLevel<T>*)tail32_.get()
                                                             : (const TailLevel<T>*)tail64_.get();
    if (!tab) throw Error(VLM_ERR_CUDA, "internal: coarse-tail table missing");
    if (tailSmem_) {
        // every operand in shared memory, one CTA per system
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(tailImg_.size()));
        cfg.blockDim = dim3(unsigned(kTailThreads));
        cfg.dynamicSmemBytes = std::is_same<T, float>::value ? tailSmem32_ : tailSmem64_;
        cfg.stream = stream_;
        cudaLaunchAttribute at[1];
        int na = 0;
        if (pdlEnabled()) {
            at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            at[na].val.programmaticStreamSerializationAllowed = 1;
            ++na;
        }
        cfg.attrs = at;
        cfg.numAttrs = unsigned(na);
        const T* vimg = std::is_same<T, float>::value ? (const T*)tailVal32_.get() : (const T*)tailVal64_.get();
        VLM_CUDA(cudaLaunchKernelEx(&cfg, k_vcycle_tail_smem<T>, (const TailImg*)tailImg_.get(), vimg,
                                    (const uint16_t*)tailStr_.get(), tab, (const double*)inv_.get(), T(jacobiOmega_),
                                    (const SysState*)st_.get(), flag));
        ++tl_launches;
        return;
    }
    // one CTA, or one thread-block cluster of tailCl_ CTAs, per system
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(tailSys_.size()) * unsigned(tailCl_));
    cfg.blockDim = dim3(unsigned(kTailThreads));
    cfg.stream = stream_;
    cudaLaunchAttribute at[2];
    int na = 0;
    if (tailCl_ > 1) {
        at[na].id = cudaLaunchAttributeClusterDimension;
        at[na].val.clusterDim.x = unsigned(tailCl_);
        at[na].val.clusterDim.y = 1;
        at[na].val.clusterDim.z = 1;
        ++na;
    }
    if (pdlEnabled()) {
        at[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        at[na].val.programmaticStreamSerializationAllowed = 1;
        ++na;
    }
    cfg.attrs = at;
    cfg.numAttrs = unsigned(na);
    auto launch = [&](auto kernel) {
        VLM_CUDA(cudaLaunchKernelEx(&cfg, kernel, (const TailSys*)tailSys_.get(), tab, (const double*)inv_.get(), r0, x0,
                                    T(jacobiOmega_), (const SysState*)st_.get(), flag, jacobi0 ? 1 : 0));
    };
    switch (tailCl_) {
    case 1: launch(k_vcycle_tail<T, 1>); break;
    case 2: launch(k_vcycle_tail<T, 2>); break;
    case 4: launch(k_vcycle_tail<T, 4>); break;
    case 8: launch(k_vcycle_tail<T, 8>); break;
    default: throw Error(VLM_ERR_BAD_ARG, "coarse-tail cluster size must be 1, 2, 4 or 8");
    }
    ++tl_launches;
}

// Per system: the first level of the single-CTA tail = the first level (below level 0) whose
// padded row count is at most kTailMaxRows (VLM_TAIL_ROWS overrides; VLM_TAIL=0 disables), else
// the coarsest level alone.
void DeviceBatch::planTail() {
    const char* tv = std::getenv("VLM_TAIL");
    if (tv && tv[0] == '0') return;
    const int ns = plan_.nsys;
    if (ns == 0) return;
    // the tail runs on one CTA or on a cluster of tailCl_ CTAs; unset row limits (0) scale with it
    if (tailCl_ != 1 && tailCl_ != 2 && tailCl_ != 4 && tailCl_ != 8)
        throw Error(VLM_ERR_BAD_ARG, "the coarse-tail cluster size must be 1, 2, 4 or 8");
    const int64_t maxRows = tailMaxRows_ > 0 ? tailMaxRows_ : int64_t(kTailMaxRows) * tailCl_;
    const int64_t fullRows =
        tailFullRows_ > 0 ? tailFullRows_ : (tailCl_ == 1 ? int64_t(kTailFullRows) : int64_t(kTailMaxRows) * tailCl_);
    const LevelPlan& L0 = plan_.levels[0];
    tailFirst_.assign(size_t(ns), 0);
    std::vector<TailSys> ts(static_cast<size_t>(ns));
    tailMaxFirst_ = 0;
    for (int b = 0; b < ns; ++b) {
        const int c = plan_.nLevels[b] - 1;
        if (c >= kTailMaxLevels) throw Error(VLM_ERR_UNSUPPORTED, "GAMG hierarchy deeper than the coarse tail supports");
        int first = c;
        const int64_t rows0 = plan_.levels[0].sysRow[b + 1] - plan_.levels[0].sysRow[b];
        if (c > 0 && rows0 <= fullRows && !plan_.levels[0].blockGS)
            first = 0;  // the whole V-cycle of a small system in one CTA
        else
            for (int k = 1; k < c; ++k)
                if (int64_t(plan_.levels[k].sysRow[b + 1] - plan_.levels[k].sysRow[b]) <= maxRows) {
                    first = k;
                    break;
                }
        tailFirst_[b] = first;
        tailMaxFirst_ = std::max(tailMaxFirst_, first);
        TailSys& t = ts[b];
        std::memset(&t, 0, sizeof t);
        t.sys = b;
        t.first = first;
        t.coarsest = c;
        const CoarsePlan& cp = plan_.coarse[b];
        t.coarseN = cp.n;
        t.invOffset = cp.invOffset;
        for (int k = 0; k <= c; ++k) {
            t.rowStart[k] = plan_.levels[k].sysRow[b];
            t.rowCount[k] = plan_.levels[k].sysRow[b + 1] - plan_.levels[k].sysRow[b];
        }
        // level-0 colour groups of this system (the chunks of the colour steps)
        t.two = L0.nSteps == 2 ? 1 : 0;
        t.nColours = 0;
        for (int q = 0; q < L0.nSteps && q < 4; ++q) {
            int s0 = -1, cnt = 0;
            for (const Chunk& ch : L0.fwd[q])
                if (ch.sys == b) {
                    if (s0 < 0) s0 = ch.start;
                    cnt += ch.count;
                }
            if (s0 < 0) break;
            t.grpStart[q] = s0;
            t.grpCount[q] = cnt;
            t.nColours = q + 1;
        }
        if (first == 0 && L0.nSteps > 4) first = c;  // (never: level 0 is block-hybrid beyond 4 colours)
        if (cp.rowStart != t.rowStart[c]) throw Error(VLM_ERR_CUDA, "internal: coarse-tail row mismatch");
    }
    tailSys_.upload(ts, stream_);
    tailOn_ = true;
    planTailSmem(ts);
}

// Images of the shared-memory tail (buildTailImages): used when every tail system qualifies.
void DeviceBatch::planTailSmem(const std::vector<TailSys>& ts) {
    tailSmem_ = false;
    if (!tailSmemAllowed_ || tailCl_ != 1) return;
    int dev = 0, optin = 0;
    VLM_CUDA(cudaGetDevice(&dev));
    VLM_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const int budget = optin - int(sizeof(TailImg)) - 256;  // the kernel's static descriptor copy
    TailImages im;
    if (!buildTailImages(plan_, ts, size_t(budget), im)) return;
    tailImg_.upload(im.imgs, stream_);
    tailCodes_.upload(im.codes, stream_);
    tailStr_.upload(im.str, stream_);
    tailVal64_.resize(im.codes.size());
    tailVal32_.resize(im.codes.size());
    tailSmem64_ = im.bytes64;
    tailSmem32_ = im.bytes32;
    // the opt-in limit is a per-function setting: raised once to what the kernels may use
    static const bool raised = [budget] {
        VLM_CUDA(cudaFuncSetAttribute(k_vcycle_tail_smem<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, budget));
        VLM_CUDA(cudaFuncSetAttribute(k_vcycle_tail_smem<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, budget));
        return true;
    }();
    (void)raised;
    VLM_CUDA(cudaStreamSynchronize(stream_));  // the host vectors are locals
    tailSmem_ = true;
}

void DeviceBatch::recordPrecond(PrecondKind pk, SmootherKind sm, const double* r, double* w, bool f32) {
    DevLevel& D0 = L_[0];
    switch (pk) {
    case PrecondKind::GAMG:
        if (f32) {
            // FP32 V-cycle inside the FP64 Krylov recurrence
            VLM_LAUNCH((k_cast_rows<double, float>), D0.all.n, kRowsPerCta, stream_, D0.ch(D0.all), r, r32_.get(),
                       st_.get(), kFlagDone);
            recordVcycle<float>(r32_.get(), w32_.get(), sm, kFlagDone);
            VLM_LAUNCH((k_cast_rows<float, double>), D0.all.n, kRowsPerCta, stream_, D0.ch(D0.all), w32_.get(), w,
                       st_.get(), kFlagDone);
        } else {
            recordVcycle<double>(r, w, sm, kFlagDone);
        }
        break;
    case PrecondKind::Diagonal:
        VLM_LAUNCH(k_precond_diag<double>, D0.all.n, kRowsPerCta, stream_, D0.ch(D0.all), rD_.get(), r, w, st_.get(),
                   kFlagDone);
        break;
    case PrecondKind::None:
        VLM_LAUNCH(k_copy_rows<double>, D0.all.n, kRowsPerCta, stream_, D0.ch(D0.all), r, w, st_.get(), kFlagDone);
        break;
    case PrecondKind::DIC:
    case PrecondKind::DILU: recordDiluApply(r, w); break;
    default: throw Error(VLM_ERR_UNSUPPORTED, "preconditioner not available on the device");
    }
}

// ====================================================================== iteration bodies
void DeviceBatch::recordIter(const SolveKey& key) {
    const bool f32 = key.prec == Precision::MixedPrecond;
    if (key.solver == SolverKind::PCG)
        recordPcgIter(key.precond, key.smoother, f32);
    else if (key.solver == SolverKind::PBiCGStab)
        recordBicgIter(key.precond, key.smoother, f32);
    else
        recordRelaxIter(key);
}

// Eager iteration loop (no graph): same kernels launched directly, convergence read back per
// iteration.  Used when graphs are disabled (VLM_GRAPH=0), e.g. to profile single kernels.
void DeviceBatch::runEager(const SolveKey& key, int maxIter) {
    cudaStream_t s = stream_;
    auto anyActive = [&](int flag) {
        VLM_CUDA(cudaMemcpyAsync(hostState_.data(), st_.get(), sizeof(SysState) * plan_.nsys, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
        for (const auto& q : hostState_)
            if (!(flag == kFlagDone ? q.done : (q.done || q.innerDone))) return true;
        return false;
    };
    const int cap = 4 * (maxIter + 2);
    if (key.prec != Precision::MixedDC) {
        for (int it = 0; it < cap && anyActive(kFlagDone); ++it) recordIter(key);
        return;
    }
    DevLevel& D0 = L_[0];
    const Chunk* ch = D0.ch(D0.all);
    const int nb = D0.all.n;
    for (int o = 0; o < cap && anyActive(kFlagDone); ++o) {
        VLM_LAUNCH(k_inner_begin, nblk(plan_.nsys), 256, s, plan_.nsys, st_.get());
        VLM_LAUNCH(k_zero_rows<float>, nb, kRowsPerCta, s, ch, e32_.get(), st_.get(), kFlagInner);
        for (int it = 0; it < cap && anyActive(kFlagInner); ++it) recordInnerPcgIter(key.precond, key.smoother);
        recordMixedTail();
    }
}

void DeviceBatch::recordRefSetup() {
    DevLevel& D0 = L_[0];
    cudaStream_t s = stream_;
    const Chunk* ch = D0.ch(D0.all);
    const int nb = D0.all.n;
    if (dL32_.size() != size_t(D0.nrows)) dL32_.resize(size_t(D0.nrows));
    VLM_LAUNCH(k_ref_reset, nblk(plan_.nsys), 256, s, plan_.nsys, st_.get());
    VLM_LAUNCH(k_ref_detect, nb, kRowsPerCta, s, ch, D0.sell(), (const double*)D0.val.get(),
               (const double*)D0.diag.get(), (const int32_t*)perm0_.get(), st_.get());
    VLM_LAUNCH(k_ref_finish, nblk(plan_.nsys), 256, s, plan_.nsys, st_.get());
    VLM_LAUNCH(k_ref_diag32, nb, kRowsPerCta, s, ch, (const double*)D0.diag.get(), dL32_.get(),
               (const SysState*)st_.get());
    VLM_LAUNCH(k_ref_sum_r, nb, kRowsPerCta, s, ch, (const double*)r_.get(), red(), st_.get());
    VLM_LAUNCH(k_ref_rhs, nblk(plan_.nsys), 256, s, plan_.nsys, (const double*)r_.get(), r32_.get(),
               (const SysState*)st_.get());
}

void DeviceBatch::recordMixedTail() {
    DevLevel& D0 = L_[0];
    cudaStream_t s = stream_;
    const Chunk* ch = D0.ch(D0.all);
    const int nb = D0.all.n;
    VLM_LAUNCH(k_mixed_correct, nb, kRowsPerCta, s, ch, x_.get(), (const float*)e32_.get(),
               (const int32_t*)perm0_.get(), (const SysState*)st_.get());
    VLM_LAUNCH(k_mixed_residual, nb, kRowsPerCta, s, ch, D0.sell(), D0.val.get(), D0.diag.get(), x_.get(), b_.get(),
               r_.get(), r32_.get(), red(), st_.get(), dctrl_.get());
    VLM_LAUNCH(k_ref_rhs, nblk(plan_.nsys), 256, s, plan_.nsys, (const double*)r_.get(), r32_.get(),
               (const SysState*)st_.get());
}

void DeviceBatch::recordPcgIter(PrecondKind pk, SmootherKind sm, bool f32) {
    if (exact_)
        recordPcgIterT<true>(pk, sm, f32);
    else
        recordPcgIterT<false>(pk, sm, f32);
}

template <bool EXACT>
void DeviceBatch::recordPcgIterT(PrecondKind pk, SmootherKind sm, bool f32) {
    DevLevel& D0 = L_[0];
    cudaStream_t s = stream_;
    const Chunk* ch = D0.ch(D0.all);
    const int nb = D0.all.n;
    const bool v32 = f32 && pk == PrecondKind::GAMG;
    if (v32) {
        // FP32 V-cycle on r32 (written by the previous update / the initial residual); its FP32
        // output feeds the dot and the direction update directly
        recordVcycle<float>(r32_.get(), w32_.get(), sm, kFlagDone);
        VLM_LAUNCH((k_pcg_dot_wr<double, kFlagDone, EXACT, float>), nb, kRowsPerCta, s, ch, w32_.get(), r_.get(), red(),
                   st_.get());
        VLM_LAUNCH((k_pcg_p<double, kFlagDone, float>), nb, kRowsPerCta, s, ch, w32_.get(), p_.get(), st_.get());
    } else {
        recordPrecond(pk, sm, r_.get(), w_.get(), f32);
        VLM_LAUNCH((k_pcg_dot_wr<double, kFlagDone, EXACT>), nb, kRowsPerCta, s, ch, w_.get(), r_.get(), red(),
                   st_.get());
        VLM_LAUNCH((k_pcg_p<double, kFlagDone>), nb, kRowsPerCta, s, ch, w_.get(), p_.get(), st_.get());
    }
    if (boxOn_) {
        int g = 0;
        const BoxRows R = boxRows(D0, D0.all, &g);
        const StreamShape* sh = EXACT ? nullptr : streamShape<double>(R);
        if (sh)
            VLM_LAUNCH_SMEM((k_box_pcg_spmv_stream<double, kFlagDone>), sh->grid, sh->threads, sh->smem, s, R.one,
                            sh->TY, sh->S, (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(),
                            (const double*)p_.get(), Ap_.get(), red(), st_.get(), &sweepSync_.get()->err);
        else if (R.ch == nullptr && R.one.H % 4 == 0)
            VLM_LAUNCH((k_box_pcg_spmv4<double, kFlagDone, EXACT>), nb, kRowsPerCta, s, ch, R.one,
                       (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(),
                       (const double*)p_.get(), Ap_.get(), red(), st_.get());
        else
            VLM_LAUNCH((k_box_pcg_spmv<double, kFlagDone, EXACT>), nb, kRowsPerCta, s, ch, R,
                       (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(),
                       (const double*)p_.get(), Ap_.get(), red(), st_.get());
    }
    else
        VLM_LAUNCH((k_pcg_spmv<double, kFlagDone, EXACT>), nb, kRowsPerCta, s, ch, D0.sell(), D0.val.get(),
                   D0.diag.get(), p_.get(), Ap_.get(), red(), st_.get());
    VLM_LAUNCH((k_pcg_update<double, kFlagDone, EXACT>), nb, kRowsPerCta, s, ch, x_.get(), r_.get(), p_.get(),
               Ap_.get(), perm0_.get(), red(), st_.get(), dctrl_.get(), v32 ? r32_.get() : (float*)nullptr);
}

void DeviceBatch::recordInnerPcgIter(PrecondKind pk, SmootherKind sm) {
    DevLevel& D0 = L_[0];
    cudaStream_t s = stream_;
    const Chunk* ch = D0.ch(D0.all);
    const int nb = D0.all.n;
    if (pk == PrecondKind::GAMG)
        recordVcycle<float>(r32_.get(), w32_.get(), sm, kFlagInner);
    else if (pk == PrecondKind::Diagonal)
        VLM_LAUNCH(k_precond_diag<float>, nb, kRowsPerCta, s, ch, rD32_.get(), r32_.get(), w32_.get(), st_.get(),
                   kFlagInner);
    else
        throw Error(VLM_ERR_UNSUPPORTED, "mixed precision needs the GAMG or diagonal preconditioner");
    // the inner operator is L (A without the reference row's refC) and the constant mode is projected
    // out of the preconditioned residual; without a reference row both reduce to A and no projection
    VLM_LAUNCH(k_inner_dot_wr, nb, kRowsPerCta, s, ch, (const float*)w32_.get(), (const float*)r32_.get(),
               (const int32_t*)perm0_.get(), (const int*)sysCells_.get(), red(), st_.get());
    VLM_LAUNCH(k_inner_p, nb, kRowsPerCta, s, ch, (const float*)w32_.get(), p32_.get(), (const int32_t*)perm0_.get(),
               (const SysState*)st_.get());
    const float* dL = dL32_.get();
    if (boxOn_) {
        int g = 0;
        const BoxRows R = boxRows(D0, D0.all, &g);
        if (R.ch == nullptr && R.one.H % 4 == 0)
            VLM_LAUNCH((k_box_pcg_spmv4<float, kFlagInner, false>), nb, kRowsPerCta, s, ch, R.one,
                       (const float*)D0.bcoef32.get(), D0.nrows, dL, (const float*)p32_.get(), Ap32_.get(), red(),
                       st_.get());
        else
            VLM_LAUNCH((k_box_pcg_spmv<float, kFlagInner, false>), nb, kRowsPerCta, s, ch, R,
                       (const float*)D0.bcoef32.get(), D0.nrows, dL, (const float*)p32_.get(), Ap32_.get(), red(),
                       st_.get());
    }
    else
        VLM_LAUNCH((k_pcg_spmv<float, kFlagInner, false>), nb, kRowsPerCta, s, ch, D0.sell(), D0.val32.get(), dL,
                   p32_.get(), Ap32_.get(), red(), st_.get());
    VLM_LAUNCH((k_pcg_update<float, kFlagInner, false>), nb, kRowsPerCta, s, ch, e32_.get(), r32_.get(), p32_.get(),
               Ap32_.get(), perm0_.get(), red(), st_.get(), dctrl_.get(), (float*)nullptr);
}

void DeviceBatch::recordBicgIter(PrecondKind pk, SmootherKind sm, bool f32) {
    if (exact_)
        recordBicgIterT<true>(pk, sm, f32);
    else
        recordBicgIterT<false>(pk, sm, f32);
}

template <bool EXACT>
void DeviceBatch::recordBicgIterT(PrecondKind pk, SmootherKind sm, bool f32) {
    DevLevel& D0 = L_[0];
    cudaStream_t s = stream_;
    const Chunk* ch = D0.ch(D0.all);
    const int nb = D0.all.n;
    SysState* st = st_.get();
    VLM_LAUNCH(k_bicg_rho<EXACT>, nb, kRowsPerCta, s, ch, r0_.get(), r_.get(), red(), st);
    VLM_LAUNCH(k_bicg_p, nb, kRowsPerCta, s, ch, r_.get(), Ay_.get(), p_.get(), st);
    recordPrecond(pk, sm, p_.get(), y_.get(), f32);
    VLM_LAUNCH(k_bicg_spmv_alpha<EXACT>, nb, kRowsPerCta, s, ch, D0.sell(), D0.val.get(), D0.diag.get(), y_.get(), Ay_.get(),
               r0_.get(), red(), st);
    VLM_LAUNCH(k_bicg_s<EXACT>, nb, kRowsPerCta, s, ch, r_.get(), Ay_.get(), s_.get(), red(), st, dctrl_.get());
    VLM_LAUNCH(k_bicg_early, nb, kRowsPerCta, s, ch, x_.get(), y_.get(), st);
    VLM_LAUNCH(k_bicg_early_close, nblk(plan_.nsys), 256, s, plan_.nsys, st);
    recordPrecond(pk, sm, s_.get(), z_.get(), f32);
    VLM_LAUNCH(k_bicg_spmv_omega<EXACT>, nb, kRowsPerCta, s, ch, D0.sell(), D0.val.get(), D0.diag.get(), z_.get(), t_.get(),
               s_.get(), red(), st);
    VLM_LAUNCH(k_bicg_update<EXACT>, nb, kRowsPerCta, s, ch, x_.get(), r_.get(), y_.get(), z_.get(), s_.get(), t_.get(), red(),
               st, dctrl_.get());
}

// ====================================================================== level-scheduled paths
void DeviceBatch::ensureDilu() {
    if (dilu_) return;
    const DiluPlan P = buildDiluPlan(topo_, plan_);
    auto D = std::make_unique<DiluDev>();
    cudaStream_t s = stream_;
    D->loPtr.upload(P.loPtr, s);
    D->loCol.upload(P.loCol, s);
    D->loFace.upload(P.loFace, s);
    D->upPtr.upload(P.upPtr, s);
    D->upCol.upload(P.upCol, s);
    D->upFace.upload(P.upFace, s);
    D->levPtr.upload(P.levPtr, s);
    D->levRows.upload(P.levRows, s);
    D->sys.upload(P.sys, s);
    D->nFaces = int(P.loCol.size());
    const size_t nf = size_t(std::max(D->nFaces, 1));
    D->loAul.resize(nf);
    D->loAlu.resize(nf);
    D->upAlu.resize(nf);
    D->rD.resize(size_t(L_[0].nrows));
    D->groups = int(P.sys.size());
    // one CTA per system; a single wide system gets a co-resident group of CTAs
    D->G = 1;
    if (D->groups == 1 && P.maxWidth > 2 * kDiluThreads) {
        int dev = 0, sms = 0, per = 0;
        VLM_CUDA(cudaGetDevice(&dev));
        VLM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        VLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dilu_apply, kDiluThreads, 0));
        int perF = 0, perG = 0;
        VLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perF, k_dilu_factor, kDiluThreads, 0));
        VLM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perG, k_gs_sweep, kDiluThreads, 0));
        const int resident = sms * std::max(1, std::min(per, std::min(perF, perG)));
        D->G = std::max(1, std::min({(P.maxWidth + kDiluThreads - 1) / kDiluThreads, resident, sms}));
    }
    // shared-memory sweeps: one CTA per system, every level at most one row per thread, the vector
    // of the largest system within the opt-in shared memory
    // (the kernels' opt-in limit is a per-function setting shared by every mesh: it is raised once to
    // the ceiling, never to one mesh's size)
    constexpr size_t kDiluSmemMax = 200 * 1024;
    const int W = std::max(1, P.maxWidth), M = std::max(1, P.maxEnt);
    const size_t streamSmem = dilu_stream_smem(P.maxRows, P.maxLevels, W, M);
    if (D->G == 1 && P.maxWidth <= kDiluThreads && streamSmem <= kDiluSmemMax) {
        static const bool raised = [] {
            VLM_CUDA(cudaFuncSetAttribute(k_dilu_factor_stream, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(kDiluSmemMax)));
            VLM_CUDA(cudaFuncSetAttribute(k_dilu_apply_stream, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          int(kDiluSmemMax)));
            return true;
        }();
        (void)raised;
        D->smem = streamSmem;
        D->threads = std::max(32, (P.maxWidth + 31) / 32 * 32);
        D->W = W;
        D->M = M;
        D->lev.upload(P.lev, s);
        D->slotRow.upload(P.slotRow, s);
        D->sLoCol.upload(P.sLoCol, s);
        D->sLoFace.upload(P.sLoFace, s);
        D->sUpCol.upload(P.sUpCol, s);
        D->sUpFace.upload(P.sUpFace, s);
        D->nLoS = int(P.sLoCol.size());
        D->nUpS = int(P.sUpCol.size());
        D->prod.resize(size_t(std::max(D->nLoS, 1)));
        D->coefLo.resize(size_t(std::max(D->nLoS, 1)));
        D->coefUp.resize(size_t(std::max(D->nUpS, 1)));
        D->rDs.resize(std::max<size_t>(P.slotRow.size(), 1));
    }
    D->bars.resize(size_t(D->groups));
    D->bars.zero(s);
    D->err.resize(1);
    D->err.zero(s);
    VLM_CUDA(cudaStreamSynchronize(s));
    dilu_ = std::move(D);
}

namespace {
// Launch of a level-scheduled kernel: groups x G CTAs, cooperative when a group spans CTAs.
template <class... Exp, class... Act>
void launchLevels(void (*kernel)(Exp...), int groups, int G, cudaStream_t s, Act&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(groups * G));
    cfg.blockDim = dim3(unsigned(kDiluThreads));
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = G > 1 ? 1 : 0;
    VLM_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Act>(args)...));
    ++tl_launches;
}
}  // namespace

void DeviceBatch::diluFactor(const double* upper, const double* lower) {
    DiluDev& Dd = *dilu_;
    cudaStream_t s = stream_;
    if (Dd.smem) {
        VLM_LAUNCH(k_dilu_stream_values, nblk(std::max(1, Dd.nLoS + Dd.nUpS)), 256, s, Dd.nLoS, Dd.nUpS,
                   (const int32_t*)Dd.sLoCol.get(), (const int32_t*)Dd.sLoFace.get(), (const int32_t*)Dd.sUpCol.get(),
                   (const int32_t*)Dd.sUpFace.get(), upper, lower, Dd.prod.get(), Dd.coefLo.get(), Dd.coefUp.get());
        k_dilu_factor_stream<<<Dd.groups, Dd.threads, Dd.smem, s>>>(Dd.sys.get(), Dd.lev.get(), Dd.W, Dd.M,
                                                                      Dd.slotRow.get(), Dd.sLoCol.get(), Dd.prod.get(),
                                                                      L_[0].diag.get(), Dd.rDs.get());
        VLM_CUDA(cudaGetLastError());
        ++tl_launches;
        return;
    }
    VLM_LAUNCH(k_dilu_values, nblk(Dd.nFaces), 256, s, Dd.nFaces, (const int32_t*)Dd.loFace.get(),
               (const int32_t*)Dd.upFace.get(), upper, lower, Dd.loAul.get(), Dd.loAlu.get(), Dd.upAlu.get());
    launchLevels(k_dilu_factor, Dd.groups, Dd.G, s, (const DiluSys*)Dd.sys.get(), Dd.G, (const int32_t*)Dd.levPtr.get(),
                 (const int32_t*)Dd.levRows.get(), (const int32_t*)Dd.loPtr.get(), (const int32_t*)Dd.loCol.get(),
                 (const double*)Dd.loAlu.get(), (const double*)Dd.loAul.get(), (const double*)L_[0].diag.get(),
                 Dd.rD.get(), Dd.bars.get(), Dd.err.get());
}

void DeviceBatch::clearLevelError() {
    if (sweepSync_.size() != 0) VLM_CUDA(cudaMemsetAsync(&sweepSync_.get()->err, 0, sizeof(unsigned), stream_));
    if (!dilu_) return;
    dilu_->err.zero(stream_);
    dilu_->bars.zero(stream_);
}

// A group barrier of a level-scheduled kernel that gave up leaves its status here.
void DeviceBatch::checkLevelError() {
    int e = 0;
    VLM_CUDA(cudaMemcpy(&e, dilu_->err.get(), sizeof(int), cudaMemcpyDeviceToHost));
    if (e != 0) {
        dilu_->err.zero(stream_);
        dilu_->bars.zero(stream_);
        VLM_CUDA(cudaStreamSynchronize(stream_));
        throw Error(VLM_ERR_TIMEOUT, "level-scheduled sweep: a group barrier wait gave up");
    }
}

void DeviceBatch::recordDiluApply(const double* r, double* w) {
    DiluDev& D = *dilu_;
    if (D.smem) {
        k_dilu_apply_stream<<<D.groups, D.threads, D.smem, stream_>>>(
            D.sys.get(), D.lev.get(), D.W, D.M, D.slotRow.get(), D.rDs.get(), D.sLoCol.get(), D.coefLo.get(),
            D.sUpCol.get(), D.coefUp.get(), r, w, st_.get(), kFlagDone);
        VLM_CUDA(cudaGetLastError());
        ++tl_launches;
        return;
    }
    launchLevels(k_dilu_apply, D.groups, D.G, stream_, (const DiluSys*)D.sys.get(), D.G, (const int32_t*)D.levPtr.get(),
                 (const int32_t*)D.levRows.get(), (const int32_t*)D.loPtr.get(), (const int32_t*)D.loCol.get(),
                 (const double*)D.loAul.get(), (const int32_t*)D.upPtr.get(), (const int32_t*)D.upCol.get(),
                 (const double*)D.upAlu.get(), (const double*)D.rD.get(), r, w, D.bars.get(), D.err.get(),
                 (const SysState*)st_.get(), int(kFlagDone));
}

// Gauss-Seidel / symmetric Gauss-Seidel / Jacobi: nSweeps sweeps, then the residual and the
// convergence test (LinearSolver.cpp:238-278)
void DeviceBatch::recordRelaxIter(const SolveKey& key) {
    if (exact_)
        recordRelaxIterT<true>(key);
    else
        recordRelaxIterT<false>(key);
}

template <bool EXACT>
void DeviceBatch::recordRelaxIterT(const SolveKey& key) {
    DevLevel& D0 = L_[0];
    cudaStream_t s = stream_;
    const Chunk* ch = D0.ch(D0.all);
    const int nb = D0.all.n;
    for (int sw = 0; sw < key.nSweeps; ++sw) {
        if (key.solver == SolverKind::Jacobi) {
            VLM_LAUNCH((k_smooth_jacobi<double, 0>), nb, kRowsPerCta, s, ch, D0.sell(), D0.val.get(), D0.diag.get(),
                       b_.get(), x_.get(), w_.get(), 1.0, (const int32_t*)nullptr, (const double*)nullptr, st_.get(),
                       kFlagDone);
            VLM_LAUNCH(k_copy_rows<double>, nb, kRowsPerCta, s, ch, w_.get(), x_.get(), st_.get(), kFlagDone);
        } else {
            DiluDev& D = *dilu_;
            for (int dir = 0; dir < (key.solver == SolverKind::SymGaussSeidel ? 2 : 1); ++dir)
                launchLevels(k_gs_sweep, D.groups, D.G, s, (const DiluSys*)D.sys.get(), D.G,
                             (const int32_t*)D.levPtr.get(), (const int32_t*)D.levRows.get(), D0.sell(),
                             (const double*)D0.val.get(), (const double*)D0.diag.get(), (const double*)b_.get(),
                             x_.get(), dir, D.bars.get(), D.err.get(), (const SysState*)st_.get(), int(kFlagDone));
        }
    }
    VLM_LAUNCH(k_relax_residual<EXACT>, nb, kRowsPerCta, s, ch, D0.sell(), D0.val.get(), D0.diag.get(), x_.get(),
               b_.get(), perm0_.get(), key.nSweeps, red(), st_.get(), dctrl_.get());
}

void DeviceBatch::recordSetCond(cudaGraphConditionalHandle h, int flag) {
    k_set_cond<<<1, 256, 0, stream_>>>(h, plan_.nsys, st_.get(), flag);
    ++tl_launches;
}

// ====================================================================== graphs
namespace {

// Stream-captures `body` into graph g after `deps`; returns the new leaf node.
template <class F>
cudaGraphNode_t captureInto(cudaStream_t s, cudaGraph_t g, const std::vector<cudaGraphNode_t>& deps, F&& body) {
    const auto before = nodesOf(g);
    const std::set<cudaGraphNode_t> old(before.begin(), before.end());
    VLM_CUDA(cudaStreamBeginCaptureToGraph(s, g, deps.empty() ? nullptr : deps.data(), nullptr, deps.size(),
                                           cudaStreamCaptureModeRelaxed));
    try {
        body();
    } catch (...) {
        cudaGraph_t junk;
        cudaStreamEndCapture(s, &junk);
        throw;
    }
    cudaGraph_t out;
    VLM_CUDA(cudaStreamEndCapture(s, &out));
    cudaGraphNode_t leaf = nullptr;
    for (cudaGraphNode_t n : nodesOf(g)) {
        if (old.count(n)) continue;
        size_t nd = 0;
        VLM_CUDA(cudaGraphNodeGetDependentNodes(n, nullptr, &nd));
        if (nd == 0) leaf = n;
    }
    if (!leaf) throw Error(VLM_ERR_CUDA, "graph capture produced no nodes");
    return leaf;
}

cudaGraphNode_t addWhile(cudaGraph_t g, cudaGraphNode_t dep, cudaGraphConditionalHandle h, cudaGraph_t* body) {
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    VLM_CUDA(cudaGraphAddNode(&node, g, dep ? &dep : nullptr, dep ? 1 : 0, &p));
    *body = p.conditional.phGraph_out[0];
    return node;
}

}  // namespace

void DeviceBatch::buildGraph(const SolveKey& key, GraphExec& G) {
    struct CaptureScope {
        bool was;
        CaptureScope() : was(tl_capturing) { tl_capturing = true; }
        ~CaptureScope() { tl_capturing = was; }
    } scope;
    // while stream_ is itself being captured, the solve's graph is recorded on the side stream
    std::unique_ptr<StreamSwap> swap;
    if (embedding_) swap = std::make_unique<StreamSwap>(this, side_);
    VLM_CUDA(cudaGraphCreate(&G.graph, 0));
    cudaStream_t s = stream_;
    const int64_t saved = tl_launches;
    int64_t mark = tl_launches;
    auto segment = [&]() {
        const int64_t k = tl_launches - mark;
        mark = tl_launches;
        return k;
    };
    if (key.prec != Precision::MixedDC) {
        cudaGraphConditionalHandle h;
        VLM_CUDA(cudaGraphConditionalHandleCreate(&h, G.graph, 0, cudaGraphCondAssignDefault));
        cudaGraphNode_t pre = captureInto(s, G.graph, {}, [&] { recordSetCond(h, kFlagDone); });
        G.preK = segment();
        cudaGraph_t body;
        addWhile(G.graph, pre, h, &body);
        captureInto(s, body, {}, [&] {
            recordIter(key);
            recordSetCond(h, kFlagDone);
        });
        G.bodyK = segment();
    } else {
        cudaGraphConditionalHandle ho;
        VLM_CUDA(cudaGraphConditionalHandleCreate(&ho, G.graph, 0, cudaGraphCondAssignDefault));
        cudaGraphNode_t pre = captureInto(s, G.graph, {}, [&] { recordSetCond(ho, kFlagDone); });
        G.preK = segment();
        cudaGraph_t outer;
        addWhile(G.graph, pre, ho, &outer);
        cudaGraphConditionalHandle hi;
        VLM_CUDA(cudaGraphConditionalHandleCreate(&hi, outer, 0, cudaGraphCondAssignDefault));
        DevLevel& D0 = L_[0];
        const Chunk* ch = D0.ch(D0.all);
        const int nb = D0.all.n;
        cudaGraphNode_t seg1 = captureInto(s, outer, {}, [&] {
            VLM_LAUNCH(k_inner_begin, nblk(plan_.nsys), 256, s, plan_.nsys, st_.get());
            VLM_LAUNCH(k_zero_rows<float>, nb, kRowsPerCta, s, ch, e32_.get(), st_.get(), kFlagInner);
            recordSetCond(hi, kFlagInner);
        });
        G.bodyK = segment();
        cudaGraph_t inner;
        cudaGraphNode_t w = addWhile(outer, seg1, hi, &inner);
        captureInto(s, inner, {}, [&] {
            recordInnerPcgIter(key.precond, key.smoother);
            recordSetCond(hi, kFlagInner);
        });
        G.innerK = segment();
        captureInto(s, outer, {w}, [&] {
            recordMixedTail();
            recordSetCond(ho, kFlagDone);
        });
        G.bodyK += segment();
    }
    tl_launches = saved;
    VLM_CUDA(cudaGraphInstantiate(&G.exec, G.graph, 0));
}

// The solve's loop inside the graph the caller is capturing on stream_: the entry kernel that sets
// the loop condition, a WHILE node after the capture's current dependencies, and the loop body
// captured into the node's body graph on the side stream (the same nodes buildGraph records).
void DeviceBatch::embedSolve(const SolveKey& key) {
    VLM_REQUIRE(key.prec != Precision::MixedDC, VLM_ERR_UNSUPPORTED,
                "defect-correction solves are not embedded in a captured step");
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    VLM_CUDA(cudaStreamGetCaptureInfo(stream_, &cs, nullptr, &cg, &deps, &nd));
    VLM_REQUIRE(cs == cudaStreamCaptureStatusActive, VLM_ERR_CUDA, "internal: embedding without a capture");
    cudaGraphConditionalHandle h;
    VLM_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 0, cudaGraphCondAssignDefault));
    recordSetCond(h, kFlagDone);
    VLM_CUDA(cudaStreamGetCaptureInfo(stream_, &cs, nullptr, &cg, &deps, &nd));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t w;
    VLM_CUDA(cudaGraphAddNode(&w, cg, deps, nd, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    VLM_CUDA(cudaStreamUpdateCaptureDependencies(stream_, &w, 1, cudaStreamSetCaptureDependencies));
    StreamSwap swap(this, side_);
    captureInto(side_, body, {}, [&] {
        recordIter(key);
        recordSetCond(h, kFlagDone);
    });
}

GraphExec& DeviceBatch::graphFor(const SolveKey& key) {
    auto it = graphs_.find(key);
    if (it != graphs_.end()) return *it->second;
    auto g = std::make_unique<GraphExec>();
    buildGraph(key, *g);
    GraphExec& ref = *g;
    graphs_.emplace(key, std::move(g));
    return ref;
}

// ====================================================================== entry points
void DeviceBatch::solve(const double* diag, const double* upper, const double* lower, const double* b, double* x,
                        const vlm_solver_ctrl& ctrl, std::vector<vlm_solver_perf>& perfOut) {
    cudaStream_t s = stream_;
    SolverKind sk = parseSolver(ctrl.solver);
    PrecondKind pk = parsePrecond(ctrl.preconditioner);
    if (ctrl.reproducible) {
        // CFD_REPRODUCIBLE semantics (LinearSolver.cpp:138-148)
        if (pk != PrecondKind::None) pk = PrecondKind::Diagonal;
        if (sk == SolverKind::GaussSeidel || sk == SolverKind::SymGaussSeidel) sk = SolverKind::Jacobi;
    }
    const bool symmetric = lower == upper;
    if (sk == SolverKind::PCG && !symmetric)
        throw Error(VLM_ERR_UNSUPPORTED, "PCG requires a symmetric matrix; use PBiCGStab");
    if (sk == SolverKind::PBiCGStab && pk == PrecondKind::DIC) pk = PrecondKind::DILU;
    const bool relax = sk != SolverKind::PCG && sk != SolverKind::PBiCGStab;
    if (relax) {
        // the relaxation solvers use no preconditioner; nSweeps < 1 would never advance the
        // iteration count (LinearSolver.cpp:260-277)
        pk = PrecondKind::None;
        if (ctrl.nSweeps < 1) throw Error(VLM_ERR_BAD_ARG, "nSweeps must be at least 1 for the relaxation solvers");
    }
    const bool levelSchedule = pk == PrecondKind::DIC || pk == PrecondKind::DILU || sk == SolverKind::GaussSeidel ||
                               sk == SolverKind::SymGaussSeidel;
    if (levelSchedule) ensureDilu();
    const SmootherKind sm = parseSmoother(ctrl.smoother);
    Precision prec = Precision::FP64;
    if (eq(ctrl.precision, "mixed"))
        prec = Precision::MixedPrecond;
    else if (eq(ctrl.precision, "mixed-dc"))
        prec = Precision::MixedDC;
    else if (ctrl.precision[0] != 0 && !eq(ctrl.precision, "fp64"))
        throw Error(VLM_ERR_BAD_ARG, std::string("unknown precision ") + ctrl.precision);
    if (prec == Precision::MixedPrecond && pk != PrecondKind::GAMG) prec = Precision::FP64;  // nothing to lower
    if (prec == Precision::MixedDC && sk != SolverKind::PCG)
        throw Error(VLM_ERR_UNSUPPORTED, "defect-correction mixed precision is implemented for PCG");
    if (prec == Precision::MixedDC && pk == PrecondKind::None)
        throw Error(VLM_ERR_UNSUPPORTED, "mixed precision needs a preconditioner");
    const bool mixed = prec != Precision::FP64;
    const bool dc = prec == Precision::MixedDC;
    ensureVectors(mixed, sk == SolverKind::PBiCGStab);
    const int64_t launch0 = tl_launches;

    setupMatrix(diag, upper, lower, pk == PrecondKind::GAMG, mixed);
    DevLevel& D0 = L_[0];
    const int n0 = D0.nrows;
    // DIC/DILU factorisation per solve (the coefficients change), before the iteration loop
    if (pk == PrecondKind::DIC || pk == PrecondKind::DILU) diluFactor(upper, lower);
    if (pk == PrecondKind::Diagonal) {
        if (rD_.size() != size_t(n0)) rD_.resize(n0);
        VLM_LAUNCH(k_recip_diag<double>, nblk(n0), 256, s, n0, perm0_.get(), D0.diag.get(), rD_.get());
        if (mixed) {
            if (rD32_.size() != size_t(n0)) rD32_.resize(n0);
            VLM_LAUNCH(k_recip_diag<float>, nblk(n0), 256, s, n0, perm0_.get(), D0.diag32.get(), rD32_.get());
        }
    }
    // the controls travel as kernel arguments: a copy from pageable host memory would wait for
    // the stream and stop the host from running ahead
    DevCtrl hc;
    hc.tolerance = ctrl.tolerance;
    hc.relTol = ctrl.relTol;
    hc.innerRelTol = ctrl.innerRelTol > 0 ? ctrl.innerRelTol : 1e-4;
    hc.maxIter = ctrl.maxIter;
    hc.minIter = ctrl.minIter;
    hc.maxInner = ctrl.maxIter;
    VLM_LAUNCH(k_set_ctrl, 1, 1, s, dctrl_.get(), hc);
    st_.zero(s);
    // b and x may still be arriving on another stream while the matrix was set up
    if (inputsReady_) {
        VLM_CUDA(cudaStreamWaitEvent(s, inputsReady_, 0));
        inputsReady_ = nullptr;
    }
    VLM_LAUNCH(k_to_solver<double>, nblk(n0), 256, s, n0, perm0_.get(), x, x_.get());
    VLM_LAUNCH(k_to_solver<double>, nblk(n0), 256, s, n0, perm0_.get(), b, b_.get());
    exact_ = ctrl.reproducible != 0;
    if (exact_ && xbins_.size() == 0) {
        xbins_.resize(size_t(plan_.nSlots) * 2 * 73);
        xbins_.zero(s);
    }
    // FP32 copy of the initial residual: the inner solve's RHS (mixed-dc) or the first FP32 V-cycle's input
    const bool r32first = dc || (prec == Precision::MixedPrecond && sk == SolverKind::PCG && pk == PrecondKind::GAMG);
    if (exact_) {
        VLM_LAUNCH((k_sum_x<double, true>), D0.all.n, kRowsPerCta, s, D0.ch(D0.all), x_.get(), red(), st_.get());
        VLM_LAUNCH(k_init_residual<true>, D0.all.n, kRowsPerCta, s, D0.ch(D0.all), D0.sell(), D0.val.get(),
                   D0.diag.get(), x_.get(), b_.get(), perm0_.get(), r_.get(), r32first ? r32_.get() : nullptr,
                   sysCells_.get(), red(), st_.get(), dctrl_.get());
    } else {
        VLM_LAUNCH((k_sum_x<double, false>), D0.all.n, kRowsPerCta, s, D0.ch(D0.all), x_.get(), red(), st_.get());
        VLM_LAUNCH(k_init_residual<false>, D0.all.n, kRowsPerCta, s, D0.ch(D0.all), D0.sell(), D0.val.get(),
                   D0.diag.get(), x_.get(), b_.get(), perm0_.get(), r_.get(), r32first ? r32_.get() : nullptr,
                   sysCells_.get(), red(), st_.get(), dctrl_.get());
    }
    if (dc) recordRefSetup();
    if (sk == SolverKind::PBiCGStab) {
        VLM_CUDA(cudaMemcpyAsync(r0_.get(), r_.get(), sizeof(double) * n0, cudaMemcpyDeviceToDevice, s));
        Ay_.zero(s);
        p_.zero(s);
    }
    const SolveKey key{sk, pk, sm, prec, exact_, relax ? ctrl.nSweeps : 0, boxOn_};
    int64_t eagerLaunches = 0;
    GraphExec* Gp = nullptr;
    if (useGraphs_ && !(timeSweeps_ && !embedding_)) {
        Gp = &graphFor(key);
        if (embedding_)
            embedSolve(key);
        else
            VLM_CUDA(cudaGraphLaunch(Gp->exec, s));
    } else {
        const int64_t e0 = tl_launches;
        runEager(key, ctrl.maxIter);
        eagerLaunches = tl_launches - e0;
        tl_launches = e0;
    }
    VLM_LAUNCH(k_from_solver, nblk(n0), 256, s, n0, perm0_.get(), x_.get(), x);
    if (deferState_) {
        SysState* so = deferState_;
        int* sto = deferStatus_;
        deferState_ = nullptr;
        deferStatus_ = nullptr;
        lastDeferred_.eager = (tl_launches - launch0) + eagerLaunches;
        lastDeferred_.pre = Gp ? Gp->preK : 0;
        lastDeferred_.body = Gp ? Gp->bodyK : 0;
        VLM_CUDA(cudaMemcpyAsync(so, st_.get(), sizeof(SysState) * plan_.nsys, cudaMemcpyDeviceToDevice, s));
        // the coarse-factor status belongs to GAMG solves only (status_ is not reset for the others)
        if (pk == PrecondKind::GAMG)
            VLM_CUDA(cudaMemcpyAsync(sto, status_.get(), sizeof(int), cudaMemcpyDeviceToDevice, s));
        else
            VLM_CUDA(cudaMemsetAsync(sto, 0, sizeof(int), s));
        if (levelSchedule)
            VLM_CUDA(cudaMemcpyAsync(sto + 1, dilu_->err.get(), sizeof(int), cudaMemcpyDeviceToDevice, s));
        else if (sweepSync_.size() != 0)
            VLM_CUDA(cudaMemcpyAsync(sto + 1, &sweepSync_.get()->err, sizeof(int), cudaMemcpyDeviceToDevice, s));
        else
            VLM_CUDA(cudaMemsetAsync(sto + 1, 0, sizeof(int), s));
        return;
    }
    int coarseStatus = 0;
    VLM_CUDA(cudaMemcpyAsync(hostState_.data(), st_.get(), sizeof(SysState) * plan_.nsys, cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaMemcpyAsync(&coarseStatus, status_.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaStreamSynchronize(s));
    // executed kernels: the eager setup + the graph's pre-node + one body per loop pass
    int64_t iters = 0, outers = 0;
    for (int bpos = 0; bpos < plan_.nsys; ++bpos) {
        iters = std::max<int64_t>(iters, hostState_[bpos].iterations);
        outers = std::max<int64_t>(outers, hostState_[bpos].outer);
    }
    if (Gp)
        launches_ += (tl_launches - launch0) + Gp->preK + (dc ? outers * Gp->bodyK + iters * Gp->innerK : iters * Gp->bodyK);
    else
        launches_ += (tl_launches - launch0) + eagerLaunches;
    if (pk == PrecondKind::GAMG && coarseStatus == VLM_ERR_SINGULAR)
        throw Error(VLM_ERR_SINGULAR, "GAMG: singular coarsest matrix");
    if (levelSchedule) checkLevelError();
    checkSweepError();
    collectSweepTimes();
    perfOut.resize(size_t(plan_.nsys));
    for (int bpos = 0; bpos < plan_.nsys; ++bpos) {
        const SysState& q = hostState_[bpos];
        vlm_solver_perf p = {};
        p.initialResidual = q.initialResidual;
        p.finalResidual = q.finalResidual;
        p.residualSum = q.residualSum;
        p.normFactor = q.normFactor;
        p.iterations = q.iterations;
        p.outerIterations = q.outer;
        p.status = q.status;
        // converged() evaluated once more at exit (LinearSolver.cpp:283)
        p.converged = (p.iterations >= ctrl.minIter) &&
                      (p.finalResidual < ctrl.tolerance ||
                       (ctrl.relTol > 0 && p.finalResidual < ctrl.relTol * p.initialResidual));
        std::snprintf(p.solver, sizeof(p.solver), "%s", sk == SolverKind::PCG ? "PCG" : "PBiCGStab");
        perfOut[size_t(plan_.order[bpos])] = p;
    }
}

void DeviceBatch::amul(const double* diag, const double* upper, const double* lower, const double* x, double* y) {
    cudaStream_t s = stream_;
    setupMatrix(diag, upper, lower, false, false);
    DevLevel& D0 = L_[0];
    const int n0 = D0.nrows;
    VLM_LAUNCH(k_to_solver<double>, nblk(n0), 256, s, n0, perm0_.get(), x, x_.get());
    VLM_LAUNCH(k_amul, D0.all.n, kRowsPerCta, s, D0.ch(D0.all), D0.sell(), D0.val.get(), D0.diag.get(), x_.get(),
               w_.get());
    VLM_LAUNCH(k_from_solver, nblk(n0), 256, s, n0, perm0_.get(), w_.get(), y);
    VLM_CUDA(cudaStreamSynchronize(s));
}

void DeviceBatch::gamgApply(const double* diag, const double* upper, const double* lower, const double* r, double* w,
                            SmootherKind sm) {
    cudaStream_t s = stream_;
    setupMatrix(diag, upper, lower, true, false);
    DevLevel& D0 = L_[0];
    const int n0 = D0.nrows;
    st_.zero(s);
    VLM_LAUNCH(k_to_solver<double>, nblk(n0), 256, s, n0, perm0_.get(), r, r_.get());
    recordVcycle<double>(r_.get(), w_.get(), sm, kFlagDone);
    VLM_LAUNCH(k_from_solver, nblk(n0), 256, s, n0, perm0_.get(), w_.get(), w);
    int coarseStatus = 0;
    VLM_CUDA(cudaMemcpyAsync(&coarseStatus, status_.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaStreamSynchronize(s));
    if (coarseStatus == VLM_ERR_SINGULAR) throw Error(VLM_ERR_SINGULAR, "GAMG: singular coarsest matrix");
}

void DeviceBatch::precondApply(const double* diag, const double* upper, const double* lower, const double* r,
                               double* w, const vlm_solver_ctrl& ctrl) {
    const PrecondKind pk = parsePrecond(ctrl.preconditioner);
    if (pk == PrecondKind::GAMG) {
        gamgApply(diag, upper, lower, r, w, parseSmoother(ctrl.smoother));
        return;
    }
    cudaStream_t s = stream_;
    const bool dilu = pk == PrecondKind::DIC || pk == PrecondKind::DILU;
    if (dilu) ensureDilu();
    setupMatrix(diag, upper, lower, false, false);
    DevLevel& D0 = L_[0];
    const int n0 = D0.nrows;
    st_.zero(s);
    VLM_LAUNCH(k_to_solver<double>, nblk(n0), 256, s, n0, perm0_.get(), r, r_.get());
    if (dilu) {
        diluFactor(upper, lower);
        recordDiluApply(r_.get(), w_.get());
    } else if (pk == PrecondKind::Diagonal) {
        if (rD_.size() != size_t(n0)) rD_.resize(n0);
        VLM_LAUNCH(k_recip_diag<double>, nblk(n0), 256, s, n0, perm0_.get(), D0.diag.get(), rD_.get());
        recordPrecond(pk, SmootherKind::MCGSJacobi, r_.get(), w_.get(), false);
    } else {
        recordPrecond(pk, SmootherKind::MCGSJacobi, r_.get(), w_.get(), false);
    }
    VLM_LAUNCH(k_from_solver, nblk(n0), 256, s, n0, perm0_.get(), w_.get(), w);
    VLM_CUDA(cudaStreamSynchronize(s));
    if (dilu) checkLevelError();
}

int groupBarrierCheck(cudaStream_t s, int G, long long spinLimit, int absent, int rounds, int* passedOut) {
    if (G < 1 || G > 64 || rounds < 1 || spinLimit < 1) throw Error(VLM_ERR_BAD_ARG, "barrier check: 1 <= ctas <= 64, rounds >= 1, spin limit >= 1");
    DBuf<DiluBar> bar(1);
    DBuf<int> err(1), passed(static_cast<size_t>(G));
    bar.zero(s);
    err.zero(s);
    passed.zero(s);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(G));
    cfg.blockDim = dim3(unsigned(kDiluThreads));
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    VLM_CUDA(cudaLaunchKernelEx(&cfg, k_group_barrier_check, bar.get(), G, err.get(), spinLimit, absent, rounds,
                                passed.get()));
    int h = 0;
    VLM_CUDA(cudaMemcpyAsync(&h, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaMemcpyAsync(passedOut, passed.get(), sizeof(int) * size_t(G), cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaStreamSynchronize(s));
    return h;
}

double exactSumOnDevice(cudaStream_t s, const double* v, int64_t n) {
    if (n <= 0) return 0.0;
    std::vector<Chunk> ch;
    for (int64_t q = 0; q < n; q += kRowsPerCta)
        ch.push_back(Chunk{int32_t(q), int32_t(std::min<int64_t>(kRowsPerCta, n - q)), 0, int32_t(q / kRowsPerCta)});
    DBuf<Chunk> dch;
    dch.upload(ch, s);
    DBuf<long long> bins(ch.size() * 73);
    DBuf<int> cnt(1), sb(1), se(1);
    cnt.zero(s);
    const int zero = 0, nsl = int(ch.size());
    VLM_CUDA(cudaMemcpyAsync(sb.get(), &zero, sizeof(int), cudaMemcpyHostToDevice, s));
    VLM_CUDA(cudaMemcpyAsync(se.get(), &nsl, sizeof(int), cudaMemcpyHostToDevice, s));
    DBuf<double> out(1);
    RedCtx R{nullptr, bins.get(), cnt.get(), sb.get(), se.get()};
    VLM_LAUNCH(k_exact_sum, nsl, kRowsPerCta, s, dch.get(), v, R, out.get());
    double h = 0;
    VLM_CUDA(cudaMemcpyAsync(&h, out.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaStreamSynchronize(s));
    return h;
}

// Reads a buffer larger than the L2 cache so that the next launch finds none of its operands there
// (clean lines: no write-backs compete with the timed kernel).  The buffer is zero, so the store
// never happens; it keeps the loads.
__global__ void k_l2_flush(const int4* __restrict__ buf, size_t n, int* __restrict__ sink) {
    int acc = 0;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const int4 v = buf[i];
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x5eed1234) *sink = acc;
}

double DeviceBatch::profileKernel(const std::string& fullName, int reps, double* bytesPerLaunch) {
    cudaStream_t s = stream_;
    const std::string warmSuffix = ":warm";
    const bool warm = fullName.size() > warmSuffix.size() &&
                      fullName.compare(fullName.size() - warmSuffix.size(), warmSuffix.size(), warmSuffix) == 0;
    const std::string name = warm ? fullName.substr(0, fullName.size() - warmSuffix.size()) : fullName;
    DevLevel& D0 = L_[0];
    const double N = double(plan_.userCells), F = double(plan_.userFaces);
    cudaEvent_t e0, e1;
    VLM_CUDA(cudaEventCreate(&e0));
    VLM_CUDA(cudaEventCreate(&e1));
    // "<kernel>_steps": a box level-0 sweep as its two colour launches instead of the fused launch
    const std::string stepsSuffix = "_steps";
    const bool steps = name.size() > stepsSuffix.size() &&
                       name.compare(name.size() - stepsSuffix.size(), stepsSuffix.size(), stepsSuffix) == 0;
    const std::string base = steps ? name.substr(0, name.size() - stepsSuffix.size()) : name;
    const bool f32 = base.size() > 2 && base.substr(base.size() - 2) == "32";
    const double sz = f32 ? 4.0 : 8.0;
    if (f32 && D0.val32.size() == 0) throw Error(VLM_ERR_BAD_ARG, "run a mixed-precision solve first");
    std::function<void()> run;
    if (name == "amul64") {
        run = [&] { VLM_LAUNCH(k_amul, D0.all.n, kRowsPerCta, s, D0.ch(D0.all), D0.sell(), D0.val.get(), D0.diag.get(), x_.get(), w_.get()); };
        *bytesPerLaunch = sz * 3 * N + sz * F + 8 * F;
    } else if ((base == "smooth64" || base == "smooth32") && boxOn_) {
        // box level 0: each face coefficient once, no column indices; one fused launch per sweep
        // unless "_steps" asks for the colour launches
        run = [&] {
            if (!steps) {
                const bool done = f32 ? recordFusedSweep<float>(D0.fwd[0], D0.fwd[1], r32_.get(), w32_.get(), true, 1,
                                                                nullptr, nullptr)
                                      : recordFusedSweep<double>(D0.fwd[0], D0.fwd[1], r_.get(), w_.get(), true, 1,
                                                                 nullptr, nullptr);
                if (done) return;
            }
            for (int t = 0; t < D0.nSteps; ++t) {
                int g = 0;
                const BoxRows R = boxRows(D0, D0.fwd[t], &g);
                if (R.ch == nullptr && R.one.H % 4 == 0) {
                    const int g4 = (R.end - R.begin + 4 * kRowsPerCta - 1) / (4 * kRowsPerCta);
                    if (f32)
                        VLM_LAUNCH((k_box_gs4<float, 0>), g4, kRowsPerCta, s, R, (const float*)D0.bcoef32.get(), D0.nrows, (const float*)D0.diag32.get(), (const float*)r32_.get(), w32_.get(), (const int32_t*)nullptr, (const float*)nullptr);
                    else
                        VLM_LAUNCH((k_box_gs4<double, 0>), g4, kRowsPerCta, s, R, (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(), (const double*)r_.get(), w_.get(), (const int32_t*)nullptr, (const double*)nullptr);
                    continue;
                }
                if (f32)
                    VLM_LAUNCH((k_box_gs<float, 0>), g, kRowsPerCta, s, R, (const float*)D0.bcoef32.get(), D0.nrows, (const float*)D0.diag32.get(), (const float*)r32_.get(), w32_.get(), (const int32_t*)nullptr, (const float*)nullptr, (const SysState*)st_.get(), kFlagDone);
                else
                    VLM_LAUNCH((k_box_gs<double, 0>), g, kRowsPerCta, s, R, (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(), (const double*)r_.get(), w_.get(), (const int32_t*)nullptr, (const double*)nullptr, (const SysState*)st_.get(), kFlagDone);
            }
        };
        *bytesPerLaunch = sz * 4 * N + sz * F;
    } else if ((name == "residual64" || name == "residual32") && boxOn_) {
        run = [&] {
            int g = 0;
            const BoxRows R = boxRows(D0, D0.active, &g);
            if (f32)
                VLM_LAUNCH(k_box_residual<float>, g, kRowsPerCta, s, R, (const float*)D0.bcoef32.get(), D0.nrows, (const float*)D0.diag32.get(), (const float*)r32_.get(), (const float*)w32_.get(), D0.t32.get(), (const SysState*)st_.get(), kFlagDone);
            else
                VLM_LAUNCH(k_box_residual<double>, g, kRowsPerCta, s, R, (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(), (const double*)r_.get(), (const double*)w_.get(), D0.t.get(), (const SysState*)st_.get(), kFlagDone);
        };
        *bytesPerLaunch = sz * 4 * N + sz * F;
    } else if (name == "spmv64") {
        // the PCG product with its fused dot (the FP64 Krylov recurrence's largest kernel)
        run = [&] {
            int g = 0;
            const BoxRows R = boxOn_ ? boxRows(D0, D0.all, &g) : BoxRows{};
            const StreamShape* sh = boxOn_ ? streamShape<double>(R) : nullptr;
            if (sh)
                VLM_LAUNCH_SMEM((k_box_pcg_spmv_stream<double, kFlagDone>), sh->grid, sh->threads, sh->smem, s, R.one,
                                sh->TY, sh->S, (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(),
                                (const double*)r_.get(), w_.get(), red(), st_.get(), &sweepSync_.get()->err);
            else if (boxOn_ && R.ch == nullptr && R.one.H % 4 == 0)
                VLM_LAUNCH((k_box_pcg_spmv4<double, kFlagDone, false>), D0.all.n, kRowsPerCta, s, D0.ch(D0.all), R.one, (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(), (const double*)r_.get(), w_.get(), red(), st_.get());
            else if (boxOn_)
                VLM_LAUNCH((k_box_pcg_spmv<double, kFlagDone, false>), D0.all.n, kRowsPerCta, s, D0.ch(D0.all), R, (const double*)D0.bcoef.get(), D0.nrows, (const double*)D0.diag.get(), (const double*)r_.get(), w_.get(), red(), st_.get());
            else
                VLM_LAUNCH((k_pcg_spmv<double, kFlagDone, false>), D0.all.n, kRowsPerCta, s, D0.ch(D0.all), D0.sell(), D0.val.get(), D0.diag.get(), r_.get(), w_.get(), red(), st_.get());
        };
        *bytesPerLaunch = boxOn_ ? 8.0 * 3 * N + 8.0 * F : 8.0 * 3 * N + 8.0 * F + 8.0 * F;
    } else if (name == "smooth64" || name == "smooth32") {
        run = [&] {
            for (int t = 0; t < D0.nSteps; ++t) {
                if (f32)
                    VLM_LAUNCH((k_smooth_gs<float, 0>), D0.fwd[t].n, kRowsPerCta, s, D0.ch(D0.fwd[t]), D0.sell(), D0.val32.get(), D0.diag32.get(), r32_.get(), w32_.get(), (const int32_t*)nullptr, (const float*)nullptr, st_.get(), kFlagDone);
                else
                    VLM_LAUNCH((k_smooth_gs<double, 0>), D0.fwd[t].n, kRowsPerCta, s, D0.ch(D0.fwd[t]), D0.sell(), D0.val.get(), D0.diag.get(), r_.get(), w_.get(), (const int32_t*)nullptr, (const double*)nullptr, st_.get(), kFlagDone);
            }
        };
        *bytesPerLaunch = sz * 4 * N + sz * F + 8 * F;
    } else if (name == "vcycle32" || name == "vcycle32_notail" || name == "tail32") {
        const bool allow = name != "vcycle32_notail";
        run = [&, allow, name] {
            if (name == "tail32") {
                if (tailOn_) recordTail<float>(r32_.get(), w32_.get(), kFlagDone, false);
            } else {
                recordVcycle<float>(r32_.get(), w32_.get(), SmootherKind::MCGSJacobi, kFlagDone, allow);
            }
        };
        *bytesPerLaunch = 0;
    } else if (name == "residual64" || name == "residual32") {
        run = [&] {
            if (f32)
                VLM_LAUNCH(k_residual<float>, D0.active.n, kRowsPerCta, s, D0.ch(D0.active), D0.sell(), D0.val32.get(), D0.diag32.get(), r32_.get(), w32_.get(), D0.t32.get(), st_.get(), kFlagDone);
            else
                VLM_LAUNCH(k_residual<double>, D0.active.n, kRowsPerCta, s, D0.ch(D0.active), D0.sell(), D0.val.get(), D0.diag.get(), r_.get(), w_.get(), D0.t.get(), st_.get(), kFlagDone);
        };
        *bytesPerLaunch = sz * 4 * N + sz * F + 8 * F;
    } else {
        throw Error(VLM_ERR_BAD_ARG, "unknown kernel " + name);
    }
    // st_ flags of a finished solve are 'done': clear them so the kernels do their work.  The
    // vectors are reset to one fixed state (right-hand side b, zero iterate) so the timing does
    // not depend on what the last solve left in them.
    st_.zero(s);
    if (r32_.size() == size_t(D0.nrows))
        VLM_LAUNCH((k_cast_rows<double, float>), D0.all.n, kRowsPerCta, s, D0.ch(D0.all), b_.get(), r32_.get(),
                   st_.get(), kFlagDone);
    VLM_CUDA(cudaMemcpyAsync(r_.get(), b_.get(), sizeof(double) * size_t(D0.nrows), cudaMemcpyDeviceToDevice, s));
    w_.zero(s);
    if (w32_.size() == size_t(D0.nrows)) w32_.zero(s);
    run();
    double total = 0.0;
    if (warm) {
        VLM_CUDA(cudaEventRecord(e0, s));
        for (int i = 0; i < reps; ++i) run();
        VLM_CUDA(cudaEventRecord(e1, s));
        VLM_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        VLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        total = ms;
    } else {
        constexpr size_t kFlushBytes = size_t(256) << 20;  // twice the B200's 126 MB L2
        if (flush_.size() == 0) {
            flush_.resize(kFlushBytes / sizeof(int4));
            flush_.zero(s);
            flushSink_.resize(1);
        }
        for (int i = 0; i < reps; ++i) {
            k_l2_flush<<<1184, 256, 0, s>>>(flush_.get(), flush_.size(), flushSink_.get());
            VLM_CUDA(cudaGetLastError());
            VLM_CUDA(cudaEventRecord(e0, s));
            run();
            VLM_CUDA(cudaEventRecord(e1, s));
            VLM_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            VLM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            total += ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return total / reps;
}

template void DeviceBatch::recordVcycle<double>(const double*, double*, SmootherKind, int, bool);
template void DeviceBatch::recordVcycle<float>(const float*, float*, SmootherKind, int, bool);

}  // namespace vlm
