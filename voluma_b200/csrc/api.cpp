// extern "C" boundary (include/voluma_b200.h): status codes in, no exceptions out.
#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "assembly.h"
#include "flow.h"
#include "meshgen.h"
#include "solver.h"
#include "voluma_b200.h"

struct vlm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    // uploads of a solve's right-hand side and initial guess, behind the matrix upload and beside
    // the matrix set-up (vlm_ldu_solve)
    cudaStream_t copyStream = nullptr;
    cudaEvent_t matrixSent = nullptr, inputsSent = nullptr;
    std::string err;
    int refs = 1;  // the handle itself + one per registered mesh
};

struct vlm_topology {
    vlm::Hierarchy H;
    std::vector<std::vector<int>> colour;
    std::vector<int> nColours;
    vlm::BoxShape box;   // n[0] == 0: not a box mesh
    bool boxLayout = false;
};

struct vlm_mesh {
    vlm_ctx* ctx = nullptr;
    int nsys = 1;
    // totals of the concatenation: cells and internal faces in system order, then every boundary face
    int nCells = 0, nInternal = 0, nFaces = 0;
    std::vector<int64_t> cellBase, faceBase, bfaceBase;  // per system
    std::vector<std::vector<int32_t>> own, nei;          // per system, local numbering (hierarchy input)
    std::vector<std::vector<double>> magSf, ndc;
    vlm::DBuf<int32_t> refCells;  // global reference cells of a batch pressure solve
    std::unique_ptr<vlm::DeviceBatch> batch;
    std::unique_ptr<vlm::DeviceGeom> geom;  // assembly geometry (when the descriptor carries it)
    // staging for the host-pointer entry points
    vlm::DBuf<double> diag, upper, lower, b, x;
    // pressure-equation work arrays
    vlm::DBuf<double> gamma, su, p, pB, pdiag, pupper, psource, ic, bs, ffc, fd, fb, flux, bcv, grad;
    // the pressure corrector as one captured graph per configuration (pointers, passes, controls):
    // its solves write their records here, read back once per call
    struct PGraph {
        std::vector<int64_t> key;
        int runs = 0;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        // kernels one call launches: the geometry kernels, and per pass the deferred solve's counts
        // (eager set-up, loop entry, one loop pass), recorded when the passes were issued
        int64_t geomK = 0;
        std::vector<vlm::DeviceBatch::LaunchCount> solveK;
        ~PGraph() {
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
        }
    };
    std::vector<std::unique_ptr<PGraph>> pgraphs;
    std::vector<int32_t> refsHost;
    vlm::DBuf<vlm::SysState> pstate;
    vlm::DBuf<int> pstatus;
    void* pinned = nullptr;
    size_t pinnedBytes = 0;
    ~vlm_mesh() {
        pgraphs.clear();
        if (pinned) cudaFreeHost(pinned);
    }
};

namespace {
// hierarchy of the first system (input order) of a mesh / batch
const vlm::Hierarchy& hierOf(vlm_mesh* m) {
    const auto& P = m->batch->plan();
    for (int b = 0; b < P.nsys; ++b)
        if (P.order[b] == 0) return P.H[b];
    return P.H[0];
}

vlm::DeviceGeom& geomOf(vlm_mesh* m) {
    VLM_REQUIRE(m->geom, VLM_ERR_BAD_ARG, "the mesh was registered without geometry (V, Sf, d, w, corrVecs)");
    return *m->geom;
}
}  // namespace

namespace {

constexpr int64_t kRowsPerCtaForSum = 256;
thread_local std::string g_lastError;

}  // namespace

void vlm::setThreadError(const std::string& msg) { g_lastError = msg; }

namespace {

vlm_status fail(vlm_ctx* ctx, vlm_status s, const std::string& msg) {
    g_lastError = msg;
    if (ctx) ctx->err = msg;
    return s;
}

template <class F> vlm_status guarded(vlm_ctx* ctx, F&& f) {
    try {
        f();
        return VLM_OK;
    } catch (const vlm::Error& e) {
        return fail(ctx, e.status, e.what());
    } catch (const std::bad_alloc&) {
        return fail(ctx, VLM_ERR_OOM, "host allocation failed");
    } catch (const std::invalid_argument& e) {
        return fail(ctx, VLM_ERR_BAD_ARG, e.what());
    } catch (const std::exception& e) {
        return fail(ctx, VLM_ERR_CUDA, e.what());
    }
}

void setDevice(vlm_ctx* ctx) { VLM_CUDA(cudaSetDevice(ctx->device)); }

// Uploads the host LDU coefficients of a mesh into its staging buffers; returns the device
// pointers (lower aliases upper when the host lower pointer is NULL).
void stageCoeffs(vlm_mesh* m, const double* diag, const double* upper, const double* lower, const double** dDiag,
                 const double** dUpper, const double** dLower) {
    cudaStream_t s = m->ctx->stream;
    VLM_REQUIRE(diag && upper, VLM_ERR_BAD_ARG, "diag and upper are required");
    m->diag.upload(diag, size_t(m->nCells), s);
    if (m->nInternal > 0)
        m->upper.upload(upper, size_t(m->nInternal), s);
    else
        m->upper.resize(1);
    *dDiag = m->diag.get();
    *dUpper = m->upper.get();
    if (lower && lower != upper) {
        if (m->nInternal > 0)
            m->lower.upload(lower, size_t(m->nInternal), s);
        else
            m->lower.resize(1);
        *dLower = m->lower.get();
    } else {
        *dLower = m->upper.get();
    }
}

}  // namespace

extern "C" {

vlm_status vlm_ctx_create(int device, vlm_ctx** out) {
    if (!out) return fail(nullptr, VLM_ERR_BAD_ARG, "out is NULL");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(nullptr, VLM_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= n) return fail(nullptr, VLM_ERR_BAD_ARG, "device index out of range");
    auto* c = new vlm_ctx;
    c->device = device;
    vlm_status st = guarded(c, [&] {
        setDevice(c);
        VLM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    });
    if (st != VLM_OK) {
        delete c;
        return st;
    }
    *out = c;
    return VLM_OK;
}

namespace {
// Drops one reference; the stream is destroyed with the last one, so meshes released after
// their context handle still find a valid stream.
void ctxUnref(vlm_ctx* ctx) {
    if (--ctx->refs > 0) return;
    cudaSetDevice(ctx->device);
    if (ctx->copyStream) {
        cudaStreamSynchronize(ctx->copyStream);
        cudaStreamDestroy(ctx->copyStream);
    }
    if (ctx->matrixSent) cudaEventDestroy(ctx->matrixSent);
    if (ctx->inputsSent) cudaEventDestroy(ctx->inputsSent);
    if (ctx->stream) {
        cudaStreamSynchronize(ctx->stream);
        cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
}
}  // namespace

vlm_status vlm_ctx_destroy(vlm_ctx* ctx) {
    if (!ctx) return VLM_OK;
    ctxUnref(ctx);
    return VLM_OK;
}

const char* vlm_last_error(const vlm_ctx* ctx) { return ctx ? ctx->err.c_str() : g_lastError.c_str(); }

void* vlm_ctx_stream(vlm_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

vlm_status vlm_ctx_device_name(vlm_ctx* ctx, char* name, int32_t capacity) {
    if (!ctx || !name || capacity <= 0) return fail(ctx, VLM_ERR_BAD_ARG, "invalid arguments");
    return guarded(ctx, [&] {
        cudaDeviceProp p;
        VLM_CUDA(cudaGetDeviceProperties(&p, ctx->device));
        std::snprintf(name, size_t(capacity), "%s", p.name);
    });
}

vlm_status vlm_mesh_register_batch(vlm_ctx* ctx, int32_t nsys, const vlm_mesh_desc* descs, int32_t mergeLevels,
                                   vlm_mesh** out) {
    return vlm_mesh_register_batch_ex(ctx, nsys, descs, mergeLevels, 0, out);
}

vlm_status vlm_mesh_register_ex(vlm_ctx* ctx, const vlm_mesh_desc* d, int32_t mergeLevels, int32_t flags,
                                vlm_mesh** out) {
    if (!ctx || !d || !out) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return vlm_mesh_register_batch_ex(ctx, 1, d, mergeLevels, flags, out);
}

vlm_status vlm_mesh_register_batch_ex(vlm_ctx* ctx, int32_t nsys, const vlm_mesh_desc* descs, int32_t mergeLevels,
                                      int32_t flags, vlm_mesh** out) {
    if (!ctx || !descs || !out || nsys <= 0) return fail(ctx, VLM_ERR_BAD_ARG, "invalid arguments");
    if ((flags & ~int32_t(VLM_MESH_DEVICE_AGGLOMERATION)) != 0) return fail(ctx, VLM_ERR_BAD_ARG, "unknown mesh flags");
    *out = nullptr;
    return guarded(ctx, [&] {
        bool geometry = true;
        int64_t nC = 0, nI = 0, nF = 0;
        for (int s = 0; s < nsys; ++s) {
            const vlm_mesh_desc* d = &descs[s];
            VLM_REQUIRE(d->n_cells > 0 && d->n_internal_faces >= 0 && d->n_faces >= d->n_internal_faces,
                        VLM_ERR_BAD_ARG, "invalid mesh sizes");
            VLM_REQUIRE(d->owner && (d->neighbour || d->n_internal_faces == 0), VLM_ERR_BAD_ARG,
                        "owner/neighbour are required");
            VLM_REQUIRE(d->magSf && d->ndc, VLM_ERR_BAD_ARG, "magSf and ndc are required (GAMG weights)");
            geometry = geometry && d->V && d->Sf && d->d && d->w && d->corrVecs;
            VLM_REQUIRE(d->two_d == descs[0].two_d && d->empty_dir == descs[0].empty_dir, VLM_ERR_BAD_ARG,
                        "every system of a batch must have the same 2D/3D setting");
            nC += d->n_cells;
            nI += d->n_internal_faces;
            nF += d->n_faces;
        }
        VLM_REQUIRE(nF < (int64_t(1) << 31) - 1, VLM_ERR_BAD_ARG, "batch exceeds 2^31 faces");
        setDevice(ctx);
        auto m = std::make_unique<vlm_mesh>();
        m->ctx = ctx;
        m->nsys = nsys;
        m->nCells = int(nC);
        m->nInternal = int(nI);
        m->nFaces = int(nF);
        std::vector<vlm::SysTopo> topo(static_cast<size_t>(nsys));
        int64_t cb = 0, fb = 0, bb = 0;
        for (int s = 0; s < nsys; ++s) {
            const vlm_mesh_desc* d = &descs[s];
            m->cellBase.push_back(cb);
            m->faceBase.push_back(fb);
            m->bfaceBase.push_back(bb);
            m->own.emplace_back(d->owner, d->owner + d->n_faces);
            m->nei.emplace_back(d->neighbour, d->neighbour + d->n_internal_faces);
            m->magSf.emplace_back(d->magSf, d->magSf + d->n_faces);
            m->ndc.emplace_back(d->ndc, d->ndc + d->n_faces);
            topo[s].nCells = d->n_cells;
            topo[s].nInternal = d->n_internal_faces;
            topo[s].own = m->own[s].data();
            topo[s].nei = m->nei[s].data();
            topo[s].magSf = m->magSf[s].data();
            topo[s].ndc = m->ndc[s].data();
            cb += d->n_cells;
            fb += d->n_internal_faces;
            bb += d->n_faces - d->n_internal_faces;
        }
        m->batch = std::make_unique<vlm::DeviceBatch>(topo, mergeLevels > 0 ? mergeLevels : 2, ctx->stream,
                                                      (flags & VLM_MESH_DEVICE_AGGLOMERATION) != 0);
        if (geometry) {
            // the union mesh: every system's internal faces, then every system's boundary faces
            const size_t F = static_cast<size_t>(nF), NI = static_cast<size_t>(std::max<int64_t>(nI, 1)),
                         NC = static_cast<size_t>(nC);
            std::vector<int32_t> own(F), nei(NI), ps, pz;
            std::vector<double> magSf(F), ndc(F), w(F), V(NC), Sf(3 * F), dd(3 * F), corr(3 * F);
            bool centres = true;  // cell / face centres (optional)
            for (int s = 0; s < nsys; ++s) centres = centres && descs[s].C && descs[s].Cf;
            std::vector<double> Cc(centres ? 3 * NC : 0), Cfc(centres ? 3 * F : 0);
            bool skews = true;  // skew vectors (optional)
            for (int s = 0; s < nsys; ++s) skews = skews && descs[s].skewVecs;
            std::vector<double> skv(skews ? 3 * F : 0);
            auto copyFace = [&](const vlm_mesh_desc* d, int f, int64_t g, int64_t base) {
                own[g] = int32_t(d->owner[f] + base);
                magSf[g] = d->magSf[f];
                ndc[g] = d->ndc[f];
                w[g] = d->w[f];
                for (int q = 0; q < 3; ++q) {
                    Sf[3 * g + q] = d->Sf[3 * f + q];
                    dd[3 * g + q] = d->d[3 * f + q];
                    corr[3 * g + q] = d->corrVecs[3 * f + q];
                    if (centres) Cfc[3 * g + q] = d->Cf[3 * f + q];
                    if (skews) skv[3 * g + q] = d->skewVecs[3 * f + q];
                }
            };
            for (int s = 0; s < nsys; ++s) {
                const vlm_mesh_desc* d = &descs[s];
                const int64_t base = m->cellBase[s];
                for (int c = 0; c < d->n_cells; ++c) {
                    V[base + c] = d->V[c];
                    if (centres)
                        for (int q = 0; q < 3; ++q) Cc[3 * (base + c) + q] = d->C[3 * c + q];
                }
                for (int f = 0; f < d->n_internal_faces; ++f) {
                    copyFace(d, f, m->faceBase[s] + f, base);
                    nei[m->faceBase[s] + f] = int32_t(d->neighbour[f] + base);
                }
                for (int f = d->n_internal_faces; f < d->n_faces; ++f)
                    copyFace(d, f, nI + m->bfaceBase[s] + (f - d->n_internal_faces), base);
                for (int p = 0; p < d->n_patches; ++p) {
                    ps.push_back(int32_t(nI + m->bfaceBase[s] + (d->patch_start[p] - d->n_internal_faces)));
                    pz.push_back(d->patch_size[p]);
                }
            }
            m->geom = std::make_unique<vlm::DeviceGeom>(int(nC), int(nI), int(nF), own.data(), nei.data(), magSf.data(),
                                                        ndc.data(), V.data(), Sf.data(), dd.data(), w.data(),
                                                        corr.data(), descs[0].two_d, descs[0].empty_dir,
                                                        int(ps.size()), ps.data(), pz.data(),
                                                        centres ? Cc.data() : nullptr, centres ? Cfc.data() : nullptr,
                                                        skews ? skv.data() : nullptr, ctx->stream);
        }
        ctx->refs++;
        *out = m.release();
    });
}

vlm_status vlm_mesh_register(vlm_ctx* ctx, const vlm_mesh_desc* d, int32_t mergeLevels, vlm_mesh** out) {
    if (!ctx || !d || !out) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return vlm_mesh_register_batch(ctx, 1, d, mergeLevels, out);
}

vlm_status vlm_mesh_release(vlm_mesh* mesh) {
    if (!mesh) return VLM_OK;
    vlm_ctx* ctx = mesh->ctx;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    delete mesh;
    ctxUnref(ctx);
    return VLM_OK;
}

vlm_status vlm_amul(vlm_ctx* ctx, vlm_mesh* m, const double* diag, const double* upper, const double* lower,
                    const double* x, double* y) {
    if (!ctx || !m || !x || !y) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        const double *dd, *du, *dl;
        stageCoeffs(m, diag, upper, lower, &dd, &du, &dl);
        m->x.upload(x, size_t(m->nCells), ctx->stream);
        m->b.resize(size_t(m->nCells));
        m->batch->amul(dd, du, dl, m->x.get(), m->b.get());
        VLM_CUDA(cudaMemcpy(y, m->b.get(), sizeof(double) * size_t(m->nCells), cudaMemcpyDeviceToHost));
    });
}

vlm_status vlm_ldu_solve_device(vlm_ctx* ctx, vlm_mesh* m, const double* diag, const double* upper,
                                const double* lower, const double* b, double* x, const vlm_solver_ctrl* ctrl,
                                vlm_solver_perf* perf) {
    if (!ctx || !m || !diag || !upper || !b || !x || !ctrl) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        std::vector<vlm_solver_perf> p;
        m->batch->solve(diag, upper, lower ? lower : upper, b, x, *ctrl, p);
        if (perf) std::copy(p.begin(), p.end(), perf);
    });
}

vlm_status vlm_ldu_solve(vlm_ctx* ctx, vlm_mesh* m, const double* diag, const double* upper, const double* lower,
                         const double* b, double* x, const vlm_solver_ctrl* ctrl, vlm_solver_perf* perf) {
    if (!ctx || !m || !diag || !upper || !b || !x || !ctrl) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        cudaStream_t s = ctx->stream;
        const double *dd, *du, *dl;
        stageCoeffs(m, diag, upper, lower, &dd, &du, &dl);
        // b and x cross the bus after the matrix (which the set-up needs first) on a second stream,
        // while the device builds the hierarchy's matrices
        if (!ctx->copyStream) {
            VLM_CUDA(cudaStreamCreateWithFlags(&ctx->copyStream, cudaStreamNonBlocking));
            VLM_CUDA(cudaEventCreateWithFlags(&ctx->matrixSent, cudaEventDisableTiming));
            VLM_CUDA(cudaEventCreateWithFlags(&ctx->inputsSent, cudaEventDisableTiming));
        }
        m->b.resize(size_t(m->nCells));
        m->x.resize(size_t(m->nCells));
        VLM_CUDA(cudaEventRecord(ctx->matrixSent, s));
        VLM_CUDA(cudaStreamWaitEvent(ctx->copyStream, ctx->matrixSent, 0));
        m->b.upload(b, size_t(m->nCells), ctx->copyStream);
        m->x.upload(x, size_t(m->nCells), ctx->copyStream);
        VLM_CUDA(cudaEventRecord(ctx->inputsSent, ctx->copyStream));
        m->batch->inputsAfter(ctx->inputsSent);
        std::vector<vlm_solver_perf> p;
        m->batch->solve(dd, du, dl, m->b.get(), m->x.get(), *ctrl, p);
        VLM_CUDA(cudaMemcpyAsync(x, m->x.get(), sizeof(double) * size_t(m->nCells), cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
        if (perf) std::copy(p.begin(), p.end(), perf);
    });
}

vlm_status vlm_gamg_apply(vlm_ctx* ctx, vlm_mesh* m, const double* diag, const double* upper, const double* lower,
                          const double* r, double* w, const vlm_solver_ctrl* ctrl) {
    if (!ctx || !m || !r || !w) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        const double *dd, *du, *dl;
        stageCoeffs(m, diag, upper, lower, &dd, &du, &dl);
        m->b.upload(r, size_t(m->nCells), ctx->stream);
        m->x.resize(size_t(m->nCells));
        const vlm::SmootherKind sm = vlm::parseSmoother(ctrl ? ctrl->smoother : "");
        m->batch->gamgApply(dd, du, dl, m->b.get(), m->x.get(), sm);
        VLM_CUDA(cudaMemcpy(w, m->x.get(), sizeof(double) * size_t(m->nCells), cudaMemcpyDeviceToHost));
    });
}

vlm_status vlm_precond_apply(vlm_ctx* ctx, vlm_mesh* m, const double* diag, const double* upper, const double* lower,
                             const double* r, double* w, const vlm_solver_ctrl* ctrl) {
    if (!ctx || !m || !r || !w || !ctrl) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        const double *dd, *du, *dl;
        stageCoeffs(m, diag, upper, lower, &dd, &du, &dl);
        m->b.upload(r, size_t(m->nCells), ctx->stream);
        m->x.resize(size_t(m->nCells));
        m->batch->precondApply(dd, du, dl, m->b.get(), m->x.get(), *ctrl);
        VLM_CUDA(cudaMemcpy(w, m->x.get(), sizeof(double) * size_t(m->nCells), cudaMemcpyDeviceToHost));
    });
}

vlm_status vlm_gamg_levels(vlm_mesh* m, int32_t* n) {
    if (!m || !n) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    *n = int32_t(hierOf(m).levels.size());
    return VLM_OK;
}

vlm_status vlm_gamg_level(vlm_mesh* m, int32_t level, int32_t* sizes, int32_t* l, int32_t* u, int32_t* agg) {
    if (!m || !sizes) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    const auto& H = hierOf(m);
    if (level < 0 || level >= int32_t(H.levels.size())) return fail(m->ctx, VLM_ERR_BAD_ARG, "level out of range");
    const auto& L = H.levels[level];
    sizes[0] = L.n;
    sizes[1] = int32_t(L.l.size());
    sizes[2] = int32_t(L.agg.size());
    if (l) std::copy(L.l.begin(), L.l.end(), l);
    if (u) std::copy(L.u.begin(), L.u.end(), u);
    if (agg) std::copy(L.agg.begin(), L.agg.end(), agg);
    return VLM_OK;
}

vlm_status vlm_gamg_colours(vlm_mesh* m, int32_t level, int32_t* n) {
    if (!m || !n) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    if (level < 0 || level >= m->batch->nLevels()) return fail(m->ctx, VLM_ERR_BAD_ARG, "level out of range");
    *n = m->batch->level(level).maxColours;
    return VLM_OK;
}

vlm_status vlm_mesh_stats(vlm_mesh* m, int64_t* launches, int64_t* bytes) {
    if (!m) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    if (launches) *launches = m->batch->launches();
    if (bytes) *bytes = int64_t(m->batch->deviceBytes());
    return VLM_OK;
}

vlm_status vlm_mesh_set_tail(vlm_mesh* m, int32_t cluster, int64_t max_rows, int64_t full_rows) {
    if (!m) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    if (cluster < 0 || max_rows < 0 || full_rows < 0) return fail(m->ctx, VLM_ERR_BAD_ARG, "negative tail setting");
    return guarded(m->ctx, [&] {
        setDevice(m->ctx);
        m->batch->setTail(cluster, max_rows, full_rows);
    });
}

vlm_status vlm_mesh_get_tail(vlm_mesh* m, int32_t* cluster, int64_t* max_rows, int64_t* full_rows) {
    if (!m || !cluster || !max_rows || !full_rows) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    int c = 0;
    m->batch->tailConfig(&c, max_rows, full_rows);
    *cluster = c;
    return VLM_OK;
}

vlm_status vlm_mesh_time_sweeps(vlm_mesh* m, int32_t on) {
    if (!m) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(m->ctx, [&] {
        setDevice(m->ctx);
        m->batch->setSweepTiming(on != 0);
    });
}

vlm_status vlm_mesh_sweep_time(vlm_mesh* m, double* ms_total, int64_t* sweeps) {
    if (!m || !ms_total || !sweeps) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    m->batch->sweepTiming(ms_total, sweeps);
    return VLM_OK;
}

vlm_status vlm_mesh_set_fusion(vlm_mesh* m, int64_t pre_rows, int64_t restrict_rows, int64_t post_rows) {
    if (!m) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(m->ctx, [&] {
        setDevice(m->ctx);
        m->batch->setFusion(pre_rows, restrict_rows, post_rows);
    });
}

vlm_status vlm_mesh_get_fusion(vlm_mesh* m, int64_t* pre_rows, int64_t* restrict_rows, int64_t* post_rows) {
    if (!m || !pre_rows || !restrict_rows || !post_rows) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    m->batch->fusionConfig(pre_rows, restrict_rows, post_rows);
    return VLM_OK;
}

vlm_status vlm_mesh_get_stream(vlm_mesh* m, int32_t* pencil_rows, int32_t* stages, int32_t* ctas) {
    if (!m || !pencil_rows || !stages || !ctas) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    m->batch->streamConfig(pencil_rows, stages, ctas);
    return VLM_OK;
}

vlm_status vlm_profile_kernel(vlm_ctx* ctx, vlm_mesh* m, const char* kernel, int32_t reps, double* ms, double* bytes) {
    if (!ctx || !m || !kernel || !ms || !bytes || reps <= 0) return fail(ctx, VLM_ERR_BAD_ARG, "invalid arguments");
    return guarded(ctx, [&] {
        setDevice(ctx);
        *ms = m->batch->profileKernel(kernel, reps, bytes);
    });
}

vlm_status vlm_topology_build(int32_t n_cells, int32_t n_internal_faces, const int32_t* owner,
                              const int32_t* neighbour, const double* magSf, const double* ndc, int32_t merge_levels,
                              vlm_topology** out) {
    if (!out || !owner || (!neighbour && n_internal_faces > 0) || !magSf || !ndc || n_cells <= 0)
        return fail(nullptr, VLM_ERR_BAD_ARG, "invalid topology arguments");
    *out = nullptr;
    return guarded(nullptr, [&] {
        auto t = std::make_unique<vlm_topology>();
        t->H = vlm::buildHierarchy(n_cells, n_internal_faces, owner, neighbour, magSf, ndc,
                                   merge_levels > 0 ? merge_levels : 2);
        for (const auto& L : t->H.levels) {
            int nc = 0;
            t->colour.push_back(vlm::greedyColour(L, &nc));
            t->nColours.push_back(nc);
        }
        if (vlm::detectBox(n_cells, n_internal_faces, owner, neighbour, &t->box))
            t->boxLayout = t->H.levels.size() <= 1 ||
                           vlm::boxParityColouring(t->box, t->colour[0].data(), t->nColours[0]);
        else
            t->box = vlm::BoxShape();
        *out = t.release();
    });
}

vlm_status vlm_topology_levels(const vlm_topology* t, int32_t* n) {
    if (!t || !n) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    *n = int32_t(t->H.levels.size());
    return VLM_OK;
}

vlm_status vlm_topology_level(const vlm_topology* t, int32_t level, int32_t* sizes, int32_t* l, int32_t* u,
                              double* weight, int32_t* agg, int32_t* face_map, int8_t* face_flip, int32_t* colour) {
    if (!t || !sizes) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    if (level < 0 || level >= int32_t(t->H.levels.size())) return fail(nullptr, VLM_ERR_BAD_ARG, "level out of range");
    const auto& L = t->H.levels[level];
    sizes[0] = L.n;
    sizes[1] = int32_t(L.l.size());
    sizes[2] = int32_t(L.agg.size());
    sizes[3] = t->nColours[level];
    if (l) std::copy(L.l.begin(), L.l.end(), l);
    if (u) std::copy(L.u.begin(), L.u.end(), u);
    if (weight) std::copy(L.weight.begin(), L.weight.end(), weight);
    if (agg) std::copy(L.agg.begin(), L.agg.end(), agg);
    if (face_map) std::copy(L.faceMap.begin(), L.faceMap.end(), face_map);
    if (face_flip)
        for (size_t k = 0; k < L.faceFlip.size(); ++k) face_flip[k] = int8_t(L.faceFlip[k]);
    if (colour) std::copy(t->colour[level].begin(), t->colour[level].end(), colour);
    return VLM_OK;
}

vlm_status vlm_topology_box(const vlm_topology* t, int32_t* shape) {
    if (!t || !shape) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    for (int d = 0; d < 3; ++d) {
        shape[d] = t->box.n[d];
        shape[3 + d] = t->box.per[d];
    }
    shape[6] = t->boxLayout ? 1 : 0;
    return VLM_OK;
}

vlm_status vlm_topology_destroy(vlm_topology* t) {
    delete t;
    return VLM_OK;
}

namespace {

// Host boundary values -> device (n_boundary doubles), NULL stays NULL.
const double* stageBC(vlm_mesh* m, const double* bcValues, cudaStream_t s) {
    const int nB = m->nFaces - m->nInternal;
    if (!bcValues || nB == 0) return nullptr;
    m->bcv.upload(bcValues, size_t(nB), s);
    return m->bcv.get();
}

void ensureWork(vlm_mesh* m) {
    const size_t nC = size_t(m->nCells), nF = size_t(m->nFaces), nI = size_t(std::max(m->nInternal, 1)),
                 nB = size_t(std::max(m->nFaces - m->nInternal, 1));
    if (m->pdiag.size() == nC) return;
    m->gamma.resize(nF);
    m->su.resize(nC);
    m->p.resize(nC);
    m->pB.resize(nB);
    m->pdiag.resize(nC);
    m->pupper.resize(nI);
    m->psource.resize(nC);
    m->ic.resize(nB);
    m->bs.resize(nB);
    m->ffc.resize(nF);
    m->fd.resize(nC);
    m->fb.resize(nC);
    m->flux.resize(nF);
    m->grad.resize(3 * nC);
}

// The corrector passes (IncompressibleFlow.cpp:322-341) on the stream: boundary values, laplacian with
// the explicit non-orthogonal correction, source, references, fold, solve (deferred: its records go to
// m->pstate / m->pstatus), and the face flux of the last pass.
void pressurePasses(vlm_mesh* m, const double* gamma, const double* divPhi, double* p, const vlm::ScalarBC& bc,
                    int nRefs, double refValue, int nNonOrth, int gradScheme, const vlm_solver_ctrl& ctrl,
                    const vlm_solver_ctrl& finalCtrl, double* flux, vlm_mesh::PGraph* g) {
    vlm::DeviceGeom& G = geomOf(m);
    cudaStream_t s = m->ctx->stream;
    const int64_t geom0 = G.launches();
    g->solveK.clear();
    for (int no = 0; no <= nNonOrth; ++no) {
        const bool last = no == nNonOrth;
        G.correctBoundary(p, bc, m->pB.get(), s);
        bool hasFfc = false;
        G.laplacian(gamma, p, m->pB.get(), bc, true, gradScheme, m->pdiag.get(), m->pupper.get(), m->psource.get(),
                    m->ic.get(), m->bs.get(), m->ffc.get(), &hasFfc, s);
        G.addVolumeSource(m->psource.get(), divPhi, s);
        if (nRefs > 0) G.setReferences(m->refCells.get(), nRefs, refValue, m->pdiag.get(), m->psource.get(), s);
        G.fold(m->pdiag.get(), m->psource.get(), m->ic.get(), m->bs.get(), m->fd.get(), m->fb.get(), s);
        std::vector<vlm_solver_perf> pf;
        m->batch->deferNextSolve(m->pstate.get() + size_t(no) * m->nsys, m->pstatus.get() + 2 * no);
        m->batch->solve(m->fd.get(), m->pupper.get(), m->pupper.get(), m->fb.get(), p, last ? finalCtrl : ctrl, pf);
        g->solveK.push_back(m->batch->lastDeferred());
        if (last && flux) G.flux(m->pupper.get(), p, m->ic.get(), m->bs.get(), hasFfc ? m->ffc.get() : nullptr, flux, s);
    }
    G.correctBoundary(p, bc, m->pB.get(), s);
    g->geomK = G.launches() - geom0;
}

std::vector<int64_t> ctrlKey(const vlm_solver_ctrl& c) {
    std::vector<int64_t> k;
    for (const char* t : {c.solver, c.preconditioner, c.smoother, c.precision}) k.push_back(int64_t(std::hash<std::string>()(t)));
    double d[4] = {c.tolerance, c.relTol, c.innerRelTol, 0.0};
    for (double v : d) {
        int64_t b;
        std::memcpy(&b, &v, sizeof b);
        k.push_back(b);
    }
    for (int v : {int(c.maxIter), int(c.minIter), int(c.nSweeps), int(c.reproducible), int(c.mergeLevels)}) k.push_back(v);
    return k;
}

// Device-pointer pressure corrector; bcv: device boundary values or null.  The first call of a
// configuration runs the passes directly (creating every lazily built resource and the solves'
// graphs); from the second call on the passes are one captured graph: one launch per call.  The
// solver records of every pass are read back once at the end.
void pressureLoop(vlm_mesh* m, const double* gamma, const double* divPhi, double* p, const int32_t* bcType,
                  const double* bcv, const int32_t* refCells, double refValue, int nNonOrth, int gradScheme,
                  const vlm_solver_ctrl& ctrl, const vlm_solver_ctrl& finalCtrl, vlm_solver_perf* perf, double* flux) {
    cudaStream_t s = m->ctx->stream;
    geomOf(m);
    ensureWork(m);
    // global reference cells (-1: none)
    std::vector<int32_t> refs;
    for (int q = 0; q < m->nsys; ++q) {
        if (!refCells || refCells[q] < 0) continue;
        const int64_t cellsOfSystem = (q + 1 < m->nsys ? m->cellBase[q + 1] : int64_t(m->nCells)) - m->cellBase[q];
        VLM_REQUIRE(refCells[q] < cellsOfSystem, VLM_ERR_BAD_ARG, "reference cell out of range");
        refs.push_back(int32_t(m->cellBase[q] + refCells[q]));
    }
    if (!refs.empty() && refs != m->refsHost) {
        m->refCells.upload(refs, s);
        m->refsHost = refs;
        m->pgraphs.clear();  // the graphs hold the old reference-cell array
    }
    const size_t nRec = size_t(nNonOrth + 1) * size_t(m->nsys);
    if (m->pstate.size() < nRec) {
        VLM_CUDA(cudaStreamSynchronize(s));
        m->pgraphs.clear();
        m->pstate.resize(nRec);
        m->pstatus.resize(2 * size_t(nNonOrth + 1));
    }
    const size_t need = sizeof(vlm::SysState) * nRec + sizeof(int) * 2 * size_t(nNonOrth + 1);
    if (m->pinnedBytes < need) {
        if (m->pinned) cudaFreeHost(m->pinned);
        m->pinned = nullptr;
        VLM_CUDA(cudaMallocHost(&m->pinned, need));
        m->pinnedBytes = need;
    }
    vlm::ScalarBC bc;
    bc.type = bcType;
    bc.value = bcv;
    std::vector<int64_t> key = {int64_t(gamma), int64_t(divPhi), int64_t(p), int64_t(bcType), int64_t(bcv),
                                int64_t(flux), int64_t(refs.size()), nNonOrth, gradScheme};
    {
        int64_t b;
        std::memcpy(&b, &refValue, sizeof b);
        key.push_back(b);
        const auto k1 = ctrlKey(ctrl), k2 = ctrlKey(finalCtrl);
        key.insert(key.end(), k1.begin(), k1.end());
        key.insert(key.end(), k2.begin(), k2.end());
    }
    const char* gv = std::getenv("VLM_GRAPH");
    const bool graphs = !(gv && gv[0] == '0') && m->batch->embeddable();
    vlm_mesh::PGraph* g = nullptr;
    for (auto& q : m->pgraphs)
        if (q->key == key) g = q.get();
    if (!g) {
        m->pgraphs.push_back(std::make_unique<vlm_mesh::PGraph>());
        g = m->pgraphs.back().get();
        g->key = key;
    }
    const int nRefs = int(refs.size());
    if (graphs && g->runs >= 1 && !g->exec) {
        VLM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        m->batch->beginEmbedding();
        try {
            pressurePasses(m, gamma, divPhi, p, bc, nRefs, refValue, nNonOrth, gradScheme, ctrl, finalCtrl, flux, g);
        } catch (...) {
            m->batch->endEmbedding();
            cudaGraph_t junk = nullptr;
            cudaStreamEndCapture(s, &junk);
            if (junk) cudaGraphDestroy(junk);
            throw;
        }
        m->batch->endEmbedding();
        VLM_CUDA(cudaStreamEndCapture(s, &g->graph));
        VLM_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
    }
    if (g->exec)
        VLM_CUDA(cudaGraphLaunch(g->exec, s));
    else
        pressurePasses(m, gamma, divPhi, p, bc, nRefs, refValue, nNonOrth, gradScheme, ctrl, finalCtrl, flux, g);
    ++g->runs;
    // every pass's solver records, read once
    vlm::SysState* hs = static_cast<vlm::SysState*>(m->pinned);
    int* hst = reinterpret_cast<int*>(hs + nRec);
    VLM_CUDA(cudaMemcpyAsync(hs, m->pstate.get(), sizeof(vlm::SysState) * nRec, cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaMemcpyAsync(hst, m->pstatus.get(), sizeof(int) * 2 * size_t(nNonOrth + 1), cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaStreamSynchronize(s));
    // executed kernels: the geometry kernels and, per pass, the solve's set-up, loop entry and one
    // loop body per pass of its WHILE loop (the most iterations over the batch's systems)
    int64_t executed = g->geomK;
    for (int no = 0; no <= nNonOrth && no < int(g->solveK.size()); ++no) {
        int64_t its = 0;
        for (int b = 0; b < m->nsys; ++b) its = std::max<int64_t>(its, hs[size_t(no) * m->nsys + b].iterations);
        const auto& k = g->solveK[size_t(no)];
        executed += k.eager + k.pre + its * k.body;
    }
    m->batch->countLaunches(executed);
    const auto& order = m->batch->plan().order;
    for (int no = 0; no <= nNonOrth; ++no) {
        if (hst[2 * no + 1] != 0) {
            m->batch->clearLevelError();
            throw vlm::Error(VLM_ERR_TIMEOUT, "level-scheduled sweep: a group barrier wait gave up");
        }
        if (hst[2 * no] == VLM_ERR_SINGULAR) throw vlm::Error(VLM_ERR_SINGULAR, "GAMG: singular coarsest matrix");
        const vlm_solver_ctrl& c = no == nNonOrth ? finalCtrl : ctrl;
        if (!perf) continue;
        for (int b = 0; b < m->nsys; ++b) {
            const vlm::SysState& q = hs[size_t(no) * m->nsys + b];
            vlm_solver_perf r = {};
            r.initialResidual = q.initialResidual;
            r.finalResidual = q.finalResidual;
            r.residualSum = q.residualSum;
            r.normFactor = q.normFactor;
            r.iterations = q.iterations;
            r.outerIterations = q.outer;
            r.status = q.status;
            // converged() evaluated once more at exit (LinearSolver.cpp:283)
            r.converged = (r.iterations >= c.minIter) &&
                          (r.finalResidual < c.tolerance || (c.relTol > 0 && r.finalResidual < c.relTol * r.initialResidual));
            std::snprintf(r.solver, sizeof(r.solver), "%s", c.solver);
            perf[size_t(no) * m->nsys + size_t(order[b])] = r;
        }
    }
}

}  // namespace

vlm_status vlm_laplacian(vlm_ctx* ctx, vlm_mesh* m, const double* gamma, const double* psi, const int32_t* bcType,
                         const double* bcValues, int32_t nonOrthCorr, int32_t gradScheme, double* diag, double* upper,
                         double* source, double* ic, double* bs, double* ffc, int32_t* hasFfc) {
    if (!ctx || !m || !gamma || !psi || !bcType || !diag || !upper || !source || !ic || !bs || !ffc)
        return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        vlm::DeviceGeom& G = geomOf(m);
        cudaStream_t s = ctx->stream;
        ensureWork(m);
        m->gamma.upload(gamma, size_t(m->nFaces), s);
        m->p.upload(psi, size_t(m->nCells), s);
        vlm::ScalarBC bc;
        bc.type = bcType;
        bc.value = stageBC(m, bcValues, s);
        m->ffc.zero(s);
        G.correctBoundary(m->p.get(), bc, m->pB.get(), s);
        bool has = false;
        G.laplacian(m->gamma.get(), m->p.get(), m->pB.get(), bc, nonOrthCorr != 0, gradScheme, m->pdiag.get(),
                    m->pupper.get(), m->psource.get(), m->ic.get(), m->bs.get(), m->ffc.get(), &has, s);
        const size_t nB = size_t(m->nFaces - m->nInternal);
        VLM_CUDA(cudaMemcpyAsync(diag, m->pdiag.get(), sizeof(double) * m->nCells, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaMemcpyAsync(upper, m->pupper.get(), sizeof(double) * m->nInternal, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaMemcpyAsync(source, m->psource.get(), sizeof(double) * m->nCells, cudaMemcpyDeviceToHost, s));
        if (nB) {
            VLM_CUDA(cudaMemcpyAsync(ic, m->ic.get(), sizeof(double) * nB, cudaMemcpyDeviceToHost, s));
            VLM_CUDA(cudaMemcpyAsync(bs, m->bs.get(), sizeof(double) * nB, cudaMemcpyDeviceToHost, s));
        }
        VLM_CUDA(cudaMemcpyAsync(ffc, m->ffc.get(), sizeof(double) * m->nFaces, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
        if (hasFfc) *hasFfc = has ? 1 : 0;
    });
}

vlm_status vlm_grad(vlm_ctx* ctx, vlm_mesh* m, const double* psi, const int32_t* bcType, const double* bcValues,
                    int32_t scheme, double* out) {
    if (!ctx || !m || !psi || !bcType || !out) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        vlm::DeviceGeom& G = geomOf(m);
        cudaStream_t s = ctx->stream;
        ensureWork(m);
        m->p.upload(psi, size_t(m->nCells), s);
        vlm::ScalarBC bc;
        bc.type = bcType;
        bc.value = stageBC(m, bcValues, s);
        G.correctBoundary(m->p.get(), bc, m->pB.get(), s);
        G.grad(m->p.get(), m->pB.get(), bc, scheme, m->grad.get(), s);
        VLM_CUDA(cudaMemcpyAsync(out, m->grad.get(), sizeof(double) * 3 * m->nCells, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
    });
}

vlm_status vlm_div(vlm_ctx* ctx, vlm_mesh* m, const double* F, double* out) {
    if (!ctx || !m || !F || !out) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        vlm::DeviceGeom& G = geomOf(m);
        cudaStream_t s = ctx->stream;
        ensureWork(m);
        m->flux.upload(F, size_t(m->nFaces), s);
        G.div(m->flux.get(), m->su.get(), s);
        VLM_CUDA(cudaMemcpyAsync(out, m->su.get(), sizeof(double) * m->nCells, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
    });
}

vlm_status vlm_pressure_solve_batch(vlm_ctx* ctx, vlm_mesh* m, const double* gamma, const double* divPhi, double* p,
                                    const int32_t* bcType, const double* bcValues, const int32_t* refCells,
                                    double refValue, int32_t nNonOrth, int32_t gradScheme, const vlm_solver_ctrl* ctrl,
                                    const vlm_solver_ctrl* finalCtrl, vlm_solver_perf* perf, double* flux,
                                    int32_t devicePointers) {
    if (!ctx || !m || !gamma || !divPhi || !p || !bcType || !ctrl || nNonOrth < 0)
        return fail(ctx, VLM_ERR_BAD_ARG, "invalid arguments");
    return guarded(ctx, [&] {
        setDevice(ctx);
        cudaStream_t s = ctx->stream;
        if (devicePointers) {
            const int nB = m->nFaces - m->nInternal;
            const double* bcvd = nullptr;
            if (bcValues && nB > 0) {
                m->bcv.resize(size_t(nB));
                VLM_CUDA(cudaMemcpyAsync(m->bcv.get(), bcValues, sizeof(double) * nB, cudaMemcpyDeviceToDevice, s));
                bcvd = m->bcv.get();
            }
            pressureLoop(m, gamma, divPhi, p, bcType, bcvd, refCells, refValue, nNonOrth, gradScheme, *ctrl,
                         finalCtrl ? *finalCtrl : *ctrl, perf, flux);
            VLM_CUDA(cudaStreamSynchronize(s));
            return;
        }
        ensureWork(m);
        m->gamma.upload(gamma, size_t(m->nFaces), s);
        m->su.upload(divPhi, size_t(m->nCells), s);
        m->p.upload(p, size_t(m->nCells), s);
        const double* bcv = stageBC(m, bcValues, s);
        pressureLoop(m, m->gamma.get(), m->su.get(), m->p.get(), bcType, bcv, refCells, refValue, nNonOrth, gradScheme,
                     *ctrl, finalCtrl ? *finalCtrl : *ctrl, perf, flux ? m->flux.get() : nullptr);
        VLM_CUDA(cudaMemcpyAsync(p, m->p.get(), sizeof(double) * m->nCells, cudaMemcpyDeviceToHost, s));
        if (flux)
            VLM_CUDA(cudaMemcpyAsync(flux, m->flux.get(), sizeof(double) * m->nFaces, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
    });
}

vlm_status vlm_pressure_solve_device(vlm_ctx* ctx, vlm_mesh* m, const double* gamma, const double* divPhi, double* p,
                                     const int32_t* bcType, const double* bcValues, int32_t refCell, double refValue,
                                     int32_t nNonOrth, int32_t gradScheme, const vlm_solver_ctrl* ctrl,
                                     const vlm_solver_ctrl* finalCtrl, vlm_solver_perf* perf, double* flux) {
    return vlm_pressure_solve_batch(ctx, m, gamma, divPhi, p, bcType, bcValues, &refCell, refValue, nNonOrth,
                                    gradScheme, ctrl, finalCtrl, perf, flux, 1);
}

vlm_status vlm_pressure_solve(vlm_ctx* ctx, vlm_mesh* m, const double* gamma, const double* divPhi, double* p,
                              const int32_t* bcType, const double* bcValues, int32_t refCell, double refValue,
                              int32_t nNonOrth, int32_t gradScheme, const vlm_solver_ctrl* ctrl,
                              const vlm_solver_ctrl* finalCtrl, vlm_solver_perf* perf, double* flux) {
    return vlm_pressure_solve_batch(ctx, m, gamma, divPhi, p, bcType, bcValues, &refCell, refValue, nNonOrth,
                                    gradScheme, ctrl, finalCtrl, perf, flux, 0);
}

vlm_status vlm_mesh_systems(vlm_mesh* m, int32_t* n_systems, int64_t* n_cells, int64_t* n_internal_faces,
                            int64_t* n_faces) {
    if (!m) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    if (n_systems) *n_systems = m->nsys;
    if (n_cells) *n_cells = m->nCells;
    if (n_internal_faces) *n_internal_faces = m->nInternal;
    if (n_faces) *n_faces = m->nFaces;
    return VLM_OK;
}

struct vlm_box {
    vlm::BoxMesh m;
};

vlm_status vlm_box_create(vlm_ctx* ctx, const vlm_box_spec* spec, vlm_box** out) {
    if (!ctx || !spec || !out) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    *out = nullptr;
    return guarded(ctx, [&] {
        setDevice(ctx);
        auto b = std::make_unique<vlm_box>();
        b->m = vlm::buildBoxMesh(*spec, ctx->stream);
        *out = b.release();
    });
}

vlm_status vlm_box_desc(const vlm_box* box, vlm_mesh_desc* d) {
    if (!box || !d) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    const vlm::BoxMesh& m = box->m;
    std::memset(d, 0, sizeof *d);
    d->n_cells = m.nCells;
    d->n_internal_faces = m.nInternal;
    d->n_faces = m.nFaces;
    d->owner = m.owner.data();
    d->neighbour = m.neighbour.data();
    d->magSf = m.magSf.data();
    d->ndc = m.ndc.data();
    d->V = m.V.data();
    d->Sf = m.Sf.data();
    d->d = m.d.data();
    d->w = m.w.data();
    d->corrVecs = m.corrVecs.data();
    d->two_d = m.twoD;
    d->empty_dir = m.emptyDir;
    d->n_patches = int32_t(m.patchStart.size());
    d->patch_start = m.patchStart.data();
    d->patch_size = m.patchSize.data();
    d->C = m.C.data();
    d->Cf = m.Cf.data();
    d->skewVecs = m.skewVecs.data();
    return VLM_OK;
}

vlm_status vlm_box_patch_sides(const vlm_box* box, int32_t* sides) {
    if (!box || !sides) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    std::copy(box->m.patchSide.begin(), box->m.patchSide.end(), sides);
    return VLM_OK;
}

vlm_status vlm_box_destroy(vlm_box* box) {
    delete box;
    return VLM_OK;
}

vlm_status vlm_barrier_check(vlm_ctx* ctx, int32_t ctas, int64_t spin_limit, int32_t absent_cta, int32_t rounds,
                             int32_t* passed, int32_t* barrier_status) {
    if (!ctx || !passed || !barrier_status) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        *barrier_status = vlm::groupBarrierCheck(ctx->stream, ctas, spin_limit, absent_cta, rounds, passed);
    });
}

vlm_status vlm_exact_sum(vlm_ctx* ctx, const double* values, int64_t n, double* out) {
    if (!ctx || (!values && n > 0) || !out || n < 0) return fail(ctx, VLM_ERR_BAD_ARG, "invalid arguments");
    return guarded(ctx, [&] {
        setDevice(ctx);
        if (n >= (int64_t(1) << 31) - kRowsPerCtaForSum) throw vlm::Error(VLM_ERR_BAD_ARG, "n too large");
        vlm::DBuf<double> d;
        d.upload(values, size_t(n), ctx->stream);
        *out = vlm::exactSumOnDevice(ctx->stream, d.get(), n);
    });
}

}  // extern "C"

// ====================================================================== incompressible step
struct vlm_flow {
    vlm_mesh* mesh = nullptr;
    std::unique_ptr<vlm::DeviceFlow> flow;
};

extern "C" {

vlm_status vlm_flow_create(vlm_ctx* ctx, vlm_mesh* m, const vlm_flow_ctrl* ctrl, const int32_t* uType,
                           const double* uValue, const int32_t* pType, const double* pValue, vlm_flow** out) {
    if (!ctx || !m || !ctrl || !out || !uType || !uValue || !pType || !pValue)
        return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(ctx, [&] {
        setDevice(ctx);
        auto f = std::make_unique<vlm_flow>();
        f->mesh = m;
        f->flow = std::make_unique<vlm::DeviceFlow>(*m->batch, geomOf(m), *ctrl, uType, uValue, pType, pValue,
                                                    ctx->stream);
        *out = f.release();
    });
}

vlm_status vlm_flow_set_state(vlm_flow* f, const double* U, const double* p) {
    if (!f) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        f->flow->setState(U, p);
    });
}

vlm_status vlm_flow_set_boundary_values(vlm_flow* f, const double* u_face, const double* p_face) {
    if (!f) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        f->flow->setBoundaryValues(u_face, p_face);
    });
}

vlm_status vlm_flow_step(vlm_flow* f, double dt, vlm_step_info* info) {
    if (!f) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        const vlm_step_info i = f->flow->step(dt);
        if (info) *info = i;
    });
}

vlm_status vlm_flow_run_steady(vlm_flow* f, int32_t maxIter, double tol, int32_t* iterations, vlm_step_info* last) {
    if (!f) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        vlm_step_info i;
        std::memset(&i, 0, sizeof i);
        int it = 0;
        for (it = 1; it <= maxIter; ++it) {
            i = f->flow->step(1.0);
            VLM_REQUIRE(std::isfinite(i.UInitialResidual) && std::isfinite(i.pInitialResidual) &&
                            std::isfinite(i.continuityError),
                        VLM_ERR_NONFINITE, "solution diverged (non-finite residual) at iteration " + std::to_string(it));
            if (it > 1 && i.UInitialResidual < tol && i.pInitialResidual < tol) break;
        }
        if (iterations) *iterations = std::min(it, maxIter);
        if (last) *last = i;
    });
}

vlm_status vlm_flow_get_state(vlm_flow* f, double* U, double* p, double* phi) {
    if (!f) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        f->flow->getState(U, p, phi);
    });
}

int64_t vlm_flow_launches(vlm_flow* f) { return f ? f->flow->launches() : 0; }

vlm_status vlm_flow_set_model(vlm_flow* f, const vlm_flow_model* model) {
    if (!f || !model) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        f->flow->setModel(*model);
    });
}

vlm_status vlm_flow_write_restart(vlm_flow* f, const char* dir) {
    if (!f || !dir) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        f->flow->writeRestart(dir);
    });
}

vlm_status vlm_flow_read_restart(vlm_flow* f, const char* dir, int32_t* found) {
    if (!f || !dir) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        const bool ok = f->flow->readRestart(dir);
        if (found) *found = ok ? 1 : 0;
    });
}

vlm_status vlm_flow_get_model_state(vlm_flow* f, double* nut, double* gradP) {
    if (!f) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    return guarded(f->mesh->ctx, [&] {
        setDevice(f->mesh->ctx);
        f->flow->modelState(nut, gradP);
    });
}

vlm_status vlm_flow_destroy(vlm_flow* f) {
    if (!f) return VLM_OK;
    cudaSetDevice(f->mesh->ctx->device);
    cudaStreamSynchronize(f->mesh->ctx->stream);
    delete f;
    return VLM_OK;
}

}  // extern "C"

