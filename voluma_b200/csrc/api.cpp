// extern "C" boundary (include/voluma_b200.h): status codes in, no exceptions out.
#include <cuda_runtime.h>

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "assembly.h"
#include "solver.h"
#include "voluma_b200.h"

struct vlm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    int refs = 1;  // the handle itself + one per registered mesh
};

struct vlm_topology {
    vlm::Hierarchy H;
    std::vector<std::vector<int>> colour;
    std::vector<int> nColours;
};

struct vlm_mesh {
    vlm_ctx* ctx = nullptr;
    int nCells = 0, nInternal = 0, nFaces = 0;
    std::vector<int32_t> own, nei;
    std::vector<double> magSf, ndc;
    std::unique_ptr<vlm::DeviceBatch> batch;
    std::unique_ptr<vlm::DeviceGeom> geom;  // assembly geometry (when the descriptor carries it)
    // staging for the host-pointer entry points
    vlm::DBuf<double> diag, upper, lower, b, x;
    // pressure-equation work arrays
    vlm::DBuf<double> gamma, su, p, pB, pdiag, pupper, psource, ic, bs, ffc, fd, fb, flux, bcv, grad;
};

namespace {
vlm::DeviceGeom& geomOf(vlm_mesh* m) {
    VLM_REQUIRE(m->geom, VLM_ERR_BAD_ARG, "the mesh was registered without geometry (V, Sf, d, w, corrVecs)");
    return *m->geom;
}
}  // namespace

namespace {

constexpr int64_t kRowsPerCtaForSum = 256;
thread_local std::string g_lastError;

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

vlm_status vlm_mesh_register(vlm_ctx* ctx, const vlm_mesh_desc* d, int32_t mergeLevels, vlm_mesh** out) {
    if (!ctx || !d || !out) return fail(ctx, VLM_ERR_BAD_ARG, "NULL argument");
    *out = nullptr;
    return guarded(ctx, [&] {
        VLM_REQUIRE(d->n_cells > 0 && d->n_internal_faces >= 0 && d->n_faces >= d->n_internal_faces, VLM_ERR_BAD_ARG,
                    "invalid mesh sizes");
        VLM_REQUIRE(d->owner && (d->neighbour || d->n_internal_faces == 0), VLM_ERR_BAD_ARG,
                    "owner/neighbour are required");
        VLM_REQUIRE(d->magSf && d->ndc, VLM_ERR_BAD_ARG, "magSf and ndc are required (GAMG weights)");
        setDevice(ctx);
        auto m = std::make_unique<vlm_mesh>();
        m->ctx = ctx;
        m->nCells = d->n_cells;
        m->nInternal = d->n_internal_faces;
        m->nFaces = d->n_faces;
        m->own.assign(d->owner, d->owner + d->n_faces);
        m->nei.assign(d->neighbour, d->neighbour + d->n_internal_faces);
        m->magSf.assign(d->magSf, d->magSf + d->n_faces);
        m->ndc.assign(d->ndc, d->ndc + d->n_faces);
        vlm::SysTopo t;
        t.nCells = m->nCells;
        t.nInternal = m->nInternal;
        t.own = m->own.data();
        t.nei = m->nei.data();
        t.magSf = m->magSf.data();
        t.ndc = m->ndc.data();
        m->batch = std::make_unique<vlm::DeviceBatch>(std::vector<vlm::SysTopo>{t}, mergeLevels > 0 ? mergeLevels : 2,
                                                      ctx->stream);
        if (d->V && d->Sf && d->d && d->w && d->corrVecs)
            m->geom = std::make_unique<vlm::DeviceGeom>(d->n_cells, d->n_internal_faces, d->n_faces, d->owner,
                                                        d->neighbour, d->magSf, d->ndc, d->V, d->Sf, d->d, d->w,
                                                        d->corrVecs, d->two_d, d->empty_dir, d->n_patches,
                                                        d->patch_start, d->patch_size, ctx->stream);
        ctx->refs++;
        *out = m.release();
    });
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
        if (perf) *perf = p[0];
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
        m->b.upload(b, size_t(m->nCells), s);
        m->x.upload(x, size_t(m->nCells), s);
        std::vector<vlm_solver_perf> p;
        m->batch->solve(dd, du, dl, m->b.get(), m->x.get(), *ctrl, p);
        VLM_CUDA(cudaMemcpyAsync(x, m->x.get(), sizeof(double) * size_t(m->nCells), cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
        if (perf) *perf = p[0];
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

vlm_status vlm_gamg_levels(vlm_mesh* m, int32_t* n) {
    if (!m || !n) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    *n = int32_t(m->batch->plan().H[0].levels.size());
    return VLM_OK;
}

vlm_status vlm_gamg_level(vlm_mesh* m, int32_t level, int32_t* sizes, int32_t* l, int32_t* u, int32_t* agg) {
    if (!m || !sizes) return fail(nullptr, VLM_ERR_BAD_ARG, "NULL argument");
    const auto& H = m->batch->plan().H[0];
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

// Device-pointer pressure corrector loop; bcv: device boundary values or null.
void pressureLoop(vlm_mesh* m, const double* gamma, const double* divPhi, double* p, const int32_t* bcType,
                  const double* bcv, int refCell, double refValue, int nNonOrth, int gradScheme,
                  const vlm_solver_ctrl& ctrl, const vlm_solver_ctrl& finalCtrl, vlm_solver_perf* perf, double* flux) {
    vlm::DeviceGeom& G = geomOf(m);
    cudaStream_t s = m->ctx->stream;
    ensureWork(m);
    vlm::ScalarBC bc;
    bc.type = bcType;
    bc.value = bcv;
    for (int no = 0; no <= nNonOrth; ++no) {
        const bool last = no == nNonOrth;
        G.correctBoundary(p, bc, m->pB.get(), s);
        bool hasFfc = false;
        G.laplacian(gamma, p, m->pB.get(), bc, true, gradScheme, m->pdiag.get(), m->pupper.get(), m->psource.get(),
                    m->ic.get(), m->bs.get(), m->ffc.get(), &hasFfc, s);
        G.addVolumeSource(m->psource.get(), divPhi, s);
        if (refCell >= 0) G.setReference(refCell, refValue, m->pdiag.get(), m->psource.get(), s);
        G.fold(m->pdiag.get(), m->psource.get(), m->ic.get(), m->bs.get(), m->fd.get(), m->fb.get(), s);
        std::vector<vlm_solver_perf> pf;
        m->batch->solve(m->fd.get(), m->pupper.get(), m->pupper.get(), m->fb.get(), p, last ? finalCtrl : ctrl, pf);
        if (perf) perf[no] = pf[0];
        if (last && flux) G.flux(m->pupper.get(), p, m->ic.get(), m->bs.get(), hasFfc ? m->ffc.get() : nullptr, flux, s);
    }
    G.correctBoundary(p, bc, m->pB.get(), s);
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

vlm_status vlm_pressure_solve_device(vlm_ctx* ctx, vlm_mesh* m, const double* gamma, const double* divPhi, double* p,
                                     const int32_t* bcType, const double* bcValues, int32_t refCell, double refValue,
                                     int32_t nNonOrth, int32_t gradScheme, const vlm_solver_ctrl* ctrl,
                                     const vlm_solver_ctrl* finalCtrl, vlm_solver_perf* perf, double* flux) {
    if (!ctx || !m || !gamma || !divPhi || !p || !bcType || !ctrl || nNonOrth < 0)
        return fail(ctx, VLM_ERR_BAD_ARG, "invalid arguments");
    return guarded(ctx, [&] {
        setDevice(ctx);
        pressureLoop(m, gamma, divPhi, p, bcType, bcValues, refCell, refValue, nNonOrth, gradScheme, *ctrl,
                     finalCtrl ? *finalCtrl : *ctrl, perf, flux);
    });
}

vlm_status vlm_pressure_solve(vlm_ctx* ctx, vlm_mesh* m, const double* gamma, const double* divPhi, double* p,
                              const int32_t* bcType, const double* bcValues, int32_t refCell, double refValue,
                              int32_t nNonOrth, int32_t gradScheme, const vlm_solver_ctrl* ctrl,
                              const vlm_solver_ctrl* finalCtrl, vlm_solver_perf* perf, double* flux) {
    if (!ctx || !m || !gamma || !divPhi || !p || !bcType || !ctrl || nNonOrth < 0)
        return fail(ctx, VLM_ERR_BAD_ARG, "invalid arguments");
    return guarded(ctx, [&] {
        setDevice(ctx);
        cudaStream_t s = ctx->stream;
        ensureWork(m);
        m->gamma.upload(gamma, size_t(m->nFaces), s);
        m->su.upload(divPhi, size_t(m->nCells), s);
        m->p.upload(p, size_t(m->nCells), s);
        const double* bcv = stageBC(m, bcValues, s);
        pressureLoop(m, m->gamma.get(), m->su.get(), m->p.get(), bcType, bcv, refCell, refValue, nNonOrth, gradScheme,
                     *ctrl, finalCtrl ? *finalCtrl : *ctrl, perf, flux ? m->flux.get() : nullptr);
        VLM_CUDA(cudaMemcpyAsync(p, m->p.get(), sizeof(double) * m->nCells, cudaMemcpyDeviceToHost, s));
        if (flux)
            VLM_CUDA(cudaMemcpyAsync(flux, m->flux.get(), sizeof(double) * m->nFaces, cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
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
