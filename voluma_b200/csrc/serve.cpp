// Serving runtime: continuous batching of incompressible solves on one device.
//
// Requests (a mesh, boundary conditions and flow controls; steady or transient) are submitted at
// any time with an arrival time on the server clock.  A dispatcher admits them in arrival order as
// soon as a slot is free and their device-memory estimate fits in the HBM budget still unused;
// admitted requests run on a pool of worker threads, each with its own context and stream, so the
// kernels of different requests overlap on the device and a request that arrives while others run
// starts without waiting for them.  Everything a request needs (mesh, GAMG hierarchy, matrices,
// fields) lives on the device from admission to completion; the host reads only residual figures.
// Each request's kernels run on its own stream and are deterministic, so its result is the same
// alone and in any mix.
//
// The runtime is a client of the library's own C ABI (vlm_ctx / vlm_mesh / vlm_flow).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "common.h"
#include "voluma_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

// A request with its own copies of every array it was submitted with.
struct Request {
    int64_t id = 0;
    int32_t nCells = 0, nInternal = 0, nFaces = 0, nPatches = 0, twoD = 0, emptyDir = 0;
    std::vector<int32_t> own, nei, patchStart, patchSize, uType, pType;
    std::vector<double> magSf, ndc, V, Sf, d, w, corr, C, Cf, skew, uValue, pValue, U0, p0, uRobin, pRobin, uAdv;
    vlm_flow_ctrl ctrl{};
    int32_t steady = 1, nSteps = 0, maxIter = 0;
    double dt = 1.0, tol = 1e-6, arrival = 0;
    int32_t meshFlags = 0;
    int64_t bytes = 0;
};

struct Done {
    vlm_flow_result r{};
    std::vector<double> U, p, phi;
};

template <class T> std::vector<T> copyOf(const T* p, size_t n) { return p ? std::vector<T>(p, p + n) : std::vector<T>(); }

}  // namespace

struct vlm_server {
    int device = 0;
    int64_t budget = 0;
    int maxActive = 1;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv;      // dispatcher and workers
    std::condition_variable doneCv;  // collectors
    std::deque<std::unique_ptr<Request>> pending, ready;
    std::map<int64_t, Done> done;
    std::vector<int64_t> doneOrder;
    int64_t nextId = 1, inUse = 0;
    int active = 0;
    bool stop = false;
    std::thread dispatcher;
    std::vector<std::thread> workers;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    void finish(Request& q, Done&& d) {
        std::lock_guard<std::mutex> lk(mu);
        inUse -= q.bytes;
        --active;
        done[q.id] = std::move(d);
        doneOrder.push_back(q.id);
        cv.notify_all();
        doneCv.notify_all();
    }

    // Admission: arrival order; a request starts once it has arrived, a slot is free and its bytes fit.
    void dispatch() {
        std::unique_lock<std::mutex> lk(mu);
        while (!stop) {
            if (pending.empty()) {
                cv.wait(lk);
                continue;
            }
            Request& q = *pending.front();
            const double wait = q.arrival - now();
            if (wait > 0) {
                cv.wait_for(lk, std::chrono::duration<double>(wait));
                continue;
            }
            if (q.bytes > budget) {
                // can never fit: completes at once with an out-of-memory status
                Done d;
                d.r.id = q.id;
                d.r.status = VLM_ERR_OOM;
                d.r.arrival = q.arrival;
                d.r.admitted = d.r.finished = now();
                d.r.device_bytes = q.bytes;
                done[q.id] = std::move(d);
                doneOrder.push_back(q.id);
                pending.pop_front();
                doneCv.notify_all();
                continue;
            }
            if (active >= maxActive || inUse + q.bytes > budget) {
                cv.wait(lk);
                continue;
            }
            inUse += q.bytes;
            ++active;
            ready.push_back(std::move(pending.front()));
            pending.pop_front();
            cv.notify_all();
        }
    }

    void work() {
        vlm_ctx* ctx = nullptr;
        const vlm_status cs = vlm_ctx_create(device, &ctx);
        for (;;) {
            std::unique_ptr<Request> q;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return stop || !ready.empty(); });
                if (stop && ready.empty()) break;
                q = std::move(ready.front());
                ready.pop_front();
            }
            Done d;
            d.r.id = q->id;
            d.r.arrival = q->arrival;
            d.r.admitted = now();
            d.r.device_bytes = q->bytes;
            d.r.status = cs != VLM_OK ? cs : run(ctx, *q, d);
            d.r.finished = now();
            finish(*q, std::move(d));
        }
        if (ctx) vlm_ctx_destroy(ctx);
    }

    static vlm_status run(vlm_ctx* ctx, Request& q, Done& d) {
        vlm_mesh_desc m;
        std::memset(&m, 0, sizeof m);
        m.n_cells = q.nCells;
        m.n_internal_faces = q.nInternal;
        m.n_faces = q.nFaces;
        m.owner = q.own.data();
        m.neighbour = q.nei.data();
        m.magSf = q.magSf.data();
        m.ndc = q.ndc.data();
        m.V = q.V.data();
        m.Sf = q.Sf.data();
        m.d = q.d.data();
        m.w = q.w.data();
        m.corrVecs = q.corr.data();
        m.two_d = q.twoD;
        m.empty_dir = q.emptyDir;
        m.n_patches = q.nPatches;
        m.patch_start = q.patchStart.data();
        m.patch_size = q.patchSize.data();
        m.C = q.C.empty() ? nullptr : q.C.data();
        m.Cf = q.Cf.empty() ? nullptr : q.Cf.data();
        m.skewVecs = q.skew.empty() ? nullptr : q.skew.data();
        vlm_mesh* mesh = nullptr;
        vlm_flow* flow = nullptr;
        vlm_status st = vlm_mesh_register_ex(ctx, &m, 0, q.meshFlags, &mesh);
        if (st == VLM_OK)
            st = vlm_flow_create(ctx, mesh, &q.ctrl, q.uType.data(), q.uValue.data(), q.pType.data(), q.pValue.data(),
                                 &flow);
        if (st == VLM_OK)
            st = vlm_flow_set_state(flow, q.U0.empty() ? nullptr : q.U0.data(), q.p0.empty() ? nullptr : q.p0.data());
        vlm_step_info info{};
        if (st == VLM_OK) {
            if (q.steady) {
                st = vlm_flow_run_steady(flow, q.maxIter, q.tol, &d.r.iterations, &info);
            } else {
                for (int k = 0; k < q.nSteps && st == VLM_OK; ++k) st = vlm_flow_step(flow, q.dt, &info);
                d.r.iterations = q.nSteps;
            }
        }
        if (st == VLM_OK) {
            d.U.resize(size_t(3) * q.nCells);
            d.p.resize(size_t(q.nCells));
            d.phi.resize(size_t(q.nFaces));
            st = vlm_flow_get_state(flow, d.U.data(), d.p.data(), d.phi.data());
        }
        if (flow) d.r.launches = vlm_flow_launches(flow);
        d.r.UInitialResidual = info.UInitialResidual;
        d.r.pInitialResidual = info.pInitialResidual;
        d.r.continuityError = info.continuityError;
        vlm_flow_destroy(flow);
        vlm_mesh_release(mesh);
        return st;
    }
};

extern "C" {

int64_t vlm_flow_request_bytes(int32_t n_cells, int32_t n_faces) {
    // device footprint of one request: hierarchy + SELL matrices (FP64 and FP32) + Krylov and
    // V-cycle vectors + geometry + flow fields and matrices (measured per cell / face, rounded up)
    return int64_t(n_cells) * 2048 + int64_t(n_faces) * 512 + (int64_t(8) << 20);
}

vlm_status vlm_server_create(int32_t device, int64_t hbm_budget, int32_t max_active, vlm_server** out) {
    if (!out || hbm_budget <= 0 || max_active < 1) {
        vlm::setThreadError("vlm_server_create: bad argument");
        return VLM_ERR_BAD_ARG;
    }
    auto* s = new vlm_server;
    s->device = device;
    s->budget = hbm_budget;
    s->maxActive = max_active;
    s->t0 = Clock::now();
    s->dispatcher = std::thread([s] { s->dispatch(); });
    for (int i = 0; i < max_active; ++i) s->workers.emplace_back([s] { s->work(); });
    *out = s;
    return VLM_OK;
}

double vlm_server_clock(vlm_server* s) { return s ? s->now() : 0.0; }

vlm_status vlm_server_submit(vlm_server* s, const vlm_flow_request* r, int64_t* id) {
    if (!s || !r || !r->mesh || !r->ctrl || !r->u_type || !r->u_value || !r->p_type || !r->p_value) {
        vlm::setThreadError("vlm_server_submit: NULL argument");
        return VLM_ERR_BAD_ARG;
    }
    const vlm_mesh_desc& m = *r->mesh;
    if (!m.V || !m.Sf || !m.d || !m.w || !m.corrVecs || m.n_cells <= 0) {
        vlm::setThreadError("vlm_server_submit: the mesh needs its geometry");
        return VLM_ERR_BAD_ARG;
    }
    auto q = std::make_unique<Request>();
    const size_t nC = size_t(m.n_cells), nI = size_t(m.n_internal_faces), nF = size_t(m.n_faces),
                 nP = size_t(std::max(m.n_patches, 0));
    q->nCells = m.n_cells;
    q->nInternal = m.n_internal_faces;
    q->nFaces = m.n_faces;
    q->nPatches = m.n_patches;
    q->twoD = m.two_d;
    q->emptyDir = m.empty_dir;
    q->own = copyOf(m.owner, nF);
    q->nei = copyOf(m.neighbour, nI);
    q->magSf = copyOf(m.magSf, nF);
    q->ndc = copyOf(m.ndc, nF);
    q->V = copyOf(m.V, nC);
    q->Sf = copyOf(m.Sf, 3 * nF);
    q->d = copyOf(m.d, 3 * nF);
    q->w = copyOf(m.w, nF);
    q->corr = copyOf(m.corrVecs, 3 * nF);
    q->C = copyOf(m.C, 3 * nC);
    q->Cf = copyOf(m.Cf, 3 * nF);
    q->skew = copyOf(m.skewVecs, 3 * nF);
    q->patchStart = copyOf(m.patch_start, nP);
    q->patchSize = copyOf(m.patch_size, nP);
    const size_t nPb = std::max<size_t>(nP, 1);
    q->uType = copyOf(r->u_type, nPb);
    q->uValue = copyOf(r->u_value, 3 * nPb);
    q->pType = copyOf(r->p_type, nPb);
    q->pValue = copyOf(r->p_value, nPb);
    q->U0 = copyOf(r->U0, 3 * nC);
    q->p0 = copyOf(r->p0, nC);
    q->ctrl = *r->ctrl;
    // the Robin coefficients are the caller's arrays: the request keeps its own copies
    q->uRobin = copyOf(r->ctrl->u_robin, 2 * nPb);
    q->pRobin = copyOf(r->ctrl->p_robin, 2 * nPb);
    q->ctrl.u_robin = q->uRobin.empty() ? nullptr : q->uRobin.data();
    q->ctrl.p_robin = q->pRobin.empty() ? nullptr : q->pRobin.data();
    q->uAdv = copyOf(r->ctrl->u_advective, 4 * nPb);
    q->ctrl.u_advective = q->uAdv.empty() ? nullptr : q->uAdv.data();
    q->steady = r->ctrl->steady;
    q->nSteps = r->n_steps;
    q->dt = r->dt;
    q->maxIter = r->max_iter;
    q->tol = r->residual_tol;
    q->arrival = r->arrival;
    q->meshFlags = r->mesh_flags;
    q->bytes = r->device_bytes > 0 ? r->device_bytes : vlm_flow_request_bytes(m.n_cells, m.n_faces);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        q->id = s->nextId++;
        if (id) *id = q->id;
        // arrival order (stable for equal times)
        auto it = std::upper_bound(s->pending.begin(), s->pending.end(), q->arrival,
                                   [](double a, const std::unique_ptr<Request>& x) { return a < x->arrival; });
        s->pending.insert(it, std::move(q));
    }
    s->cv.notify_all();
    return VLM_OK;
}

vlm_status vlm_server_collect(vlm_server* s, vlm_flow_result* out, int32_t capacity, int32_t* n, double timeout) {
    if (!s || !n || (capacity > 0 && !out)) {
        vlm::setThreadError("vlm_server_collect: bad argument");
        return VLM_ERR_BAD_ARG;
    }
    std::unique_lock<std::mutex> lk(s->mu);
    if (timeout > 0 && s->doneOrder.empty())
        s->doneCv.wait_for(lk, std::chrono::duration<double>(timeout), [&] { return !s->doneOrder.empty(); });
    int32_t k = 0;
    size_t i = 0;
    for (; i < s->doneOrder.size() && k < capacity; ++i) out[k++] = s->done[s->doneOrder[i]].r;
    s->doneOrder.erase(s->doneOrder.begin(), s->doneOrder.begin() + long(i));
    *n = k;
    return VLM_OK;
}

vlm_status vlm_server_result_fields(vlm_server* s, int64_t id, double* U, double* p, double* phi) {
    if (!s) return VLM_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->done.find(id);
    if (it == s->done.end() || it->second.U.empty()) {
        vlm::setThreadError("vlm_server_result_fields: no fields for this request");
        return VLM_ERR_BAD_ARG;
    }
    if (U) std::copy(it->second.U.begin(), it->second.U.end(), U);
    if (p) std::copy(it->second.p.begin(), it->second.p.end(), p);
    if (phi) std::copy(it->second.phi.begin(), it->second.phi.end(), phi);
    return VLM_OK;
}

vlm_status vlm_server_destroy(vlm_server* s) {
    if (!s) return VLM_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->pending.clear();
    }
    s->cv.notify_all();
    s->dispatcher.join();
    for (auto& t : s->workers) t.join();
    delete s;
    return VLM_OK;
}

}  // extern "C"
