// Level-0 box products that stream z-planes through shared memory with bulk asynchronous copies.
//
// The four-slot kernels of boxkernels.cuh read every operand with per-thread vector loads: a row's
// six neighbours come from four other rows of the iterate, so each value of it is requested seven
// times and each coefficient twice, and with three CTAs of 256 threads per SM the loads in flight do
// not cover the DRAM latency (the FP64 product ran at 0.30 of the copy bandwidth).  Here a CTA owns
// y-pencils of TY x-rows (both colours, the whole x extent) over runs of z-planes.  The bulk-copy
// engine (cp.async.bulk, completing on one mbarrier per stage) fills a ring of S plane stages several
// planes ahead of the plane being computed; a plane's product reads its own stage, the p rows of the
// next plane's stage, and the previous plane's p and cz rows that each thread carried in registers,
// so every operand crosses DRAM once per launch (the y-halo rows of p and cy are read again from L2
// by the neighbouring pencil, and each run of planes reads one plane of p and cz on either side).
// Each consumer thread takes 16 bytes of slots (two FP64 or four FP32), so a warp's shared-memory
// loads cover consecutive words, and adds each row's terms in BoxGroup4::accumulate's order: the
// product is bit-identical to the four-slot kernels'.
//
// Every wait on a stage is bounded: a wait that gives up sets bit 1 of the level-0 error word and
// the CTA stops computing, waits (bounded) for the copies it has in flight, and still takes part in
// the reduction, so the per-system counters stay consistent.
#pragma once

#include "boxkernels.cuh"

namespace vlm {

// ---------------------------------------------------------------- mbarrier and bulk-copy primitives
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint32_t bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Arrives on the barrier and adds `bytes` to the transaction count its current phase waits for;
// returns the barrier state before the arrival.
__device__ __forceinline__ uint64_t mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
    uint64_t state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
                 : "=l"(state)
                 : "r"(bar), "r"(bytes)
                 : "memory");
    return state;
}

// Plain arrival (count 1) on a barrier; returns the barrier state before it.
__device__ __forceinline__ uint64_t mbar_arrive(uint32_t bar) {
    uint64_t state;
    asm volatile("mbarrier.arrive.shared::cta.b64 %0, [%1];" : "=l"(state) : "r"(bar) : "memory");
    return state;
}

// One bounded test of phase `parity`: the thread may be suspended for up to about a microsecond.
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, P;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(1000u)
        : "memory");
    return ok != 0;
}

constexpr long long kStreamSpinLimit = 1ll << 20;  // tests of a stage before its wait gives up (about a second)

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long long n = 0; n < kStreamSpinLimit; ++n)
        if (mbar_try(bar, parity)) return true;
    return false;
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned) from global memory into this
// CTA's shared memory, completing on barrier `bar`.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// A thread's slot group in the streamed kernels: 16 bytes, two FP64 or four FP32 slots, so a warp's
// shared-memory vector load covers consecutive 16-byte words (no bank conflicts).
template <class T> struct SG {
    static constexpr int N = 16 / int(sizeof(T));
    T v[N];
};

__device__ __forceinline__ SG<float> ldg16s(const float* p) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    return SG<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ SG<double> ldg16s(const double* p) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    return SG<double>{{a.x, a.y}};
}
__device__ __forceinline__ void stg16(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void stg16(double* p, const double (&v)[2]) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
}

// ---------------------------------------------------------------- plane stages
// One stage holds one z-plane of a y-pencil (rows j0 .. j0+TY-1 of both colours, H slots a row),
// elements of T at these offsets:
//   p  [2][TY + 2][H]  rows j0-1 .. j0+TY (the y halo, wrapped)
//   cx [2][TY][H]
//   cy [2][TY + 1][H]  rows j0-1 .. j0+TY-1
//   cz [2][TY][H]
//   dg [2][TY][H]
__host__ __device__ inline int stream_stage_elems(int H, int TY) { return 2 * (5 * TY + 3) * H; }

struct StreamStage {
    int H, TY;
    __device__ int p(int C, int r) const { return (C * (TY + 2) + r) * H; }
    __device__ int cx(int C, int r) const { return (2 * (TY + 2) + C * TY + r) * H; }
    __device__ int cy(int C, int r) const { return (2 * (2 * TY + 2) + C * (TY + 1) + r) * H; }
    __device__ int cz(int C, int r) const { return (2 * (3 * TY + 3) + C * TY + r) * H; }
    __device__ int dg(int C, int r) const { return (2 * (4 * TY + 3) + C * TY + r) * H; }
};

// The plane steps of one CTA: its pencil-planes [w0, w1) (w = pencil * nz + plane) split into runs
// inside one pencil; a run of n planes ka .. ka+n-1 takes n + 2 load steps, the planes ka-1 .. ka+n
// (wrapped): the first only p and cz rows (carried into the run's first plane), the last only p rows.
struct StreamWalker {
    int w;  // run start
    __device__ void run(int w1, int nz, int* P, int* ka, int* n) const {
        *P = w / nz;
        *ka = w - *P * nz;
        *n = min(nz - *ka, w1 - w);
    }
};

// Position of a step in the ring: its slot and the parity of the slot's phase that it fills.
struct RingPos {
    int slot;
    uint32_t par;
    __device__ RingPos next(int S) const { return slot + 1 == S ? RingPos{0, par ^ 1u} : RingPos{slot + 1, par}; }
};

// Ap = A p ; wApA = sum Ap.p ; alpha = wArA / wApA for one box system (k_box_pcg_spmv4's product and
// dot, range form).  Warp 0 is the producer: lane 0 issues each plane step's copies once its ring
// slot is empty.  The 2 * TY * H / N consumer threads behind it (colour C, x-row jj, slots m0 ..
// m0+N-1) wait for a step's copies on its full barrier and, after their last read of a step, each
// warp arrives on its empty barrier; there is no CTA-wide barrier per plane.  Requires H % 4 == 0,
// ny % TY == 0, nz >= 3, a multiple of 32 and at most 256 consumers, 3 <= S <= 8 stages, and
// gridDim.x <= the system's reduction slots.
constexpr int kStreamMaxThreads = 32 + 256;

template <class T, int FLAG>
__global__ void __launch_bounds__(kStreamMaxThreads, 2)
    k_box_pcg_spmv_stream(BoxSys B, int TY, int S, const T* __restrict__ coef, int nrows, const T* __restrict__ diag,
                          const T* __restrict__ p, T* __restrict__ Ap, RedCtx Rc, SysState* st, unsigned* err) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);  // S <= 8 full and 8 empty barriers: 128 bytes
    uint64_t* empty = full + 8;
    T* ring = reinterpret_cast<T*>(smem + 128);
    __shared__ volatile int sAbort;
    pdl_launch();
    const int H = B.H, ny = B.ny, nz = B.nz;
    const int E = stream_stage_elems(H, TY);
    const StreamStage L{H, TY};
    const int consumerWarps = int(blockDim.x >> 5) - 1;
    if (threadIdx.x == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(smem_addr(full + i), 1);
            mbar_init(smem_addr(empty + i), unsigned(consumerWarps));
        }
        mbar_fence_init();
        sAbort = 0;
    }
    __syncthreads();
    pdl_wait();
    if (sys_idle(st[0], FLAG)) return;

    const int W = (ny / TY) * nz;
    const int w0 = int((long long)blockIdx.x * W / gridDim.x);
    const int w1 = int((long long)(blockIdx.x + 1) * W / gridDim.x);
    long long issued = 0;
    DD dot[4] = {DD{0.0, 0.0}, DD{0.0, 0.0}, DD{0.0, 0.0}, DD{0.0, 0.0}};  // one chain per slot
    if (threadIdx.x < 32) {
        // ---------------------------------------------------------------- producer
        if (threadIdx.x == 0) {
            const T* cx = coef;
            const T* cy = coef + nrows;
            const T* cz = coef + 2 * size_t(nrows);
            const uint32_t rowB = uint32_t(H) * uint32_t(sizeof(T));
            RingPos q{0, 0u};  // the next step's position
            for (int w = w0; w < w1 && !sAbort;) {
                int P, ka, n;
                StreamWalker{w}.run(w1, nz, &P, &ka, &n);
                const int j0 = P * TY;
                const int jm = j0 > 0 ? j0 - 1 : ny - 1, jp = j0 + TY < ny ? j0 + TY : 0;
                for (int t = 0; t < n + 2; ++t) {
                    const int slot = q.slot;
                    // the slot's previous step (issued - S, the phase before) must be released by
                    // every consumer warp
                    if (issued >= S && !mbar_wait(smem_addr(empty + slot), q.par ^ 1u)) {
                        sAbort = 1;
                        break;
                    }
                    const int kk = ka - 1 + t;
                    const int plane = kk < 0 ? kk + nz : (kk >= nz ? kk - nz : kk);
                    T* stg = ring + size_t(slot) * E;
                    const uint32_t bar = smem_addr(full + slot);
                    const bool main = t >= 1 && t <= n;
                    const bool withCz = t <= n;
                    uint32_t bytes = 2u * TY * rowB;
                    if (main) bytes += 2u * (2u + TY + (TY + 1) + TY) * rowB;
                    if (withCz) bytes += 2u * TY * rowB;
                    (void)mbar_arrive_tx(bar, bytes);
#pragma unroll
                    for (int C = 0; C < 2; ++C) {
                        const size_t base = size_t(C ? B.base1 : B.base0) + size_t(plane) * ny * H;
                        bulk_load(smem_addr(stg + L.p(C, 1)), p + base + size_t(j0) * H, TY * rowB, bar);
                        if (withCz) bulk_load(smem_addr(stg + L.cz(C, 0)), cz + base + size_t(j0) * H, TY * rowB, bar);
                        if (main) {
                            bulk_load(smem_addr(stg + L.p(C, 0)), p + base + size_t(jm) * H, rowB, bar);
                            bulk_load(smem_addr(stg + L.p(C, TY + 1)), p + base + size_t(jp) * H, rowB, bar);
                            bulk_load(smem_addr(stg + L.cx(C, 0)), cx + base + size_t(j0) * H, TY * rowB, bar);
                            bulk_load(smem_addr(stg + L.cy(C, 0)), cy + base + size_t(jm) * H, rowB, bar);
                            bulk_load(smem_addr(stg + L.cy(C, 1)), cy + base + size_t(j0) * H, TY * rowB, bar);
                            bulk_load(smem_addr(stg + L.dg(C, 0)), diag + base + size_t(j0) * H, TY * rowB, bar);
                        }
                    }
                    ++issued;
                    q = q.next(S);
                }
                w += n;
            }
        }
    } else {
        // ---------------------------------------------------------------- consumers
        constexpr int N = SG<T>::N;
        const int tpr = H / N;
        const int tc = int(threadIdx.x) - 32;
        const int C = tc / (TY * tpr);
        const int o = 1 - C;
        const int rem = tc - C * TY * tpr;
        const int jj = rem / tpr;
        const int m0 = N * (rem - jj * tpr);
        const bool leader = (threadIdx.x & 31) == 0;
        const bool px = B.per & 1, py = B.per & 2, pz = B.per & 4;
        RingPos pos{0, 0u};  // this consumer's next step
        bool ok = true;
        auto wait_full = [&](RingPos r) {
            if (ok && !mbar_wait(smem_addr(full + r.slot), r.par)) {
                ok = false;
                sAbort = 1;
            }
        };
        auto release = [&](RingPos r) {  // this warp's last read of the step at r is done
            __syncwarp();
            if (leader) (void)mbar_arrive(smem_addr(empty + r.slot));
        };
        SG<T> pmo, czmo;  // the previous plane's p and cz of the other colour at this thread's slots
        for (int w = w0; w < w1 && ok;) {
            int P, ka, n;
            StreamWalker{w}.run(w1, nz, &P, &ka, &n);
            const int j = P * TY + jj;
            const RingPos p0 = pos;  // the run's first step: plane ka - 1
            wait_full(p0);
            {
                const T* sg = ring + size_t(p0.slot) * E;
                pmo = ldg16s(sg + L.p(o, jj + 1) + m0);
                czmo = ldg16s(sg + L.cz(o, jj) + m0);
            }
            release(p0);
            RingPos pcur = p0.next(S);
            const int fy = (j > 0 ? 2 : (py ? 2 << 6 : 0)) | (j < ny - 1 ? 16 : (py ? 16 << 6 : 0));
            for (int c = 0; c < n && ok; ++c) {
                const int k = ka + c;
                const RingPos pnxt = pcur.next(S);
                wait_full(pcur);
                wait_full(pnxt);
                if (sAbort) ok = false;
                const T* cur = ring + size_t(pcur.slot) * E;
                const T* nxt = ring + size_t(pnxt.slot) * E;
                const int par = (j + k + C) & 1;
                const int fz = (k > 0 ? 1 : (pz ? 1 << 6 : 0)) | (k < nz - 1 ? 32 : (pz ? 32 << 6 : 0));
                // the other colour's x-row: slots m0 .. m0+N-1 and the one just outside the group
                const T* xrow = cur + L.p(o, jj + 1);
                const int xe = par == 0 ? (m0 > 0 ? m0 - 1 : H - 1) : (m0 + N < H ? m0 + N : 0);
                const SG<T> xr = ldg16s(xrow + m0), xmy = ldg16s(cur + L.p(o, jj) + m0);
                const SG<T> xpy = ldg16s(cur + L.p(o, jj + 2) + m0), xpz = ldg16s(nxt + L.p(o, jj + 1) + m0);
                const SG<T> xmz = pmo;
                const T vx = xrow[xe];
                const SG<T> dg = ldg16s(cur + L.dg(C, jj) + m0), pc = ldg16s(cur + L.p(C, jj + 1) + m0);
                const SG<T> cpx = ldg16s(cur + L.cx(C, jj) + m0), cmx = ldg16s(cur + L.cx(o, jj) + m0);
                const SG<T> cpy = ldg16s(cur + L.cy(C, jj + 1) + m0), cmy = ldg16s(cur + L.cy(o, jj) + m0);
                const SG<T> cpz = ldg16s(cur + L.cz(C, jj) + m0), cmz = czmo;
                const T cme = par == 0 ? cur[L.cx(o, jj) + xe] : T(0);
                T s[N];
#pragma unroll
                for (int v = 0; v < N; ++v) {
                    // BoxGroup4::accumulate's terms for slot v, in its order: internal -z, -y, -x, +x,
                    // +y, +z, then the cyclic faces of x, y, z
                    const int i = 2 * (m0 + v) + par;
                    const int fx = (i > 0 ? 4 : (px ? 4 << 6 : 0)) | (i < B.nx - 1 ? 8 : (px ? 8 << 6 : 0));
                    const int f = fx | fy | fz;
                    const T am = par == 0 ? (v == 0 ? cme : cmx.v[v - 1]) : cmx.v[v];
                    const T vm = par == 0 ? (v == 0 ? vx : xr.v[v - 1]) : xr.v[v];
                    const T vp = par == 0 ? xr.v[v] : (v == N - 1 ? vx : xr.v[v + 1]);
                    T a = dg.v[v] * pc.v[v];
                    if (f & 1) a += cmz.v[v] * xmz.v[v];
                    if (f & 2) a += cmy.v[v] * xmy.v[v];
                    if (f & 4) a += am * vm;
                    if (f & 8) a += cpx.v[v] * vp;
                    if (f & 16) a += cpy.v[v] * xpy.v[v];
                    if (f & 32) a += cpz.v[v] * xpz.v[v];
                    if (f & (4 << 6)) a += am * vm;
                    if (f & (8 << 6)) a += cpx.v[v] * vp;
                    if (f & (2 << 6)) a += cmy.v[v] * xmy.v[v];
                    if (f & (16 << 6)) a += cpy.v[v] * xpy.v[v];
                    if (f & (1 << 6)) a += cmz.v[v] * xmz.v[v];
                    if (f & (32 << 6)) a += cpz.v[v] * xpz.v[v];
                    s[v] = a;
                }
                pmo = xr;
                czmo = ldg16s(cur + L.cz(o, jj) + m0);
                release(pcur);
                if (c == n - 1) release(pnxt);
                pcur = pnxt;
                const size_t row = size_t(C ? B.base1 : B.base0) + (size_t(k) * ny + j) * H + m0;
                stg16(Ap + row, s);
#pragma unroll
                for (int v = 0; v < N; ++v) dot[v & 3] = dd_add(dot[v & 3], DD{(double)s[v] * (double)pc.v[v], 0.0});
            }
            pos = pcur.next(S);  // pcur: the run's last step (plane ka + n)
            w += n;
        }
    }
    __syncthreads();
    if (sAbort) {
        // a wait gave up: flag it, and let the copies still in flight (at most the last S steps the
        // producer issued) land before the CTA's shared memory is released
        if (threadIdx.x == 0) {
            atomicOr(err, 2u);
            for (long long s = issued > S ? issued - S : 0; s < issued; ++s)
                mbar_wait(smem_addr(full + int(s % S)), uint32_t((s / S) & 1));
        }
        __syncthreads();
    }
    DD acc[1] = {dd_add(dd_add(dot[0], dot[1]), dd_add(dot[2], dot[3]))};
    double out[1];
    const int b = Rc.slotBegin[0];
    if (reduce_dd_span<1, kStreamMaxThreads / 32>(acc, b + int(blockIdx.x), 0, b, b + int(gridDim.x), Rc, out)) {
        SysState& q = st[0];
        if (fabs(out[0]) < kVSMALL) {
            if (FLAG == kFlagDone) {
                q.done = 1;
            } else {
                q.innerDone = 1;
                q.s1 = 1.0;
            }
        } else {
            q.alpha = q.wArA / out[0];
        }
    }
}

}  // namespace vlm
