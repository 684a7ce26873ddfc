// Device kernels of the LDU / GAMG solve path (sm_100a).
//
// All kernels are memory-bound row kernels over a SELL-32 layout: one thread per row,
// one warp per 32-row slice, so the entry arrays of a slice are read fully coalesced.
// Sums over a row's off-diagonal entries run in the row's face order, which is the order
// the reference accumulates them in (LinearSolver.cpp:121-133, GAMG.cpp:363-401); together
// with -fmad=false this makes every row update bit-identical to the reference's.
// No atomics touch floating-point data: reductions write one compensated partial per CTA
// and the last CTA of a system combines them in a fixed order.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"
#include "devtypes.h"
#include "exactsum.cuh"

namespace vlm {

// ------------------------------------------------------------------ programmatic dependent launch
// Every kernel of the solver is launched with programmatic stream serialisation: the next kernel
// may start (its CTAs become resident) while this one drains, and each kernel waits at entry until
// its predecessor has completed and its writes are visible (griddepcontrol.wait returns at once
// when the launch had no programmatic predecessor).  It then lets its own successor launch.
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Split form for the row kernels of the solve loop: the kernel lets its successor launch at once,
// loads what no earlier kernel of the loop writes (chunk descriptors, matrix structure, values and
// diagonals, transfer maps: fixed for a whole solve) while its predecessor drains, and only then
// waits for the predecessor's results.  On the small coarse levels this takes the dependent loads
// of the row structure off the critical path.
__device__ __forceinline__ void pdl_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }


constexpr double kVSMALL = 1.0e-300;  // core/Types.h VSMALL
constexpr double kGREAT = 1.0e15;     // core/Types.h GREAT


// ------------------------------------------------------------------ compensated sums

__device__ __forceinline__ DD dd_add(DD a, DD b) {
    // TwoSum of the leading parts, trailing parts added, then renormalised.
    const double s = a.hi + b.hi;
    const double bb = s - a.hi;
    const double e = (a.hi - (s - bb)) + (b.hi - bb);
    const double t = a.lo + b.lo + e;
    const double hi = s + t;
    const double lo = t - (hi - s);
    return DD{hi, lo};
}

__device__ __forceinline__ DD dd_shfl_down(DD v, int o) {
    return DD{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
}

// Reduces NV values over the CTA (fixed tree), returns the totals in thread 0.
template <int NV, int MAXW = kRowsPerCta / 32>
__device__ __forceinline__ void block_reduce(DD (&v)[NV]) {
    __shared__ DD sm[NV][MAXW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] = dd_add(v[q], dd_shfl_down(v[q], o));
        if (lane == 0) sm[q][warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            v[q] = lane < (int)(blockDim.x >> 5) ? sm[q][lane] : DD{0.0, 0.0};
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[q] = dd_add(v[q], dd_shfl_down(v[q], o));
        }
    }
}


// Writes this CTA's partials into `slot`; returns true in thread 0 of the CTA that completes
// system `sys`, whose CTAs write the slots [b, e), with the totals (summed over the slots in a
// fixed order) in `out`.
template <int NV, int MAXW = kRowsPerCta / 32>
__device__ bool reduce_dd_span(DD (&v)[NV], int slot, int sys, int b, int e, const RedCtx& R, double (&out)[NV]) {
    block_reduce<NV, MAXW>(v);
    __shared__ int isLast;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) R.partials[(size_t)slot * NV + q] = v[q];
        __threadfence();
        const int ticket = atomicAdd(&R.counters[sys], 1);
        isLast = ticket == e - b - 1;
    }
    __syncthreads();
    if (!isLast) return false;
    __threadfence();
    DD acc[NV];
#pragma unroll
    for (int q = 0; q < NV; ++q) acc[q] = DD{0.0, 0.0};
    // slots s = b + t + 256 m, combined in ascending m; loads issued 4 at a time
    const double2* P = reinterpret_cast<const double2*>(R.partials);
    int s = b + (int)threadIdx.x;
    for (; s + 3 * (int)blockDim.x < e; s += 4 * blockDim.x) {
        double2 w[4][NV];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < NV; ++q) w[u][q] = __ldcg(&P[(size_t)(s + u * blockDim.x) * NV + q]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int q = 0; q < NV; ++q) acc[q] = dd_add(acc[q], DD{w[u][q].x, w[u][q].y});
    }
    for (; s < e; s += blockDim.x)
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            const double2 w = __ldcg(&P[(size_t)s * NV + q]);
            acc[q] = dd_add(acc[q], DD{w.x, w.y});
        }
    __syncthreads();  // the shared tree below is reused
    block_reduce<NV, MAXW>(acc);
    if (threadIdx.x != 0) return false;
    R.counters[sys] = 0;
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = acc[q].hi + acc[q].lo;
    return true;
}

// reduce_dd_span over the slots of chunk c's system, one slot per chunk.
template <int NV>
__device__ bool reduce_dd(DD (&v)[NV], const Chunk& c, const RedCtx& R, double (&out)[NV]) {
    return reduce_dd_span<NV>(v, c.slot, c.sys, R.slotBegin[c.sys], R.slotEnd[c.sys], R, out);
}

// Writes this CTA's exact bins as its partial; the last CTA of the system adds every partial
// (int64, exact in any order) and converts the total like binsToDouble.
template <int NV>
__device__ bool reduce_exact_bins(long long (*bins)[kRowsPerCta / 32][kExactBins], int (*flags)[kRowsPerCta / 32],
                                  const Chunk& c, const RedCtx& R, double (&out)[NV]) {
    constexpr int kWarps = kRowsPerCta / 32;
    __shared__ int isLast;
    __syncthreads();
    long long* dst = R.xbins + (size_t)c.slot * NV * kExactStride;
    for (int idx = threadIdx.x; idx < NV * kExactBins; idx += blockDim.x) {
        const int q = idx / kExactBins, k = idx % kExactBins;
        long long s = 0;
        for (int w = 0; w < kWarps; ++w) s += bins[q][w][k];
        dst[q * kExactStride + k] = s;
    }
    if ((int)threadIdx.x < NV) {
        int f = 0;
        for (int w = 0; w < kWarps; ++w) f |= flags[threadIdx.x][w];
        dst[threadIdx.x * kExactStride + kExactBins] = f;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nslots = R.slotEnd[c.sys] - R.slotBegin[c.sys];
        isLast = atomicAdd(&R.counters[c.sys], 1) == nslots - 1;
    }
    __syncthreads();
    if (!isLast) return false;
    __threadfence();
    __shared__ long long tot[NV][kExactStride];
    const int b0 = R.slotBegin[c.sys], b1 = R.slotEnd[c.sys];
    for (int idx = threadIdx.x; idx < NV * kExactStride; idx += blockDim.x) {
        const int q = idx / kExactStride, k = idx % kExactStride;
        long long s = 0;
        for (int sl = b0; sl < b1; ++sl) {
            const long long v = __ldcg(R.xbins + (size_t)sl * NV * kExactStride + q * kExactStride + k);
            if (k < kExactBins)
                s += v;
            else
                s |= v;
        }
        tot[q][k] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return false;
    R.counters[c.sys] = 0;
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = exact_value(tot[q], (int)tot[q][kExactBins]);
    return true;
}

template <int NV>
__device__ bool reduce_exact(DD (&v)[NV], const Chunk& c, const RedCtx& R, double (&out)[NV]) {
    constexpr int kWarps = kRowsPerCta / 32;
    __shared__ long long bins[NV][kWarps][kExactBins];
    __shared__ int flags[NV][kWarps];
    for (int q = threadIdx.x; q < NV * kWarps * kExactBins; q += blockDim.x) (&bins[0][0][0])[q] = 0;
    if ((int)threadIdx.x < NV * kWarps) (&flags[0][0])[threadIdx.x] = 0;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) exact_add(bins[q][threadIdx.x >> 5], &flags[q][threadIdx.x >> 5], v[q].hi);
    return reduce_exact_bins<NV>(bins, flags, c, R, out);
}

template <int NV, bool EXACT = false>
__device__ __forceinline__ bool reduce_to_system(DD (&v)[NV], const Chunk& c, const RedCtx& R, double (&out)[NV]) {
    if constexpr (EXACT)
        return reduce_exact<NV>(v, c, R, out);
    else
        return reduce_dd<NV>(v, c, R, out);
}

// Per-CTA accumulator used by the reduction kernels: add() values (any number per thread),
// then finish() -> true in the thread that completes the system, with the totals.
template <int NV, bool EXACT> struct BlockSum;

template <int NV> struct BlockSum<NV, false> {
    DD v[NV];
    __device__ void begin() {
#pragma unroll
        for (int q = 0; q < NV; ++q) v[q] = DD{0.0, 0.0};
    }
    __device__ void add(int q, double x) { v[q] = dd_add(v[q], DD{x, 0.0}); }
    __device__ bool finish(const Chunk& c, const RedCtx& R, double (&out)[NV]) { return reduce_dd<NV>(v, c, R, out); }
};

template <int NV> struct BlockSum<NV, true> {
    static constexpr int kWarps = kRowsPerCta / 32;
    long long (*bins)[kWarps][kExactBins];
    int (*flags)[kWarps];
    __device__ void begin() {
        __shared__ long long b[NV][kWarps][kExactBins];
        __shared__ int f[NV][kWarps];
        bins = b;
        flags = f;
        for (int q = threadIdx.x; q < NV * kWarps * kExactBins; q += blockDim.x) (&b[0][0][0])[q] = 0;
        if ((int)threadIdx.x < NV * kWarps) (&f[0][0])[threadIdx.x] = 0;
        __syncthreads();
    }
    __device__ void add(int q, double x) { exact_add(bins[q][threadIdx.x >> 5], &flags[q][threadIdx.x >> 5], x); }
    __device__ bool finish(const Chunk& c, const RedCtx& R, double (&out)[NV]) {
        return reduce_exact_bins<NV>(bins, flags, c, R, out);
    }
};

// Exact sum of a plain array (vlm_exact_sum): one system, chunks of kRowsPerCta values.
__global__ void __launch_bounds__(kRowsPerCta) k_exact_sum(const Chunk* __restrict__ ch, const double* __restrict__ v,
                                                           RedCtx R, double* out) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    DD a[1] = {DD{0.0, 0.0}};
    if ((int)threadIdx.x < c.count) a[0].hi = v[c.start + threadIdx.x];
    double o[1];
    if (reduce_exact<1>(a, c, R, o)) *out = o[0];
}

// ------------------------------------------------------------------ SELL row access

__device__ __forceinline__ int sell_base(const Sell& S, int row) { return __ldg(S.slPtr + (row >> 5)) + (row & 31); }

// s -= (MINUS) or += a_row,e * X(col_e) over the row's entries in entry order.  The loads are issued
// in batches of kRowBatch (all column indices and values, then all gathers, then the arithmetic in
// order), so a row costs two memory round trips instead of two per entry; the arithmetic and its
// order are those of the plain entry loop.
constexpr int kRowBatch = 8;

// The matrix (structure and values) is read-only in every kernel that walks rows, so it is read
// through the non-coherent cache; how X is read is the caller's choice (xf).
template <bool MINUS, class T, class XF, int B = kRowBatch>
__device__ __forceinline__ T row_accumulate(const Sell& S, const T* __restrict__ val, XF xf, int row, T s) {
    const int len = __ldg(S.rlen + row);
    const int base = sell_base(S, row);
    if (B == 1) {
        for (int k = 0; k < len; ++k) {
            const int e = base + (k << 5);
            if (MINUS)
                s -= __ldg(val + e) * xf(__ldg(S.col + e));
            else
                s += __ldg(val + e) * xf(__ldg(S.col + e));
        }
        return s;
    }
    for (int k0 = 0; k0 < len; k0 += B) {
        int cj[B];
        T a[B], xv[B];
#pragma unroll
        for (int q = 0; q < B; ++q)
            if (k0 + q < len) {
                const int e = base + ((k0 + q) << 5);
                cj[q] = __ldg(S.col + e);
                a[q] = __ldg(val + e);
            }
#pragma unroll
        for (int q = 0; q < B; ++q)
            if (k0 + q < len) xv[q] = xf(cj[q]);
#pragma unroll
        for (int q = 0; q < B; ++q)
            if (k0 + q < len) {
                if (MINUS)
                    s -= a[q] * xv[q];
                else
                    s += a[q] * xv[q];
            }
    }
    return s;
}

// x must not be written by the running kernel (it is read through the non-coherent cache).
template <class T>
__device__ __forceinline__ T row_minus(const Sell& S, const T* __restrict__ val, const T* __restrict__ x, int row, T s) {
    return row_accumulate<true>(S, val, [&](int j) { return __ldg(x + j); }, row, s);
}

template <class T>
__device__ __forceinline__ T row_plus(const Sell& S, const T* __restrict__ val, const T* __restrict__ x, int row, T s) {
    return row_accumulate<false>(S, val, [&](int j) { return __ldg(x + j); }, row, s);
}

// The first P entries of a SELL row (structure and values) loaded ahead of the gathers: before the
// kernel waits for its predecessor.  accumulate() then gathers X and sums every entry in entry order
// (entries past P are loaded there, in batches), the same arithmetic as row_accumulate.
constexpr int kRowPre = 16;

template <class T, int P = kRowPre>
struct RowPre {
    int len = 0, base = 0;
    int col[P];
    T a[P];
    __device__ __forceinline__ void load(const Sell& S, const T* __restrict__ val, int row) {
        len = __ldg(S.rlen + row);
        base = sell_base(S, row);
#pragma unroll
        for (int q = 0; q < P; ++q)
            if (q < len) {
                const int e = base + (q << 5);
                col[q] = __ldg(S.col + e);
                a[q] = __ldg(val + e);
            }
    }
    template <bool MINUS, class XF>
    __device__ __forceinline__ T accumulate(const Sell& S, const T* __restrict__ val, XF xf, T s) const {
        T xv[P];
#pragma unroll
        for (int q = 0; q < P; ++q)
            if (q < len) xv[q] = xf(col[q]);
#pragma unroll
        for (int q = 0; q < P; ++q)
            if (q < len) {
                if (MINUS)
                    s -= a[q] * xv[q];
                else
                    s += a[q] * xv[q];
            }
        for (int k = P; k < len; ++k) {  // rows longer than P: one entry at a time
            const int e = base + (k << 5);
            if (MINUS)
                s -= __ldg(val + e) * xf(__ldg(S.col + e));
            else
                s += __ldg(val + e) * xf(__ldg(S.col + e));
        }
        return s;
    }
};

// Which SysState flag a kernel honours: the outer "done" or the inner-solve "innerDone".
enum : int { kFlagDone = 0, kFlagInner = 1 };

__device__ __forceinline__ bool sys_idle(const SysState& s, int flag) {
    return flag == kFlagDone ? s.done != 0 : (s.innerDone != 0 || s.done != 0);
}

__device__ __forceinline__ bool chunk_skip(const Chunk& c, const SysState* st, int flag) {
    return st != nullptr && sys_idle(st[c.sys], flag);
}

// x = 0 on the rows of the chunks (multicolour GS starts from zero)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_zero_rows(const Chunk* __restrict__ ch, T* __restrict__ x,
                                                           const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    for (int row = c.start + threadIdx.x; row < c.start + c.count; row += kRowsPerCta) x[row] = T(0);
}

// w = r on the rows of the chunks (the "none" preconditioner)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_copy_rows(const Chunk* __restrict__ ch, const T* __restrict__ r,
                                                           T* __restrict__ w, const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    for (int row = c.start + threadIdx.x; row < c.start + c.count; row += kRowsPerCta) w[row] = r[row];
}

// b = (To) a on the rows of the chunks
template <class From, class To>
__global__ void __launch_bounds__(kRowsPerCta) k_cast_rows(const Chunk* __restrict__ ch, const From* __restrict__ a,
                                                           To* __restrict__ b, const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    for (int row = c.start + threadIdx.x; row < c.start + c.count; row += kRowsPerCta) b[row] = (To)a[row];
}

// ------------------------------------------------------------------ smoothers
// Gauss-Seidel row update (GAMG.cpp:368-380) on the rows of one colour step.  Neighbours belong to
// other colours and are not written by this launch.
// MODE 0: plain.  MODE 1: first colour of a sweep from x = 0 (every neighbour is still zero:
// x = r / D without reading the row).  MODE 2: first colour of the first post-sweep of a
// two-colour level; the neighbours (the other colour, not yet swept) get the coarse-grid
// correction x + xc[agg] (GAMG.cpp:437-438) on the fly, which replaces the separate prolongation.
// The colour step is bound by the latency of its three dependent loads per row (structure, entries,
// gathers): the more rows in flight per SM the better.  Batches of 6 entries (one batch for the
// rows of a hex mesh) fit 32 registers in FP32, so 8 CTAs of 256 threads stay resident.
template <class T, int MODE = 0>
__global__ void __launch_bounds__(kRowsPerCta, sizeof(T) == 4 ? 6 : 4) k_smooth_gs(const Chunk* __restrict__ ch, Sell S, const T* __restrict__ val,
                                                           const T* __restrict__ diag, const T* __restrict__ r, T* x,
                                                           const int32_t* __restrict__ agg, const T* __restrict__ xc,
                                                           const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    if ((int)threadIdx.x >= c.count) return;
    const int row = c.start + threadIdx.x;
    const T dg = __ldg(diag + row);
    RowPre<T, 6> pre;
    if (MODE != 1) pre.load(S, val, row);
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    if (MODE == 1) {
        x[row] = r[row] / dg;
        return;
    }
    auto xf = [&](int j) -> T {
        T v = __ldg(x + j);
        if (MODE == 2) {
            const int a = __ldg(agg + j);
            if (a >= 0) v += __ldg(xc + a);
        }
        return v;
    };
    const T s = pre.template accumulate<true>(S, val, xf, r[row]);
    x[row] = s / dg;
}

// Block-hybrid Gauss-Seidel sweep.  One CTA per block of <= kBlockRows rows: the block's x lives
// in shared memory and is updated colour by colour (block-local colouring, forward or reversed
// order); neighbours outside the block are read from xi (the previous sweep), so the result does
// not depend on the order CTAs run in.  Each thread reads its row once per sweep: the terms of
// neighbours outside the block are summed first (face order), the in-block entries are kept in
// registers, and every colour step then subtracts the in-block terms (face order) from shared
// memory — no global-memory latency inside the synchronised colour loop.
// x_i = (r_i - sum_out a_ij x_j - sum_in a_ij x_j) / a_ii.
// MODE 0: x = xi; MODE 1: x starts at 0 (first pre-sweep); MODE 2: x = xi + xc[agg] (the
// coarse-grid correction of GAMG.cpp:437-438, fused in).
constexpr int kBgsRegEntries = 24;  // in-block entries held in registers; longer rows spill to loads

template <class T, int MODE, bool FWD>
__global__ void __launch_bounds__(kBlockRows, 1) k_smooth_bgs(const Chunk* __restrict__ blocks, Sell S,
                                                              const T* __restrict__ val, const T* __restrict__ diag,
                                                              const T* __restrict__ r, const T* __restrict__ xi,
                                                              T* __restrict__ xo, const int8_t* __restrict__ rcol,
                                                              const int32_t* __restrict__ agg,
                                                              const T* __restrict__ xc, const SysState* st, int flag) {
    pdl_entry();
    __shared__ T xs[kBlockRows + 1];  // xs[kBlockRows] == 0: target of inactive register slots
    const Chunk c = blocks[blockIdx.x];
    if (chunk_skip(c, st, flag)) return;
    const int t = threadIdx.x;
    const bool mine = t < c.count;
    const int row = c.start + t;
    auto xval = [&](int j) -> T {
        if (MODE == 1) return T(0);
        T v = xi[j];
        if (MODE == 2) {
            const int a = agg[j];
            if (a >= 0) v += xc[a];
        }
        return v;
    };
    if (t == 0) xs[kBlockRows] = T(0);
    const int len = mine ? S.rlen[row] : 0;
    const int base = mine ? sell_base(S, row) : 0;
    T s = mine ? r[row] : T(0);
    int16_t li[kBgsRegEntries];
    T lv[kBgsRegEntries];
#pragma unroll
    for (int k = 0; k < kBgsRegEntries; ++k) {
        li[k] = kBlockRows;  // the zero slot: q -= 0 * 0 leaves q unchanged bit for bit
        lv[k] = T(0);
        if (k < len) {
            const int e = base + (k << 5);
            const int j = S.col[e];
            const T a = val[e];
            const int jl = j - c.start;
            if (jl >= 0 && jl < c.count) {
                li[k] = (int16_t)jl;
                lv[k] = a;
            } else {
                s -= a * xval(j);
            }
        }
    }
    for (int k = kBgsRegEntries; k < len; ++k) {  // rare: rows longer than the register window
        const int e = base + (k << 5);
        const int jl = S.col[e] - c.start;
        if (!(jl >= 0 && jl < c.count)) s -= val[e] * xval(S.col[e]);
    }
    if (mine) xs[t] = xval(row);
    __syncthreads();
    const int nc = c.slot;
    const int mycol = mine ? (int)rcol[row] : -1;
    const T dd = mine ? diag[row] : T(1);
    for (int step = 0; step < nc; ++step) {
        const int colour = FWD ? step : nc - 1 - step;
        if (mycol == colour) {
            T q = s;
#pragma unroll
            for (int k = 0; k < kBgsRegEntries; ++k) q -= lv[k] * xs[li[k]];
            for (int k = kBgsRegEntries; k < len; ++k) {
                const int e = base + (k << 5);
                const int jl = S.col[e] - c.start;
                if (jl >= 0 && jl < c.count) q -= val[e] * xs[jl];
            }
            xs[t] = q / dd;
        }
        __syncthreads();
    }
    if (mine) xo[row] = xs[t];
}

// Jacobi sweep xo = (r - offdiag*xi)/D.  MODE 0: plain; MODE 1: xi == 0 (first pre-sweep);
// MODE 2: xi + xc[agg] (the coarse-grid correction, GAMG.cpp:437-438, fused in); MODE 3: both
// pre-sweeps from zero in one pass (the neighbours' first-sweep values recomputed from r and D).
// Launch bounds: 3 resident CTAs per SM for FP32 (at most 80 registers: the 16 preloaded entries of
// RowPre), 2 for FP64.
template <class T, int MODE>
__global__ void __launch_bounds__(kRowsPerCta, sizeof(T) == 4 ? 3 : 2) k_smooth_jacobi(const Chunk* __restrict__ ch, Sell S,
                                                               const T* __restrict__ val, const T* __restrict__ diag,
                                                               const T* __restrict__ r, const T* __restrict__ xi,
                                                               T* __restrict__ xo, T omega,
                                                               const int32_t* __restrict__ agg,
                                                               const T* __restrict__ xc, const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    // the thread's first row: structure, values and diagonal ahead of the wait
    const int row0 = c.start + threadIdx.x;
    const bool has = (int)threadIdx.x < c.count;
    RowPre<T> pre;
    T d0 = T(1);
    if (has) {
        d0 = __ldg(diag + row0);
        if (MODE != 1) pre.load(S, val, row0);
    }
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    auto xv = [&](int j) -> T {
        if (MODE == 3) {
            // the first sweep from zero, recomputed where the second reads it (the MODE 1 value)
            const T v = __ldg(r + j) / __ldg(diag + j);
            return omega == T(1) ? v : omega * v;
        }
        T v = __ldg(xi + j);
        if (MODE == 2) {
            const int a = __ldg(agg + j);
            if (a >= 0) v += __ldg(xc + a);
        }
        return v;
    };
    // chunks of up to kRowsPerCta rows (one pass), or wider level-0 chunks (strided)
    T dg = d0;
    for (int row = row0; row < c.start + c.count; row += kRowsPerCta) {
        if (row != row0) {
            dg = diag[row];
            if (MODE != 1) pre.load(S, val, row);
        }
        if (MODE == 1) {
            const T v = r[row] / dg;
            xo[row] = omega == T(1) ? v : omega * v;
            continue;
        }
        const T s = pre.template accumulate<true>(S, val, xv, r[row]);
        const T v = s / dg;
        if (omega == T(1)) {
            xo[row] = v;
        } else {
            const T x0 = xv(row);
            xo[row] = x0 + omega * (v - x0);
        }
    }
}

// res = r - A x  (GAMG.cpp:387-401: diagonal first, then the faces in order)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta, sizeof(T) == 4 ? 4 : 2) k_residual(const Chunk* __restrict__ ch, Sell S, const T* __restrict__ val,
                                                          const T* __restrict__ diag, const T* __restrict__ r,
                                                          const T* __restrict__ x, T* __restrict__ res,
                                                          const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    if ((int)threadIdx.x >= c.count) return;
    const int row = c.start + threadIdx.x;
    RowPre<T> pre;
    pre.load(S, val, row);
    const T dg = __ldg(diag + row);
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    res[row] = pre.template accumulate<true>(S, val, [&](int j) { return __ldg(x + j); }, r[row] - dg * x[row]);
}

// rc[R] = sum of res over the children of R in ascending natural order (GAMG.cpp:434-435)
constexpr int kChildPre = 8;

template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_restrict(const Chunk* __restrict__ ch, const int32_t* __restrict__ cptr,
                                                          const int32_t* __restrict__ child, const T* __restrict__ res,
                                                          T* __restrict__ rc, const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    if ((int)threadIdx.x >= c.count) return;
    const int R = c.start + threadIdx.x;
    const int k0 = __ldg(cptr + R), k1 = __ldg(cptr + R + 1);
    int kid[kChildPre];
#pragma unroll
    for (int q = 0; q < kChildPre; ++q)
        if (k0 + q < k1) kid[q] = __ldg(child + k0 + q);
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    T v[kChildPre];
#pragma unroll
    for (int q = 0; q < kChildPre; ++q)
        if (k0 + q < k1) v[q] = res[kid[q]];
    T s = T(0);
#pragma unroll
    for (int q = 0; q < kChildPre; ++q)
        if (k0 + q < k1) s += v[q];
    for (int k = k0 + kChildPre; k < k1; ++k) s += res[child[k]];
    rc[R] = s;
}

// k_residual and k_restrict in one pass over the coarse rows: each aggregate computes its
// children's residuals (the same row operations as k_residual) and sums them in child order, as
// k_restrict sums the stored ones.  For coarse levels, where a launch costs more than the
// scattered row reads it saves.
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_residual_restrict(const Chunk* __restrict__ ch, Sell S,
                                                                   const T* __restrict__ val,
                                                                   const T* __restrict__ diag, const T* __restrict__ r,
                                                                   const T* __restrict__ x,
                                                                   const int32_t* __restrict__ cptr,
                                                                   const int32_t* __restrict__ child,
                                                                   T* __restrict__ rc, const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    if ((int)threadIdx.x >= c.count) return;
    const int R = c.start + threadIdx.x;
    const int k0 = __ldg(cptr + R), k1 = __ldg(cptr + R + 1);
    int i0 = 0;
    RowPre<T, 8> pre;
    T dg = T(1);
    if (k0 < k1) {  // the first child's structure, values and diagonal ahead of the wait
        i0 = __ldg(child + k0);
        pre.load(S, val, i0);
        dg = __ldg(diag + i0);
    }
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    auto xf = [&](int j) { return __ldg(x + j); };
    T s = T(0);
    for (int k = k0; k < k1; ++k) {
        int i = i0;
        if (k != k0) {
            i = __ldg(child + k);
            pre.load(S, val, i);
            dg = __ldg(diag + i);
        }
        s += pre.template accumulate<true>(S, val, xf, r[i] - dg * x[i]);
    }
    rc[R] = s;
}

// x += xc[agg]  (GAMG.cpp:437-438)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_prolong(const Chunk* __restrict__ ch, const int32_t* __restrict__ agg,
                                                         const T* __restrict__ xc, T* __restrict__ x, const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    if ((int)threadIdx.x >= c.count) return;
    const int row = c.start + threadIdx.x;
    const int a = __ldg(agg + row);
    pdl_wait();
    if (chunk_skip(c, st, flag)) return;
    if (a >= 0) x[row] += xc[a];
}

// ------------------------------------------------------------------ coarsest level

// Dense coarsest matrix, un-pivoted LU in place (GAMG.cpp:317-343) and the explicit
// inverse from the LU by substituting unit vectors (GAMG.cpp:413-418 per column).
// One CTA per system.  The factorisation runs in shared memory when the matrix fits
// (smemN >= n: 2 n^2 doubles of dynamic shared memory), else in the global scratch `lu`.
__global__ void k_coarse_factor(const CoarseDev* __restrict__ cs, Sell S, const double* __restrict__ val,
                                const double* __restrict__ diag, double* __restrict__ lu, double* __restrict__ inv,
                                int* status, int smemN) {
    pdl_entry();
    extern __shared__ double sh[];
    const CoarseDev c = cs[blockIdx.x];
    const int n = c.n;
    const bool inShared = n <= smemN;
    double* A = inShared ? sh : lu + c.invOffset;
    double* X = inShared ? sh + (size_t)n * n : inv + c.invOffset;
    for (int q = threadIdx.x; q < n * n; q += blockDim.x) A[q] = 0.0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int row = c.rowStart + i;
        A[(size_t)i * n + i] = diag[row];
        const int len = S.rlen[row], base = sell_base(S, row);
        for (int k = 0; k < len; ++k) {
            const int e = base + (k << 5);
            A[(size_t)i * n + (S.col[e] - c.rowStart)] += val[e];
        }
    }
    __syncthreads();
    // LU without pivoting, one pivot at a time: multipliers of column k, then the trailing block
    // element-parallel (each element receives its updates in the order k = 0, 1, ...).  The block
    // loops run over a (blockDim.x / 32) x 32 grid of rows x columns (no index division).
    const int nt = blockDim.x;
    const int tx = int(threadIdx.x) & 31, ty = int(threadIdx.x) >> 5, ny = nt >> 5;
    for (int k = 0; k < n; ++k) {
        const double piv = A[(size_t)k * n + k];
        if (fabs(piv) < kVSMALL) {  // uniform: every thread reads the same pivot
            if (threadIdx.x == 0) atomicExch(status, (int)VLM_ERR_SINGULAR);
            return;
        }
        for (int i = k + 1 + threadIdx.x; i < n; i += nt) A[(size_t)i * n + k] /= piv;
        __syncthreads();
        for (int i = k + 1 + ty; i < n; i += ny) {
            const double fct = A[(size_t)i * n + k];
            if (fct == 0.0) continue;
            for (int j = k + 1 + tx; j < n; j += 32) A[(size_t)i * n + j] -= fct * A[(size_t)k * n + j];
        }
        __syncthreads();
    }
    // inverse = U^-1 L^-1, all columns at once.  Forward (unit L): X = I, then for k ascending
    // X[i][j] -= L[i][k] X[k][j] for i > k (X[k][j] = 0 for j > k, so j <= k).
    for (int i = ty; i < n; i += ny)
        for (int j = tx; j < n; j += 32) X[(size_t)i * n + j] = i == j ? 1.0 : 0.0;
    __syncthreads();
    for (int k = 0; k + 1 < n; ++k) {
        for (int i = k + 1 + ty; i < n; i += ny) {
            const double l = A[(size_t)i * n + k];
            for (int j = tx; j <= k; j += 32) X[(size_t)i * n + j] -= l * X[(size_t)k * n + j];
        }
        __syncthreads();
    }
    // backward (U): for k descending, X[k][:] /= U[k][k], then X[i][j] -= U[i][k] X[k][j] for i < k
    for (int k = n - 1; k >= 0; --k) {
        const double ukk = A[(size_t)k * n + k];
        for (int j = threadIdx.x; j < n; j += nt) X[(size_t)k * n + j] /= ukk;
        __syncthreads();
        for (int i = ty; i < k; i += ny) {
            const double u = A[(size_t)i * n + k];
            for (int j = tx; j < n; j += 32) X[(size_t)i * n + j] -= u * X[(size_t)k * n + j];
        }
        __syncthreads();
    }
    if (inShared) {
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) inv[c.invOffset + q] = X[q];
    }
}

// x_c = inv * r_c (one CTA per system)
template <class T>
__global__ void k_coarse_apply(const CoarseDev* __restrict__ cs, const double* __restrict__ inv, const T* __restrict__ r,
                               T* __restrict__ x, const SysState* st, int flag) {
    pdl_entry();
    const CoarseDev c = cs[blockIdx.x];
    if (st != nullptr && sys_idle(st[c.sys], flag)) return;
    const double* X = inv + c.invOffset;
    for (int i = threadIdx.x; i < c.n; i += blockDim.x) {
        double g = 0.0;
        for (int j = 0; j < c.n; ++j) g += X[(size_t)i * c.n + j] * (double)r[c.rowStart + j];
        x[c.rowStart + i] = (T)g;
    }
}

// ------------------------------------------------------------------ coarse tail of the V-cycle
// Levels first..coarsest of one system (GAMG.cpp:403-443 with Jacobi smoothing) in ONE CTA: the
// levels at the bottom of the hierarchy are a few thousand rows or fewer, too small to fill the
// GPU, and as separate launches their cost is launch latency.  One CTA per system runs them with
// __syncthreads() in place of the kernel boundaries; the matrix stays in the SM's L1 across the
// phases and the vectors are coherent inside the CTA.  Every row is computed with the same
// operations in the same order as k_smooth_jacobi / k_residual / k_restrict / k_coarse_apply, so
// the result is bit-identical to the per-level launch sequence.
constexpr int kTailThreads = 1024;
constexpr int kTailBatch = 4;      // entries in flight per row (64 registers at 1024 threads)
constexpr int kTailMaxRows = 1024;  // levels at most this many rows (padded) go to the tail
constexpr int kTailFullRows = 2048;  // systems at most this many level-0 rows run the whole V-cycle there

// CL: CTAs of the thread-block cluster that runs one system's tail (CL == 1: one CTA).  With CL > 1
// the rows of each step are spread over the cluster's threads and the steps are separated by the
// cluster's hardware barrier (barrier.cluster arrive.release / wait.acquire); vectors that other CTAs
// of the cluster write are read through L2, and the restriction's residuals go through the level's
// x2 scratch vector (free while the V-cycle descends) instead of shared memory.
template <int CL>
__device__ __forceinline__ void tail_sync() {
    if (CL == 1) {
        __syncthreads();
    } else {
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
}

template <class T, int CL>
__device__ __forceinline__ T tail_ld(const T* p) {
    if (CL == 1) return *p;
    return __ldcg(p);
}

template <class T, int CL = 1>
__global__ void __launch_bounds__(kTailThreads, 1) k_vcycle_tail(const TailSys* __restrict__ tsys,
                                                                 const TailLevel<T>* __restrict__ lev,
                                                                 const double* __restrict__ inv, const T* r0, T* x0,
                                                                 T omega, const SysState* st, int flag, int jacobi0) {
    pdl_entry();
    __shared__ T resS[CL == 1 ? kTailFullRows : 1];  // one level's residuals (restriction), one CTA
    const TailSys& ts = tsys[blockIdx.x / CL];
    if (st != nullptr && sys_idle(st[ts.sys], flag)) return;  // uniform over the CTA / cluster
    const int tid = int(blockIdx.x % CL) * int(blockDim.x) + int(threadIdx.x), nthr = CL * int(blockDim.x);
    const int c = ts.coarsest;
    auto rOf = [&](int k) -> const T* { return k == 0 ? r0 : lev[k].r; };
    auto xOf = [&](int k) -> T* { return k == 0 ? x0 : lev[k].x; };

    // level 0 with global multicolour Gauss-Seidel (k_smooth_gs colour steps, k_zero_rows, k_prolong)
    auto gsRows = [&](const TailLevel<T>& L, const T* r, T* x, int g0, int g1, int mode, const T* xc) {
        for (int i = g0 + tid; i < g1; i += nthr) {
            if (mode == 1) {
                x[i] = tail_ld<T, CL>(r + i) / __ldg(L.diag + i);
                continue;
            }
            auto xf = [&](int j) -> T {
                T v = tail_ld<T, CL>(x + j);
                if (mode == 2) {
                    const int a = __ldg(L.agg + j);
                    if (a >= 0) v += tail_ld<T, CL>(xc + a);
                }
                return v;
            };
            const T s = row_accumulate<true, T, decltype(xf), kTailBatch>(L.S, L.val, xf, i, tail_ld<T, CL>(r + i));
            x[i] = s / __ldg(L.diag + i);
        }
    };
    for (int k = ts.first; k < c; ++k) {
        const TailLevel<T>& L = lev[k];
        const T* r = rOf(k);
        T* x = xOf(k);
        const int a0 = ts.rowStart[k], a1 = a0 + ts.rowCount[k];
        if (k == 0 && !jacobi0) {
            const int nc = ts.nColours;
            if (!ts.two) {
                for (int i = a0 + tid; i < a1; i += nthr) x[i] = T(0);
                tail_sync<CL>();
            }
            for (int sweep = 0; sweep < 2; ++sweep)
                for (int t = 0; t < nc; ++t) {
                    gsRows(L, r, x, ts.grpStart[t], ts.grpStart[t] + ts.grpCount[t],
                           (ts.two && sweep == 0 && t == 0) ? 1 : 0, nullptr);
                    tail_sync<CL>();
                }
        } else {
        // two pre-sweeps from zero; the first sweep's value of a neighbour is recomputed where
        // the second sweep needs it (MODE 1 then MODE 0 of k_smooth_jacobi)
        auto first = [&](int j) -> T {
            const T v = tail_ld<T, CL>(r + j) / __ldg(L.diag + j);
            return omega == T(1) ? v : omega * v;
        };
        for (int i = a0 + tid; i < a1; i += nthr) {
            const T s = row_accumulate<true, T, decltype(first), kTailBatch>(L.S, L.val, first, i, tail_ld<T, CL>(r + i));
            const T v = s / __ldg(L.diag + i);
            if (omega == T(1)) {
                x[i] = v;
            } else {
                const T xv = first(i);
                x[i] = xv + omega * (v - xv);
            }
        }
        tail_sync<CL>();
        }
        // k_residual + k_restrict: every row's residual (one row per thread, into shared memory where
        // the level fits), then each aggregate sums its children's residuals in child order
        T* rn = lev[k + 1].r;
        auto xr = [&](int j) -> T { return tail_ld<T, CL>(x + j); };
        const int b0 = ts.rowStart[k + 1], b1 = b0 + ts.rowCount[k + 1];
        if (CL > 1) {
            T* res = L.x2;  // free while descending
            for (int i = a0 + tid; i < a1; i += nthr)
                res[i] = row_accumulate<true, T, decltype(xr), kTailBatch>(L.S, L.val, xr, i,
                                                                           tail_ld<T, CL>(r + i) - __ldg(L.diag + i) * tail_ld<T, CL>(x + i));
            tail_sync<CL>();
            for (int R = b0 + tid; R < b1; R += nthr) {
                T s = T(0);
                const int q1 = __ldg(L.cptr + R + 1);
                for (int q = __ldg(L.cptr + R); q < q1; ++q) s += __ldcg(res + __ldg(L.child + q));
                rn[R] = s;
            }
        } else if (a1 - a0 <= kTailFullRows) {
            for (int i = a0 + tid; i < a1; i += nthr)
                resS[i - a0] = row_accumulate<true, T, decltype(xr), kTailBatch>(L.S, L.val, xr, i,
                                                                                 r[i] - __ldg(L.diag + i) * x[i]);
            tail_sync<CL>();
            for (int R = b0 + tid; R < b1; R += nthr) {
                T s = T(0);
                const int q1 = __ldg(L.cptr + R + 1);
                for (int q = __ldg(L.cptr + R); q < q1; ++q) s += resS[__ldg(L.child + q) - a0];
                rn[R] = s;
            }
        } else {
            for (int R = b0 + tid; R < b1; R += nthr) {
                T s = T(0);
                const int q1 = __ldg(L.cptr + R + 1);
                for (int q = __ldg(L.cptr + R); q < q1; ++q) {
                    const int i = __ldg(L.child + q);
                    const T t = row_accumulate<true, T, decltype(xr), kTailBatch>(L.S, L.val, xr, i,
                                                                                   r[i] - __ldg(L.diag + i) * x[i]);
                    s += t;
                }
                rn[R] = s;
            }
        }
        tail_sync<CL>();
    }
    {
        // coarsest level: x = inv * r (k_coarse_apply)
        const T* r = rOf(c);
        T* x = xOf(c);
        const int n = ts.coarseN, rs = ts.rowStart[c];
        const double* X = inv + ts.invOffset;
        for (int i = tid; i < n; i += nthr) {
            double g = 0.0;
            for (int j = 0; j < n; ++j) g += __ldg(X + (size_t)i * n + j) * (double)tail_ld<T, CL>(r + rs + j);
            x[rs + i] = (T)g;
        }
    }
    for (int k = c - 1; k >= ts.first; --k) {
        tail_sync<CL>();
        const TailLevel<T>& L = lev[k];
        const T* r = rOf(k);
        T* x = xOf(k);
        const T* xc = xOf(k + 1);
        T* x2 = L.x2;
        const int a0 = ts.rowStart[k], a1 = a0 + ts.rowCount[k];
        if (k == 0 && !jacobi0) {
            // post-smoothing: colours reversed; two colours fuse the prolongation into the first step
            const int nc = ts.nColours;
            if (!ts.two) {
                for (int i = a0 + tid; i < a1; i += nthr) {
                    const int a = __ldg(L.agg + i);
                    if (a >= 0) x[i] += tail_ld<T, CL>(xc + a);
                }
                tail_sync<CL>();
            }
            for (int sweep = 0; sweep < 2; ++sweep)
                for (int t = 0; t < nc; ++t) {
                    const int q = nc - 1 - t;
                    gsRows(L, r, x, ts.grpStart[q], ts.grpStart[q] + ts.grpCount[q],
                           (ts.two && sweep == 0 && t == 0) ? 2 : 0, xc);
                    if (sweep + 1 < 2 || t + 1 < nc) tail_sync<CL>();
                }
            continue;
        }
        // the coarse-grid correction x += xc[agg] as its own phase, then post-sweep 1 into x2 (the same
        // values as adding xc[agg[j]] to every neighbour read, without the two dependent loads per entry)
        for (int i = a0 + tid; i < a1; i += nthr) {
            const int a = __ldg(L.agg + i);
            if (a >= 0) x[i] += tail_ld<T, CL>(xc + a);
        }
        tail_sync<CL>();
        auto xv = [&](int j) -> T { return tail_ld<T, CL>(x + j); };
        for (int i = a0 + tid; i < a1; i += nthr) {
            const T s = row_accumulate<true, T, decltype(xv), kTailBatch>(L.S, L.val, xv, i, tail_ld<T, CL>(r + i));
            const T v = s / __ldg(L.diag + i);
            if (omega == T(1)) {
                x2[i] = v;
            } else {
                const T x0v = xv(i);
                x2[i] = x0v + omega * (v - x0v);
            }
        }
        tail_sync<CL>();
        // post-sweep 2 (MODE 0), back into x
        for (int i = a0 + tid; i < a1; i += nthr) {
            auto x2f = [&](int j) -> T { return tail_ld<T, CL>(x2 + j); };
            const T s = row_accumulate<true, T, decltype(x2f), kTailBatch>(L.S, L.val, x2f, i, tail_ld<T, CL>(r + i));
            const T v = s / __ldg(L.diag + i);
            if (omega == T(1)) {
                x[i] = v;
            } else {
                const T x0v = tail_ld<T, CL>(x2 + i);
                x[i] = x0v + omega * (v - x0v);
            }
        }
    }
}

// ------------------------------------------------------------------ shared-memory coarse tail
// The value image of the shared-memory tail, gathered once per solve: code < 0 -> 0, else level
// code >> 26, diagonal when bit 25 is set, index code & 0x1ffffff into that level's values.
template <class T>
__global__ void k_tail_values(int count, const int32_t* __restrict__ codes, const TailLevel<T>* __restrict__ lev,
                              T* __restrict__ img) {
    pdl_entry();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= count) return;
    const int c = codes[v];
    T a = T(0);
    if (c >= 0) {
        const TailLevel<T>& L = lev[c >> 26];
        const int i = c & 0x1ffffff;
        a = (c >> 25) & 1 ? L.diag[i] : L.val[i];
    }
    img[v] = a;
}

// The coarse tail of k_vcycle_tail (levels first..coarsest of one system, one CTA) with every
// operand in shared memory: the images are copied in while the predecessor drains, then each step
// (Jacobi sweep, residual, restriction, coarse solve, prolongation) reads shared memory only and ends
// at a CTA barrier.  The row arithmetic is k_vcycle_tail's, term for term, so the results are the
// same bit for bit; the first-sweep values are stored instead of recomputed.
template <class T>
__global__ void __launch_bounds__(kTailThreads, 1) k_vcycle_tail_smem(const TailImg* __restrict__ imgs,
                                                                      const T* __restrict__ vimg,
                                                                      const uint16_t* __restrict__ simg,
                                                                      const TailLevel<T>* __restrict__ lev,
                                                                      const double* __restrict__ inv, T omega,
                                                                      const SysState* st, int flag) {
    pdl_launch();
    extern __shared__ __align__(16) unsigned char smraw[];
    __shared__ __align__(16) TailImg I;  // the descriptor, read at every step
    {
        static_assert(sizeof(TailImg) % 4 == 0, "TailImg is copied as words");
        const int* src = reinterpret_cast<const int*>(imgs + blockIdx.x);
        int* dst = reinterpret_cast<int*>(&I);
        for (int i = threadIdx.x; i < int(sizeof(TailImg) / 4); i += blockDim.x) dst[i] = __ldg(src + i);
    }
    __syncthreads();
    const int nc = I.nc;
    T* t = reinterpret_cast<T*>(smraw);
    double* sinv = reinterpret_cast<double*>(smraw + tail_align16(size_t(I.tCount) * sizeof(T)));
    uint16_t* u = reinterpret_cast<uint16_t*>(reinterpret_cast<unsigned char*>(sinv) +
                                              tail_align16(size_t(nc) * nc * sizeof(double)));
    // images (fixed for the solve) while the predecessor drains: 16-byte copies (both images are
    // padded to whole 16-byte words), the inverse by doubles
    {
        const int4* vs = reinterpret_cast<const int4*>(vimg + I.valOff);
        int4* vd = reinterpret_cast<int4*>(t);
        const int nv = int(size_t(I.valCount) * sizeof(T) / 16);
        for (int i = threadIdx.x; i < nv; i += blockDim.x) vd[i] = __ldg(vs + i);
        const int4* ss = reinterpret_cast<const int4*>(simg + I.strOff);
        int4* sd = reinterpret_cast<int4*>(u);
        const int ns = int(size_t(I.strCount) * sizeof(uint16_t) / 16);
        for (int i = threadIdx.x; i < ns; i += blockDim.x) sd[i] = __ldg(ss + i);
        const double* X = inv + I.invOffset;
        for (int i = threadIdx.x; i < nc * nc; i += blockDim.x) sinv[i] = __ldg(X + i);
    }
    pdl_wait();
    if (st != nullptr && sys_idle(st[I.sys], flag)) return;  // uniform over the CTA
    const int f = I.first, c = I.coarsest;
    {
        const T* rg = lev[f].r + I.rowStart[f];
        T* r = t + I.tR[f];
        for (int i = threadIdx.x; i < I.n[f]; i += blockDim.x) r[i] = __ldcg(rg + i);
    }
    __syncthreads();
    // s -= a_ij v_j over row i's entries in order (ELL, column-major, local columns)
    auto rowMinus = [](const T* A, const uint16_t* col, int len, int n, int i, const T* v, T s) -> T {
        for (int q = 0; q < len; ++q) s -= A[q * n + i] * v[col[q * n + i]];
        return s;
    };
    for (int k = f; k < c; ++k) {
        const int n = I.n[k];
        const T* A = t + I.tVal[k];
        const uint16_t* col = u + I.uCol[k];
        const uint16_t* rl = u + I.uRlen[k];
        const T* D = t + I.tDiag[k];
        const T* r = t + I.tR[k];
        T* x = t + I.tX[k];
        T* x2 = t + I.tX2[k];
        // two pre-sweeps from zero (k_smooth_jacobi MODE 1, then MODE 0)
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const T v = r[i] / D[i];
            x2[i] = omega == T(1) ? v : omega * v;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const T v = rowMinus(A, col, rl[i], n, i, x2, r[i]) / D[i];
            x[i] = omega == T(1) ? v : x2[i] + omega * (v - x2[i]);
        }
        __syncthreads();
        // residual (k_residual) into x2, then the restriction (k_restrict) into the next level's r
        for (int i = threadIdx.x; i < n; i += blockDim.x) x2[i] = rowMinus(A, col, rl[i], n, i, x, r[i] - D[i] * x[i]);
        __syncthreads();
        const uint16_t* cp = u + I.uCptr[k];
        const uint16_t* ch = u + I.uChild[k];
        T* rn = t + I.tR[k + 1];
        for (int R = threadIdx.x; R < I.n[k + 1]; R += blockDim.x) {
            T s = T(0);
            for (int q = cp[R]; q < cp[R + 1]; ++q) s += x2[ch[q]];
            rn[R] = s;
        }
        __syncthreads();
    }
    {
        // coarsest level: x = inv * r (k_coarse_apply)
        const T* r = t + I.tR[c];
        T* x = t + I.tX[c];
        for (int i = threadIdx.x; i < nc; i += blockDim.x) {
            double g = 0.0;
            for (int j = 0; j < nc; ++j) g += sinv[i * nc + j] * (double)r[j];
            x[i] = (T)g;
        }
        for (int i = nc + threadIdx.x; i < I.n[c]; i += blockDim.x) x[i] = T(0);
    }
    for (int k = c - 1; k >= f; --k) {
        __syncthreads();
        const int n = I.n[k];
        const T* D = t + I.tDiag[k];
        const T* A = t + I.tVal[k];
        const uint16_t* col = u + I.uCol[k];
        const uint16_t* rl = u + I.uRlen[k];
        const T* r = t + I.tR[k];
        T* x = t + I.tX[k];
        T* x2 = t + I.tX2[k];
        const uint16_t* agg = u + I.uAgg[k];
        const T* xc = t + I.tX[k + 1];
        // the coarse-grid correction, then the two post-sweeps (x -> x2 -> x)
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const int a = agg[i];
            if (a != 0xffff) x[i] += xc[a];
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const T v = rowMinus(A, col, rl[i], n, i, x, r[i]) / D[i];
            x2[i] = omega == T(1) ? v : x[i] + omega * (v - x[i]);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const T v = rowMinus(A, col, rl[i], n, i, x2, r[i]) / D[i];
            x[i] = omega == T(1) ? v : x2[i] + omega * (v - x2[i]);
        }
    }
    __syncthreads();
    {
        T* xg = lev[f].x + I.rowStart[f];
        const T* x = t + I.tX[f];
        for (int i = threadIdx.x; i < I.n[f]; i += blockDim.x) xg[i] = x[i];
    }
}

// ------------------------------------------------------------------ per-solve setup
// Level-0 diagonal in solver order (padding rows get 1 so smoothers leave them at 0).
template <class T>
__global__ void k_gather_diag0(int n, const int32_t* __restrict__ perm, const double* __restrict__ d, T* __restrict__ out) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    out[i] = p >= 0 ? (T)d[p] : T(1);
}

// Entry values from LDU face coefficients: src >= 0 -> upper[src], else lower[~src].
__global__ void k_materialize(int nent, const int32_t* __restrict__ src, const double* __restrict__ upper,
                              const double* __restrict__ lower, double* __restrict__ val, float* __restrict__ val32) {
    pdl_entry();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nent) return;
    const int s = src[e];
    const double v = s >= 0 ? upper[s] : lower[~s];
    val[e] = v;
    if (val32) val32[e] = (float)v;
}

// Galerkin coarse diagonal (GAMG.cpp:285-292): children's diagonals in ascending order,
// then upper+lower of the faces inside the aggregate in face order.
__global__ void k_galerkin_diag(int nrows, const int32_t* __restrict__ cptr, const int32_t* __restrict__ child,
                                const int32_t* __restrict__ iptr, const int32_t* __restrict__ iface,
                                const double* __restrict__ dfine, const double* __restrict__ up,
                                const double* __restrict__ lo, double* __restrict__ dc, float* __restrict__ dc32) {
    pdl_entry();
    const int R = blockIdx.x * blockDim.x + threadIdx.x;
    if (R >= nrows) return;
    double s;
    if (cptr[R] == cptr[R + 1]) {
        s = 1.0;  // padding row
    } else {
        s = 0.0;
        for (int k = cptr[R]; k < cptr[R + 1]; ++k) s += dfine[child[k]];
        for (int k = iptr[R]; k < iptr[R + 1]; ++k) {
            const int f = iface[k];
            s += up[f] + lo[f];
        }
    }
    dc[R] = s;
    if (dc32) dc32[R] = (float)s;
}

// Galerkin coarse faces (GAMG.cpp:289-300): flip-aware sums in fine-face order.
__global__ void k_galerkin_faces(int nfaces, const int32_t* __restrict__ fptr, const int32_t* __restrict__ fsrc,
                                 const double* __restrict__ up, const double* __restrict__ lo, double* __restrict__ cu,
                                 double* __restrict__ cl) {
    pdl_entry();
    const int F = blockIdx.x * blockDim.x + threadIdx.x;
    if (F >= nfaces) return;
    double su = 0.0, sl = 0.0;
    for (int k = fptr[F]; k < fptr[F + 1]; ++k) {
        const uint32_t e = (uint32_t)fsrc[k];
        const int f = (int)(e & 0x7fffffffu);
        if (e & 0x80000000u) {
            su += lo[f];
            sl += up[f];
        } else {
            su += up[f];
            sl += lo[f];
        }
    }
    cu[F] = su;
    cl[F] = sl;
}

// Permute a user vector into solver order (padding -> 0) and back.
template <class T>
__global__ void k_to_solver(int n, const int32_t* __restrict__ perm, const double* __restrict__ u, T* __restrict__ v) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    v[i] = p >= 0 ? (T)u[p] : T(0);
}

__global__ void k_from_solver(int n, const int32_t* __restrict__ perm, const double* __restrict__ v, double* __restrict__ u) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    if (p >= 0) u[p] = v[i];
}

__global__ void k_cast_f64_to_f32(int n, const double* __restrict__ a, float* __restrict__ b) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

}  // namespace vlm
