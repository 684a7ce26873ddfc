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
template <int NV>
__device__ __forceinline__ void block_reduce(DD (&v)[NV]) {
    __shared__ DD sm[NV][kRowsPerCta / 32];
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


// Writes this CTA's partials; returns true in thread 0 of the CTA that completes the
// system, with the system totals (summed over slots in a fixed order) in `out`.
template <int NV>
__device__ bool reduce_dd(DD (&v)[NV], const Chunk& c, const RedCtx& R, double (&out)[NV]) {
    block_reduce<NV>(v);
    __shared__ int isLast;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) R.partials[(size_t)c.slot * NV + q] = v[q];
        __threadfence();
        const int nslots = R.slotEnd[c.sys] - R.slotBegin[c.sys];
        const int ticket = atomicAdd(&R.counters[c.sys], 1);
        isLast = ticket == nslots - 1;
    }
    __syncthreads();
    if (!isLast) return false;
    __threadfence();
    const int b = R.slotBegin[c.sys], e = R.slotEnd[c.sys];
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
    block_reduce<NV>(acc);
    if (threadIdx.x != 0) return false;
    R.counters[c.sys] = 0;
#pragma unroll
    for (int q = 0; q < NV; ++q) out[q] = acc[q].hi + acc[q].lo;
    return true;
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
    const Chunk c = ch[blockIdx.x];
    DD a[1] = {DD{0.0, 0.0}};
    if ((int)threadIdx.x < c.count) a[0].hi = v[c.start + threadIdx.x];
    double o[1];
    if (reduce_exact<1>(a, c, R, o)) *out = o[0];
}

// ------------------------------------------------------------------ SELL row access

__device__ __forceinline__ int sell_base(const Sell& S, int row) { return S.slPtr[row >> 5] + (row & 31); }

template <class T>
__device__ __forceinline__ T row_minus(const Sell& S, const T* __restrict__ val, const T* __restrict__ x, int row, T s) {
    const int len = S.rlen[row];
    const int base = sell_base(S, row);
    for (int k = 0; k < len; ++k) {
        const int e = base + (k << 5);
        s -= val[e] * x[S.col[e]];
    }
    return s;
}

template <class T>
__device__ __forceinline__ T row_plus(const Sell& S, const T* __restrict__ val, const T* __restrict__ x, int row, T s) {
    const int len = S.rlen[row];
    const int base = sell_base(S, row);
    for (int k = 0; k < len; ++k) {
        const int e = base + (k << 5);
        s += val[e] * x[S.col[e]];
    }
    return s;
}

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
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag)) return;
    for (int row = c.start + threadIdx.x; row < c.start + c.count; row += kRowsPerCta) x[row] = T(0);
}

// w = r on the rows of the chunks (the "none" preconditioner)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_copy_rows(const Chunk* __restrict__ ch, const T* __restrict__ r,
                                                           T* __restrict__ w, const SysState* st, int flag) {
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag)) return;
    for (int row = c.start + threadIdx.x; row < c.start + c.count; row += kRowsPerCta) w[row] = r[row];
}

// b = (To) a on the rows of the chunks
template <class From, class To>
__global__ void __launch_bounds__(kRowsPerCta) k_cast_rows(const Chunk* __restrict__ ch, const From* __restrict__ a,
                                                           To* __restrict__ b, const SysState* st, int flag) {
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag)) return;
    for (int row = c.start + threadIdx.x; row < c.start + c.count; row += kRowsPerCta) b[row] = (To)a[row];
}

// ------------------------------------------------------------------ smoothers
// Gauss-Seidel row update (GAMG.cpp:368-380) on the rows of one colour step.
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_smooth_gs(const Chunk* __restrict__ ch, Sell S, const T* __restrict__ val,
                                                           const T* __restrict__ diag, const T* __restrict__ r, T* x,
                                                           const SysState* st, int flag) {
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag) || (int)threadIdx.x >= c.count) return;
    const int row = c.start + threadIdx.x;
    const T s = row_minus(S, val, x, row, r[row]);
    x[row] = s / diag[row];
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
// MODE 2: xi + xc[agg] (the coarse-grid correction, GAMG.cpp:437-438, fused in).
template <class T, int MODE>
__global__ void __launch_bounds__(kRowsPerCta) k_smooth_jacobi(const Chunk* __restrict__ ch, Sell S,
                                                               const T* __restrict__ val, const T* __restrict__ diag,
                                                               const T* __restrict__ r, const T* __restrict__ xi,
                                                               T* __restrict__ xo, T omega,
                                                               const int32_t* __restrict__ agg,
                                                               const T* __restrict__ xc, const SysState* st, int flag) {
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag) || (int)threadIdx.x >= c.count) return;
    const int row = c.start + threadIdx.x;
    if (MODE == 1) {
        const T v = r[row] / diag[row];
        xo[row] = omega == T(1) ? v : omega * v;
        return;
    }
    auto xv = [&](int j) -> T {
        T v = xi[j];
        if (MODE == 2) {
            const int a = agg[j];
            if (a >= 0) v += xc[a];
        }
        return v;
    };
    T s = r[row];
    const int len = S.rlen[row], base = sell_base(S, row);
    for (int k = 0; k < len; ++k) {
        const int e = base + (k << 5);
        s -= val[e] * xv(S.col[e]);
    }
    const T v = s / diag[row];
    if (omega == T(1)) {
        xo[row] = v;
    } else {
        const T x0 = xv(row);
        xo[row] = x0 + omega * (v - x0);
    }
}

// res = r - A x  (GAMG.cpp:387-401: diagonal first, then the faces in order)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_residual(const Chunk* __restrict__ ch, Sell S, const T* __restrict__ val,
                                                          const T* __restrict__ diag, const T* __restrict__ r,
                                                          const T* __restrict__ x, T* __restrict__ res,
                                                          const SysState* st, int flag) {
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag) || (int)threadIdx.x >= c.count) return;
    const int row = c.start + threadIdx.x;
    const T s = row_minus(S, val, x, row, r[row] - diag[row] * x[row]);
    res[row] = s;
}

// rc[R] = sum of res over the children of R in ascending natural order (GAMG.cpp:434-435)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_restrict(const Chunk* __restrict__ ch, const int32_t* __restrict__ cptr,
                                                          const int32_t* __restrict__ child, const T* __restrict__ res,
                                                          T* __restrict__ rc, const SysState* st, int flag) {
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag) || (int)threadIdx.x >= c.count) return;
    const int R = c.start + threadIdx.x;
    T s = T(0);
    for (int k = cptr[R]; k < cptr[R + 1]; ++k) s += res[child[k]];
    rc[R] = s;
}

// x += xc[agg]  (GAMG.cpp:437-438)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_prolong(const Chunk* __restrict__ ch, const int32_t* __restrict__ agg,
                                                         const T* __restrict__ xc, T* __restrict__ x, const SysState* st, int flag) {
    const Chunk c = ch[blockIdx.x];
    if (chunk_skip(c, st, flag) || (int)threadIdx.x >= c.count) return;
    const int row = c.start + threadIdx.x;
    const int a = agg[row];
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
    __shared__ int singular;
    if (threadIdx.x == 0) singular = 0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double piv = A[(size_t)k * n + k];
        if (fabs(piv) < kVSMALL) {
            if (threadIdx.x == 0) singular = 1;
            break;
        }
        for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) {
            const double fct = A[(size_t)i * n + k] / piv;
            A[(size_t)i * n + k] = fct;
            if (fct == 0.0) continue;
            for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= fct * A[(size_t)k * n + j];
        }
        __syncthreads();
    }
    __syncthreads();
    if (singular) {
        if (threadIdx.x == 0) atomicExch(status, (int)VLM_ERR_SINGULAR);
        return;
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        // column j of the inverse: solve L U g = e_j
        for (int i = 0; i < n; ++i) {
            double g = i == j ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) g -= A[(size_t)i * n + k] * X[(size_t)k * n + j];
            X[(size_t)i * n + j] = g;
        }
        for (int i = n - 1; i >= 0; --i) {
            double g = X[(size_t)i * n + j];
            for (int k = i + 1; k < n; ++k) g -= A[(size_t)i * n + k] * X[(size_t)k * n + j];
            X[(size_t)i * n + j] = g / A[(size_t)i * n + i];
        }
    }
    if (inShared) {
        __syncthreads();
        for (int q = threadIdx.x; q < n * n; q += blockDim.x) inv[c.invOffset + q] = X[q];
    }
}

// x_c = inv * r_c (one CTA per system)
template <class T>
__global__ void k_coarse_apply(const CoarseDev* __restrict__ cs, const double* __restrict__ inv, const T* __restrict__ r,
                               T* __restrict__ x, const SysState* st, int flag) {
    const CoarseDev c = cs[blockIdx.x];
    if (st != nullptr && sys_idle(st[c.sys], flag)) return;
    const double* X = inv + c.invOffset;
    for (int i = threadIdx.x; i < c.n; i += blockDim.x) {
        double g = 0.0;
        for (int j = 0; j < c.n; ++j) g += X[(size_t)i * c.n + j] * (double)r[c.rowStart + j];
        x[c.rowStart + i] = (T)g;
    }
}

// ------------------------------------------------------------------ per-solve setup
// Level-0 diagonal in solver order (padding rows get 1 so smoothers leave them at 0).
template <class T>
__global__ void k_gather_diag0(int n, const int32_t* __restrict__ perm, const double* __restrict__ d, T* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    out[i] = p >= 0 ? (T)d[p] : T(1);
}

// Entry values from LDU face coefficients: src >= 0 -> upper[src], else lower[~src].
__global__ void k_materialize(int nent, const int32_t* __restrict__ src, const double* __restrict__ upper,
                              const double* __restrict__ lower, double* __restrict__ val, float* __restrict__ val32) {
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
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    v[i] = p >= 0 ? (T)u[p] : T(0);
}

__global__ void k_from_solver(int n, const int32_t* __restrict__ perm, const double* __restrict__ v, double* __restrict__ u) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int p = perm[i];
    if (p >= 0) u[p] = v[i];
}

__global__ void k_cast_f64_to_f32(int n, const double* __restrict__ a, float* __restrict__ b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

}  // namespace vlm
