// Level-scheduled kernels: DIC/DILU factorisation and application (LinearSolver.cpp:56-112), and
// the Gauss-Seidel / symmetric Gauss-Seidel / Jacobi solvers (LinearSolver.cpp:238-278).
//
// One group of G CTAs works on one system and walks its levels (dilu.h) in order; rows of one
// level are independent, so they are spread over the group's threads, and the group synchronises
// between levels.  With G == 1 that is __syncthreads(); with G > 1 (one large system, launched
// cooperatively so the group is co-resident) it is a counter barrier in global memory whose wait
// gives up after a bounded number of polls, sets VLM_ERR_TIMEOUT in *err and lets the kernel run
// to its end.  Values written by other CTAs of the group are read through L2 (ld.global.cg).
#pragma once

#include "krylov.cuh"
#include "dilu.h"

namespace vlm {

constexpr int kDiluThreads = 512;
constexpr long long kDiluSpinLimit = 1ll << 22;  // polls of >= 64 ns: a wait gives up within seconds

struct DiluBar {
    unsigned count, gen;
};

__device__ __forceinline__ void group_sync(DiluBar* bar, int G, int* err) {
    __syncthreads();
    if (G > 1) {
        if (threadIdx.x == 0) {
            volatile unsigned* vg = &bar->gen;
            const unsigned g = *vg;
            __threadfence();
            if (atomicAdd(&bar->count, 1u) == unsigned(G - 1)) {
                atomicExch(&bar->count, 0u);
                __threadfence();
                atomicAdd(&bar->gen, 1u);
            } else {
                // once any wait of this launch has given up, later waits return at once
                long long it = 0;
                while (*vg == g) {
                    if (*(volatile int*)err != 0) break;
                    if (++it > kDiluSpinLimit) {
                        atomicExch(err, int(VLM_ERR_TIMEOUT));
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __threadfence();
        }
        __syncthreads();
    }
}

#define VLM_LEVEL_ROWS(d, t, idx)                                                          \
    for (int idx = levPtr[(d).levBegin + (t)] + tid; idx < levPtr[(d).levBegin + (t) + 1]; \
         idx += nthr)

// Per-solve coefficients in schedule order: A_ul and A_lu of every lower entry, A_lu of every
// upper entry (LinearSolver.cpp:70-72, 99, 104).
__global__ void k_dilu_values(int n, const int32_t* __restrict__ loFace, const int32_t* __restrict__ upFace,
                              const double* __restrict__ upper, const double* __restrict__ lower,
                              double* __restrict__ loAul, double* __restrict__ loAlu, double* __restrict__ upAlu) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int32_t a = loFace[k], b = upFace[k];
    const int fa = a & 0x7fffffff, fb = b & 0x7fffffff;
    const bool la = a < 0, lb = b < 0;  // ownerIsL
    loAul[k] = la ? lower[fa] : upper[fa];
    loAlu[k] = la ? upper[fa] : lower[fa];
    upAlu[k] = lb ? upper[fb] : lower[fb];
}

// rD[u] = D[u] - sum_l A_lu A_ul / rD[l] in level order, then rD = 1 / rD (LinearSolver.cpp:66-77)
__global__ void __launch_bounds__(kDiluThreads) k_dilu_factor(const DiluSys* __restrict__ ds, int G,
                                                              const int32_t* __restrict__ levPtr,
                                                              const int32_t* __restrict__ levRows,
                                                              const int32_t* __restrict__ loPtr,
                                                              const int32_t* __restrict__ loCol,
                                                              const double* __restrict__ loAlu,
                                                              const double* __restrict__ loAul,
                                                              const double* __restrict__ diag, double* rD,
                                                              DiluBar* bars, int* err) {
    const DiluSys d = ds[blockIdx.x / G];
    const int tid = int(blockIdx.x % G) * blockDim.x + threadIdx.x, nthr = G * blockDim.x;
    DiluBar* bar = bars + blockIdx.x / G;
    for (int t = 0; t < d.nLev; ++t) {
        VLM_LEVEL_ROWS(d, t, idx) {
            const int c = levRows[idx];
            double v = diag[c];
            for (int k = loPtr[c]; k < loPtr[c + 1]; ++k) v -= loAlu[k] * loAul[k] / __ldcg(rD + loCol[k]);
            rD[c] = v;
        }
        group_sync(bar, G, err);
    }
    for (int t = 0; t < d.nLev; ++t) VLM_LEVEL_ROWS(d, t, idx) {
            const int c = levRows[idx];
            rD[c] = 1.0 / __ldcg(rD + c);
        }
}

// w = M^-1 r: w = rD r; forward w[u] -= rD[u] A_ul w[l]; backward w[l] -= rD[l] A_lu w[u]
// (LinearSolver.cpp:87-106)
__global__ void __launch_bounds__(kDiluThreads) k_dilu_apply(const DiluSys* __restrict__ ds, int G,
                                                             const int32_t* __restrict__ levPtr,
                                                             const int32_t* __restrict__ levRows,
                                                             const int32_t* __restrict__ loPtr,
                                                             const int32_t* __restrict__ loCol,
                                                             const double* __restrict__ loAul,
                                                             const int32_t* __restrict__ upPtr,
                                                             const int32_t* __restrict__ upCol,
                                                             const double* __restrict__ upAlu,
                                                             const double* __restrict__ rD, const double* r, double* w,
                                                             DiluBar* bars, int* err, const SysState* st, int flag) {
    pdl_entry();
    const DiluSys d = ds[blockIdx.x / G];
    if (st != nullptr && sys_idle(st[d.sys], flag)) return;  // uniform over the group
    const int tid = int(blockIdx.x % G) * blockDim.x + threadIdx.x, nthr = G * blockDim.x;
    DiluBar* bar = bars + blockIdx.x / G;
    for (int t = 0; t < d.nLev; ++t) {
        VLM_LEVEL_ROWS(d, t, idx) {
            const int c = levRows[idx];
            const double rd = rD[c];
            double wc = rd * r[c];
            for (int k = loPtr[c]; k < loPtr[c + 1]; ++k) wc -= rd * loAul[k] * __ldcg(w + loCol[k]);
            w[c] = wc;
        }
        group_sync(bar, G, err);
    }
    for (int t = d.nLev - 1; t >= 0; --t) {
        VLM_LEVEL_ROWS(d, t, idx) {
            const int c = levRows[idx];
            const double rd = rD[c];
            double wc = __ldcg(w + c);
            for (int k = upPtr[c]; k < upPtr[c + 1]; ++k) wc -= rd * upAlu[k] * __ldcg(w + upCol[k]);
            w[c] = wc;
        }
        if (t > 0) group_sync(bar, G, err);
    }
}

// ---------------------------------------------------------------- shared-memory variants
// One CTA per system whose level-0 vector fits in shared memory and whose levels are at most one
// row per thread.  The swept vector lives in shared memory, and each thread loads its rows of the
// next three levels (row index, scalars and the first kDiluPre coefficients) ahead of the barriers,
// so a level costs a barrier and shared-memory reads, not an L2 round trip.
// Same arithmetic in the same order as k_dilu_factor / k_dilu_apply.
constexpr int kDiluPre = 4;

struct DiluRow {
    int c, k0, k1;
    double a, b;                      // apply: rD[c], r[c]; factor: diag[c]
    int col[kDiluPre];
    double v0[kDiluPre], v1[kDiluPre];  // apply: A_ul (fwd) / A_lu (bwd); factor: A_lu, A_ul
};

__device__ __forceinline__ void dilu_row_load(const DiluSys& d, int t, int tid, const int32_t* __restrict__ levPtr,
                                              const int32_t* __restrict__ levRows, const int32_t* __restrict__ ptr,
                                              const int32_t* __restrict__ col, const double* __restrict__ c0,
                                              const double* __restrict__ c1, const double* __restrict__ sa,
                                              const double* __restrict__ sb, DiluRow& p) {
    p.c = -1;
    if (t < 0 || t >= d.nLev) return;
    const int idx = levPtr[d.levBegin + t] + tid;
    if (idx >= levPtr[d.levBegin + t + 1]) return;
    p.c = levRows[idx];
    p.a = sa[p.c];
    p.b = sb ? sb[p.c] : 0.0;
    p.k0 = ptr[p.c];
    p.k1 = ptr[p.c + 1];
#pragma unroll
    for (int q = 0; q < kDiluPre; ++q)
        if (p.k0 + q < p.k1) {
            p.col[q] = col[p.k0 + q];
            p.v0[q] = c0[p.k0 + q];
            p.v1[q] = c1 ? c1[p.k0 + q] : 0.0;
        }
}

__global__ void __launch_bounds__(kDiluThreads) k_dilu_factor_smem(const DiluSys* __restrict__ ds,
                                                                   const int32_t* __restrict__ levPtr,
                                                                   const int32_t* __restrict__ levRows,
                                                                   const int32_t* __restrict__ loPtr,
                                                                   const int32_t* __restrict__ loCol,
                                                                   const double* __restrict__ loAlu,
                                                                   const double* __restrict__ loAul,
                                                                   const double* __restrict__ diag,
                                                                   double* __restrict__ rD) {
    extern __shared__ double sh[];
    const DiluSys d = ds[blockIdx.x];
    const int base = d.rowBegin, tid = threadIdx.x;
    DiluRow r0, r1, r2, r3;  // levels t .. t+3 in flight
    dilu_row_load(d, 0, tid, levPtr, levRows, loPtr, loCol, loAlu, loAul, diag, nullptr, r0);
    dilu_row_load(d, 1, tid, levPtr, levRows, loPtr, loCol, loAlu, loAul, diag, nullptr, r1);
    dilu_row_load(d, 2, tid, levPtr, levRows, loPtr, loCol, loAlu, loAul, diag, nullptr, r2);
    for (int t = 0; t < d.nLev; ++t) {
        dilu_row_load(d, t + 3, tid, levPtr, levRows, loPtr, loCol, loAlu, loAul, diag, nullptr, r3);
        if (r0.c >= 0) {
            double v = r0.a;
            const int np = min(r0.k1 - r0.k0, kDiluPre);
            for (int q = 0; q < np; ++q) v -= r0.v0[q] * r0.v1[q] / sh[r0.col[q] - base];
            for (int k = r0.k0 + kDiluPre; k < r0.k1; ++k) v -= loAlu[k] * loAul[k] / sh[loCol[k] - base];
            sh[r0.c - base] = v;
        }
        __syncthreads();
        r0 = r1;
        r1 = r2;
        r2 = r3;
    }
    for (int i = tid; i < d.rowCount; i += blockDim.x) rD[base + i] = 1.0 / sh[i];
}

__global__ void __launch_bounds__(kDiluThreads) k_dilu_apply_smem(const DiluSys* __restrict__ ds,
                                                                  const int32_t* __restrict__ levPtr,
                                                                  const int32_t* __restrict__ levRows,
                                                                  const int32_t* __restrict__ loPtr,
                                                                  const int32_t* __restrict__ loCol,
                                                                  const double* __restrict__ loAul,
                                                                  const int32_t* __restrict__ upPtr,
                                                                  const int32_t* __restrict__ upCol,
                                                                  const double* __restrict__ upAlu,
                                                                  const double* __restrict__ rD, const double* r,
                                                                  double* w, const SysState* st, int flag) {
    pdl_entry();
    extern __shared__ double sh[];
    const DiluSys d = ds[blockIdx.x];
    if (st != nullptr && sys_idle(st[d.sys], flag)) return;
    const int base = d.rowBegin, tid = threadIdx.x;
    DiluRow r0, r1, r2, r3;  // levels t .. t+3 in flight
    dilu_row_load(d, 0, tid, levPtr, levRows, loPtr, loCol, loAul, nullptr, rD, r, r0);
    dilu_row_load(d, 1, tid, levPtr, levRows, loPtr, loCol, loAul, nullptr, rD, r, r1);
    dilu_row_load(d, 2, tid, levPtr, levRows, loPtr, loCol, loAul, nullptr, rD, r, r2);
    for (int t = 0; t < d.nLev; ++t) {
        dilu_row_load(d, t + 3, tid, levPtr, levRows, loPtr, loCol, loAul, nullptr, rD, r, r3);
        if (r0.c >= 0) {
            const double rd = r0.a;
            double wc = rd * r0.b;
            const int np = min(r0.k1 - r0.k0, kDiluPre);
            for (int q = 0; q < np; ++q) wc -= rd * r0.v0[q] * sh[r0.col[q] - base];
            for (int k = r0.k0 + kDiluPre; k < r0.k1; ++k) wc -= rd * loAul[k] * sh[loCol[k] - base];
            sh[r0.c - base] = wc;
        }
        __syncthreads();
        r0 = r1;
        r1 = r2;
        r2 = r3;
    }
    const int L = d.nLev - 1;
    dilu_row_load(d, L, tid, levPtr, levRows, upPtr, upCol, upAlu, nullptr, rD, nullptr, r0);
    dilu_row_load(d, L - 1, tid, levPtr, levRows, upPtr, upCol, upAlu, nullptr, rD, nullptr, r1);
    dilu_row_load(d, L - 2, tid, levPtr, levRows, upPtr, upCol, upAlu, nullptr, rD, nullptr, r2);
    for (int t = L; t >= 0; --t) {
        dilu_row_load(d, t - 3, tid, levPtr, levRows, upPtr, upCol, upAlu, nullptr, rD, nullptr, r3);
        if (r0.c >= 0) {
            const double rd = r0.a;
            double wc = sh[r0.c - base];
            const int np = min(r0.k1 - r0.k0, kDiluPre);
            for (int q = 0; q < np; ++q) wc -= rd * r0.v0[q] * sh[r0.col[q] - base];
            for (int k = r0.k0 + kDiluPre; k < r0.k1; ++k) wc -= rd * upAlu[k] * sh[upCol[k] - base];
            sh[r0.c - base] = wc;
        }
        __syncthreads();
        r0 = r1;
        r1 = r2;
        r2 = r3;
    }
    for (int i = tid; i < d.rowCount; i += blockDim.x) w[base + i] = sh[i];
}

// Gauss-Seidel sweep in natural order (forward) or reversed (backward), in place:
// x[c] = (b[c] - sum over the row's entries in face order of a * x) / D[c], where the lower
// neighbours already hold this sweep's value (LinearSolver.cpp:245-275, sweepCell)
__global__ void __launch_bounds__(kDiluThreads) k_gs_sweep(const DiluSys* __restrict__ ds, int G,
                                                           const int32_t* __restrict__ levPtr,
                                                           const int32_t* __restrict__ levRows, Sell S,
                                                           const double* __restrict__ val,
                                                           const double* __restrict__ diag,
                                                           const double* __restrict__ b, double* x, int backward,
                                                           DiluBar* bars, int* err, const SysState* st, int flag) {
    pdl_entry();
    const DiluSys d = ds[blockIdx.x / G];
    if (st != nullptr && sys_idle(st[d.sys], flag)) return;
    const int tid = int(blockIdx.x % G) * blockDim.x + threadIdx.x, nthr = G * blockDim.x;
    DiluBar* bar = bars + blockIdx.x / G;
    for (int q = 0; q < d.nLev; ++q) {
        const int t = backward ? d.nLev - 1 - q : q;
        VLM_LEVEL_ROWS(d, t, idx) {
            const int c = levRows[idx];
            const double s = row_accumulate<true>(S, val, [&](int j) { return __ldcg(x + j); }, c, b[c]);
            x[c] = s / diag[c];
        }
        if (q + 1 < d.nLev) group_sync(bar, G, err);
    }
}

// r = b - A x (amul order), finalResidual = sum|r| / normFactor, iterations += nSweeps, convergence
// (LinearSolver.cpp:272-277)
template <bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_relax_residual(const Chunk* __restrict__ ch, Sell S,
                                                                const double* __restrict__ val,
                                                                const double* __restrict__ diag,
                                                                const double* __restrict__ x,
                                                                const double* __restrict__ b,
                                                                const int32_t* __restrict__ perm, int nSweeps,
                                                                RedCtx R, SysState* st,
                                                                const DevCtrl* __restrict__ ctrlp) {
    pdl_entry();
    const Chunk c = ch[blockIdx.x];
    if (sys_idle(st[c.sys], kFlagDone)) return;
    BlockSum<1, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) {
        const double wA = row_plus(S, val, x, row, diag[row] * x[row]);
        const double rr = b[row] - wA;
        if (perm[row] >= 0) acc.add(0, fabs(rr));
    }
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        s.iterations += nSweeps;
        s.finalResidual = out[0] / s.normFactor;
        if (!isfinite(s.finalResidual)) {
            s.status = VLM_ERR_NONFINITE;
            s.done = 1;
        } else if (s.iterations >= ctrlp->maxIter ||
                   dev_converged(*ctrlp, s.iterations, s.finalResidual, s.initialResidual)) {
            s.done = 1;
        }
    }
}

}  // namespace vlm
