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

// spinLimit: polls before a wait gives up (kDiluSpinLimit in the solver kernels).
__device__ __forceinline__ void group_sync(DiluBar* bar, int G, int* err, long long spinLimit = kDiluSpinLimit) {
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
                    if (++it > spinLimit) {
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

// Self-test of the group barrier's failure path: G co-resident CTAs (cooperative launch) pass
// `rounds` barriers; CTA `absent` (when 0 <= absent < G) returns before its first arrival, so the
// others' first wait runs out after spinLimit polls, sets VLM_ERR_TIMEOUT in *err, and every later
// wait returns at once: the kernel ends and the status reaches the host.  passed[b]: barriers CTA b
// got through.
__global__ void k_group_barrier_check(DiluBar* bar, int G, int* err, long long spinLimit, int absent, int rounds,
                                      int* passed) {
    if ((int)blockIdx.x == absent) return;
    for (int q = 0; q < rounds; ++q) {
        group_sync(bar, G, err, spinLimit);
        if (threadIdx.x == 0 && *(volatile int*)err == 0) passed[blockIdx.x] = q + 1;
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

// ---------------------------------------------------------------- shared-memory (streamed) variants
// One CTA per system whose level-0 vector fits in shared memory and whose levels are at most one
// row per thread.  The swept vector lives in shared memory.  The schedule is streamed (dilu.h,
// DiluLevel): each level's rows, scalars and entries are contiguous in global memory, and cp.async
// copies them into a ring of kDiluRing shared-memory stages, kDiluRing - 1 levels ahead of the
// sweep, so a level costs one barrier and shared-memory reads instead of a chain of L2 round trips.
//
// The factor's A_lu * A_ul is formed once per factorisation (the product the reference's
// rD[u] -= A_lu A_ul / rD[l] forms first); every other operation is the reference's, in its order,
// so the results are those of k_dilu_factor / k_dilu_apply bit for bit.
constexpr int kDiluRing = 8;

__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(unsigned(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(unsigned(__cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__host__ __device__ constexpr size_t dilu_align16(size_t b) { return (b + 15) / 16 * 16; }

// One ring stage for levels of at most W slots and M entries per slot: a[W] (slot scalar),
// v[M * W] (entry coefficient), row[W], col[M * W].
__host__ __device__ constexpr size_t dilu_stage_bytes(int W, int M) {
    return dilu_align16(size_t(W) * (M + 1) * (sizeof(double) + sizeof(int32_t)));
}

// Shared memory of a streamed kernel: the vector, the level table and the ring.
__host__ __device__ constexpr size_t dilu_stream_smem(int rows, int levels, int W, int M) {
    return dilu_align16(size_t(rows) * sizeof(double)) + dilu_align16(size_t(levels) * sizeof(DiluLevel)) +
           kDiluRing * dilu_stage_bytes(W, M);
}

struct DiluStage {
    double *a, *v;
    int32_t *row, *col;
    __device__ DiluStage(char* base, int W, int M) {
        a = reinterpret_cast<double*>(base);
        v = a + W;
        row = reinterpret_cast<int32_t*>(v + size_t(M) * W);
        col = row + W;
    }
};

// Starts the copies of one level's slots (rows and, if sa, one scalar per slot) and its m entries per
// slot (columns and coefficients) into a stage.
__device__ __forceinline__ void dilu_stage_issue(const DiluStage& S, const DiluLevel& L, int ent, int m,
                                                 const int32_t* __restrict__ slotRow, const double* __restrict__ sa,
                                                 const int32_t* __restrict__ col, const double* __restrict__ v) {
    const int tid = threadIdx.x;
    if (tid < L.width) {
        cp_async4(S.row + tid, slotRow + L.s0 + tid);
        if (sa != nullptr) cp_async8(S.a + tid, sa + L.s0 + tid);
    }
    const int n = m * L.width;
    for (int k = tid; k < n; k += blockDim.x) {
        cp_async4(S.col + k, col + ent + k);
        cp_async8(S.v + k, v + ent + k);
    }
}

// Streamed sweep over levels t = 0 .. nLev-1 (or reversed) of one system: before level t is
// processed, the copies of level t + kDiluRing - 1 are started into the stage level t - 1 used.
// body(stage, level) runs for every slot thread of the level.
template <bool LOWER, bool REVERSE, class Body>
__device__ __forceinline__ void dilu_stream(const DiluLevel* lt, int nLev, char* ring, int W, int M,
                                            const int32_t* __restrict__ slotRow, const double* __restrict__ sa,
                                            const int32_t* __restrict__ col, const double* __restrict__ v,
                                            Body body) {
    const size_t SB = dilu_stage_bytes(W, M);
    auto issue = [&](int q) {
        if (q < nLev) {
            const DiluLevel& L = lt[REVERSE ? nLev - 1 - q : q];
            dilu_stage_issue(DiluStage(ring + size_t(q % kDiluRing) * SB, W, M), L, LOWER ? L.lo : L.up,
                             LOWER ? L.mlo : L.mup, slotRow, sa, col, v);
        }
        cp_async_commit();
    };
    for (int q = 0; q < kDiluRing - 1; ++q) issue(q);
    for (int q = 0; q < nLev; ++q) {
        cp_async_wait<kDiluRing - 2>();
        __syncthreads();  // level q staged by every thread; level q - 1's vector writes visible
        issue(q + kDiluRing - 1);
        const DiluLevel& L = lt[REVERSE ? nLev - 1 - q : q];
        if (threadIdx.x < L.width) body(DiluStage(ring + size_t(q % kDiluRing) * SB, W, M), L);
    }
    cp_async_wait<0>();
    __syncthreads();
}

// Shared memory of a streamed kernel: the vector sh[rowCount] (filled from src by cp.async), the
// level table and the ring.  Both copies are waited for before the function returns.
__device__ __forceinline__ char* dilu_stream_setup(char* smem, const DiluSys& d, const DiluLevel* __restrict__ lev,
                                                   const double* __restrict__ src, double*& sh, DiluLevel*& lt) {
    sh = reinterpret_cast<double*>(smem);
    lt = reinterpret_cast<DiluLevel*>(smem + dilu_align16(size_t(d.rowCount) * sizeof(double)));
    const int32_t* lg = reinterpret_cast<const int32_t*>(lev + d.levBegin);
    int32_t* ls = reinterpret_cast<int32_t*>(lt);
    const int nw = d.nLev * int(sizeof(DiluLevel) / sizeof(int32_t));
    for (int i = threadIdx.x; i < nw; i += blockDim.x) cp_async4(ls + i, lg + i);
    for (int i = threadIdx.x; i < d.rowCount; i += blockDim.x) cp_async8(sh + i, src + d.rowBegin + i);
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    return reinterpret_cast<char*>(lt) + dilu_align16(size_t(d.nLev) * sizeof(DiluLevel));
}

// Per-solve coefficients of the streamed schedule: prod = A_lu A_ul and coefLo = A_ul per lower
// entry, coefUp = A_lu per upper entry.
__global__ void k_dilu_stream_values(int nLo, int nUp, const int32_t* __restrict__ loCol,
                                     const int32_t* __restrict__ loFace, const int32_t* __restrict__ upCol,
                                     const int32_t* __restrict__ upFace, const double* __restrict__ upper,
                                     const double* __restrict__ lower, double* __restrict__ prod,
                                     double* __restrict__ coefLo, double* __restrict__ coefUp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nLo) {
        double p = 0.0, c = 0.0;
        if (loCol[k] >= 0) {
            const int32_t a = loFace[k];
            const int fa = a & 0x7fffffff;
            const double aul = a < 0 ? lower[fa] : upper[fa];
            const double alu = a < 0 ? upper[fa] : lower[fa];
            p = alu * aul;
            c = aul;
        }
        prod[k] = p;
        coefLo[k] = c;
    } else if (k - nLo < nUp) {
        const int q = k - nLo;
        double c = 0.0;
        if (upCol[q] >= 0) {
            const int32_t b = upFace[q];
            const int fb = b & 0x7fffffff;
            c = b < 0 ? upper[fb] : lower[fb];
        }
        coefUp[q] = c;
    }
}

// rD = D - sum_l A_lu A_ul / rD[l] in level order; rDs[slot] = 1 / rD[row] as each level completes.
__global__ void __launch_bounds__(kDiluThreads) k_dilu_factor_stream(
    const DiluSys* __restrict__ ds, const DiluLevel* __restrict__ lev, int W, int M,
    const int32_t* __restrict__ slotRow, const int32_t* __restrict__ loCol, const double* __restrict__ prod,
    const double* __restrict__ diag, double* __restrict__ rDs) {
    extern __shared__ __align__(16) char dsm[];
    const DiluSys d = ds[blockIdx.x];
    double* sh;
    DiluLevel* lt;
    char* ring = dilu_stream_setup(dsm, d, lev, diag, sh, lt);
    dilu_stream<true, false>(lt, d.nLev, ring, W, M, slotRow, nullptr, loCol, prod,
                             [&](const DiluStage& S, const DiluLevel& L) {
                                 const int q = threadIdx.x, c = S.row[q];
                                 double v = sh[c];
                                 for (int j = 0; j < L.mlo; ++j) {
                                     const int l = S.col[j * L.width + q];
                                     if (l < 0) break;
                                     v -= S.v[j * L.width + q] / sh[l];
                                 }
                                 sh[c] = v;
                                 rDs[L.s0 + q] = 1.0 / v;
                             });
}

// w = M^-1 r: forward w[u] = rD[u] r[u] - sum rD[u] A_ul w[l], backward w[l] -= sum rD[l] A_lu w[u]
// (each product formed left to right, as the reference's expressions do)
__global__ void __launch_bounds__(kDiluThreads) k_dilu_apply_stream(
    const DiluSys* __restrict__ ds, const DiluLevel* __restrict__ lev, int W, int M,
    const int32_t* __restrict__ slotRow, const double* __restrict__ rDs, const int32_t* __restrict__ loCol,
    const double* __restrict__ coefLo, const int32_t* __restrict__ upCol, const double* __restrict__ coefUp,
    const double* r, double* w, const SysState* st, int flag) {
    pdl_entry();
    extern __shared__ __align__(16) char dsm[];
    const DiluSys d = ds[blockIdx.x];
    if (st != nullptr && sys_idle(st[d.sys], flag)) return;
    double* sh;
    DiluLevel* lt;
    char* ring = dilu_stream_setup(dsm, d, lev, r, sh, lt);
    dilu_stream<true, false>(lt, d.nLev, ring, W, M, slotRow, rDs, loCol, coefLo,
                             [&](const DiluStage& S, const DiluLevel& L) {
                                 const int q = threadIdx.x, c = S.row[q];
                                 const double rd = S.a[q];
                                 double wc = rd * sh[c];
                                 for (int j = 0; j < L.mlo; ++j) {
                                     const int l = S.col[j * L.width + q];
                                     if (l < 0) break;
                                     wc -= rd * S.v[j * L.width + q] * sh[l];
                                 }
                                 sh[c] = wc;
                             });
    dilu_stream<false, true>(lt, d.nLev, ring, W, M, slotRow, rDs, upCol, coefUp,
                             [&](const DiluStage& S, const DiluLevel& L) {
                                 const int q = threadIdx.x, c = S.row[q];
                                 const double rd = S.a[q];
                                 double wc = sh[c];
                                 for (int j = 0; j < L.mup; ++j) {
                                     const int u = S.col[j * L.width + q];
                                     if (u < 0) break;
                                     wc -= rd * S.v[j * L.width + q] * sh[u];
                                 }
                                 sh[c] = wc;
                             });
    for (int i = threadIdx.x; i < d.rowCount; i += blockDim.x) w[d.rowBegin + i] = sh[i];
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
