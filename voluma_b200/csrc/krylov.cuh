// Krylov-level kernels: initial residual + normFactor, PCG and PBiCGStab vector updates
// fused with their global reductions, FP64 defect correction around an FP32 inner solve.
// Scalar recurrences (alpha, beta, omega, convergence) are evaluated on the device by the
// CTA that completes a system's reduction, so an iteration needs no host round trip.
//
// Level-0 chunks may hold up to kWideRows rows: every thread walks rows t, t+256, ... of its
// chunk and accumulates into a BlockSum (compensated, or exact in reproducible mode).
#pragma once

#include "kernels.cuh"

namespace vlm {

static_assert(kWideRows == 4 * kRowsPerCta, "the level-0 products take four rows per thread");

#define VLM_ROWS(c) for (int row = (c).start + (int)threadIdx.x; row < (c).start + (c).count; row += kRowsPerCta)

// A full level-0 chunk (kWideRows rows): this thread's four rows t, t + 256, ... in VLM_ROWS order,
// so a kernel can issue every row's loads before its arithmetic.
#define VLM_FULL(c) ((c).count == kWideRows)
__device__ __forceinline__ int full_row(const Chunk& c, int q) { return c.start + int(threadIdx.x) + q * kRowsPerCta; }

// converged() of LinearSolver.cpp:114-117
__device__ __forceinline__ bool dev_converged(const DevCtrl& c, int iters, double finalRes, double initRes) {
    if (iters < c.minIter) return false;
    return finalRes < c.tolerance || (c.relTol > 0 && finalRes < c.relTol * initRes);
}

// ------------------------------------------------------------------ initial residual
// Sum of x (for the normFactor reference value x̄, LinearSolver.cpp:157-159).
template <class T, bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_sum_x(const Chunk* __restrict__ ch, const T* __restrict__ x, RedCtx R,
                                                       SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    BlockSum<1, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) acc.add(0, (double)x[row]);
    double out[1];
    if (acc.finish(c, R, out)) st[c.sys].s0 = out[0];
}

// wA = A x, pA = A x̄, r = b - wA; normFactor = Σ|wA-pA|+|b-pA| + 1e-20; residualSum = Σ|r|
// (LinearSolver.cpp:149-174).  r32 (optional) receives (float)r for the mixed inner solve.
template <bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_init_residual(const Chunk* __restrict__ ch, Sell S,
                                                               const double* __restrict__ val,
                                                               const double* __restrict__ diag,
                                                               const double* __restrict__ x, const double* __restrict__ b,
                                                               const int32_t* __restrict__ perm, double* __restrict__ r,
                                                               float* __restrict__ r32, const int32_t* __restrict__ nCells,
                                                               RedCtx R, SysState* st, const DevCtrl* __restrict__ ctrlp) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    const double xRef = st[c.sys].s0 / (double)nCells[c.sys];
    BlockSum<2, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) {
        const double wA = row_plus(S, val, x, row, diag[row] * x[row]);
        // A x̄ with the same entry order as amul on a constant vector
        const int len = S.rlen[row], base = sell_base(S, row);
        double pA = diag[row] * xRef;
        for (int k = 0; k < len; ++k) pA += val[base + (k << 5)] * xRef;
        const double rr = b[row] - wA;
        r[row] = rr;
        if (r32) r32[row] = (float)rr;
        if (perm[row] >= 0) {
            acc.add(0, fabs(wA - pA) + fabs(b[row] - pA));
            acc.add(1, fabs(rr));
        }
    }
    double out[2];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        s.normFactor = out[0] + 1e-20;
        s.residualSum = out[1];
        s.initialResidual = s.residualSum / s.normFactor;
        s.finalResidual = s.initialResidual;
        s.iterations = 0;
        s.outer = 0;
        s.wArA = kGREAT;
        s.rho = 0.0;
        s.alpha = 0.0;
        s.omega = 0.0;
        s.innerInit = out[1];
        if (s.initialResidual < ctrlp->tolerance && ctrlp->minIter <= 0) {
            s.converged = 1;
            s.done = 1;
        }
        if (!isfinite(s.initialResidual)) {
            s.status = VLM_ERR_NONFINITE;
            s.done = 1;
        }
    }
}

// ------------------------------------------------------------------ preconditioners
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_precond_diag(const Chunk* __restrict__ ch, const T* __restrict__ rD,
                                                              const T* __restrict__ r, T* __restrict__ w,
                                                              const SysState* st, int flag) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (sys_idle(st[c.sys], flag)) return;
    VLM_ROWS(c) w[row] = rD[row] * r[row];
}

// rD = 1/diag (LinearSolver.cpp:66,78); padding rows: 0
template <class T>
__global__ void k_recip_diag(int n, const int32_t* __restrict__ valid, const T* __restrict__ d, T* __restrict__ rD) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    rD[i] = valid[i] >= 0 ? T(1) / d[i] : T(0);
}

// wArA = sum w.r of the iteration and beta = wArA / wArAold (0 on the first), in the CTA that
// completes the reduction.
template <int FLAG>
__device__ __forceinline__ void pcg_dot_wr_done(SysState& s, double wr) {
    const int it = FLAG == kFlagDone ? s.iterations : s.innerIterations;
    s.wArAold = s.wArA;
    s.wArA = wr;
    s.beta = it == 0 ? 0.0 : s.wArA / s.wArAold;
}

// ------------------------------------------------------------------ PCG (LinearSolver.cpp:176-201)
// wArA = Σ w·r ; beta = wArA / wArAold
// W: type of the preconditioned residual w (float when an FP32 V-cycle produced it; widening it
// here gives the same doubles a separate cast would).
template <class T, int FLAG, bool EXACT, class W = T>
__global__ void __launch_bounds__(kRowsPerCta) k_pcg_dot_wr(const Chunk* __restrict__ ch, const W* __restrict__ w,
                                                            const T* __restrict__ r, RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (sys_idle(st[c.sys], FLAG)) return;
    BlockSum<1, EXACT> acc;
    acc.begin();
    if (VLM_FULL(c)) {
        W wv[4];
        T rv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            wv[q] = w[full_row(c, q)];
            rv[q] = r[full_row(c, q)];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) acc.add(0, (double)wv[q] * (double)rv[q]);
    } else {
        VLM_ROWS(c) acc.add(0, (double)w[row] * (double)r[row]);
    }
    double out[1];
    if (acc.finish(c, R, out)) pcg_dot_wr_done<FLAG>(st[c.sys], out[0]);
}

// p = w (first iteration) or w + beta p
template <class T, int FLAG, class W = T>
__global__ void __launch_bounds__(kRowsPerCta) k_pcg_p(const Chunk* __restrict__ ch, const W* __restrict__ w,
                                                       T* __restrict__ p, const SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    const SysState& s = st[c.sys];
    if (sys_idle(s, FLAG)) return;
    const int it = FLAG == kFlagDone ? s.iterations : s.innerIterations;
    const T beta = (T)s.beta;
    if (it == 0) {
        VLM_ROWS(c) p[row] = (T)w[row];
    } else if (VLM_FULL(c)) {
        W wv[4];
        T pv[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            wv[q] = w[full_row(c, q)];
            pv[q] = p[full_row(c, q)];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) p[full_row(c, q)] = (T)wv[q] + beta * pv[q];
    } else {
        VLM_ROWS(c) p[row] = (T)w[row] + beta * p[row];
    }
}

// Ap = A p ; wApA = Σ Ap·p ; alpha = wArA / wApA (break when |wApA| < VSMALL)
template <class T, int FLAG, bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_pcg_spmv(const Chunk* __restrict__ ch, Sell S, const T* __restrict__ val,
                                                          const T* __restrict__ diag, const T* __restrict__ p,
                                                          T* __restrict__ Ap, RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (sys_idle(st[c.sys], FLAG)) return;
    BlockSum<1, EXACT> acc;
    acc.begin();
    // four consecutive rows per thread (the box layout's product adds the same partial sums)
    for (int v = 0; v < 4; ++v) {
        const int row = c.start + 4 * int(threadIdx.x) + v;
        if (row >= c.start + c.count) break;
        const T y = row_plus(S, val, p, row, diag[row] * p[row]);
        Ap[row] = y;
        acc.add(0, (double)y * (double)p[row]);
    }
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        if (fabs(out[0]) < kVSMALL) {
            if (FLAG == kFlagDone) {
                s.done = 1;
            } else {
                s.innerDone = 1;
                s.s1 = 1.0;  // inner breakdown: the outer loop stops after this correction
            }
        } else {
            s.alpha = s.wArA / out[0];
        }
    }
}

// x += alpha p ; r -= alpha Ap ; finalResidual = Σ|r| / normFactor ; convergence.
// r32 (optional): FP32 copy of the new r, the next FP32 V-cycle's input.
template <class T, int FLAG, bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_pcg_update(const Chunk* __restrict__ ch, T* __restrict__ x, T* __restrict__ r,
                                                            const T* __restrict__ p, const T* __restrict__ Ap,
                                                            const int32_t* __restrict__ perm, RedCtx R, SysState* st,
                                                            const DevCtrl* __restrict__ ctrlp, float* __restrict__ r32) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (sys_idle(st[c.sys], FLAG)) return;
    const T alpha = (T)st[c.sys].alpha;
    BlockSum<1, EXACT> acc;
    acc.begin();
    if (VLM_FULL(c)) {
        T xv[4], pv[4], rv[4], av[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int row = full_row(c, q);
            xv[q] = x[row];
            pv[q] = p[row];
            rv[q] = r[row];
            av[q] = Ap[row];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int row = full_row(c, q);
            x[row] = xv[q] + alpha * pv[q];
            const T rr = rv[q] - alpha * av[q];
            r[row] = rr;
            if (r32 != nullptr) r32[row] = (float)rr;
            acc.add(0, fabs((double)rr));
        }
    } else {
        VLM_ROWS(c) {
            x[row] += alpha * p[row];
            const T rr = r[row] - alpha * Ap[row];
            r[row] = rr;
            if (r32 != nullptr) r32[row] = (float)rr;
            acc.add(0, fabs((double)rr));
        }
    }
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        if (FLAG == kFlagDone) {
            s.finalResidual = out[0] / s.normFactor;
            s.iterations += 1;
            if (!isfinite(s.finalResidual)) {
                s.status = VLM_ERR_NONFINITE;
                s.done = 1;
            } else if (s.iterations >= ctrlp->maxIter ||
                       dev_converged(*ctrlp, s.iterations, s.finalResidual, s.initialResidual)) {
                s.done = 1;
            }
        } else {
            s.innerFinal = out[0];
            s.innerIterations += 1;
            s.iterations += 1;
            if (!isfinite(out[0])) {
                s.status = VLM_ERR_NONFINITE;
                s.innerDone = 1;
                s.done = 1;
            } else if (s.innerIterations >= ctrlp->maxInner || s.iterations >= ctrlp->maxIter ||
                       s.innerFinal < ctrlp->innerRelTol * s.innerInit) {
                s.innerDone = 1;
            }
        }
    }
}

// ------------------------------------------------------------------ mixed precision outer loop
// start of an inner solve: e = 0 is done by a zero kernel; reset the inner recurrences.
__global__ void k_inner_begin(int nsys, SysState* st) {
    pdl_entry();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    SysState& q = st[s];
    q.innerIterations = 0;
    q.innerDone = q.done;
    q.s1 = 0.0;
    q.wArA = kGREAT;
}

// ---- reference row of the defect correction
// A pressure matrix with setReference (FvMatrix.h:134-141) is A = L + refC e_ref e_ref^T: L, the
// pure-Neumann operator, has rows that sum to zero, so its constant vector is a null mode and A's
// smallest eigenvalue is about refC / N, which FP32 cannot resolve.  The defect correction then
// solves L y = r - (sum r) e_ref in FP32 with the constant mode projected out of each preconditioned
// residual (well conditioned on the complement), and restores the constant in FP64:
// e = y + ((sum r) / refC - y_ref) 1, which makes A e = r.  The reference row is the one row whose
// sum exceeds 1e-9 of its diagonal; with none or several (Dirichlet rows), nothing is projected.
__global__ void k_ref_reset(int nsys, SysState* st) {
    pdl_entry();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    st[s].refRow = -1;
    st[s].refCount = 0;
    st[s].refC = 0.0;
    st[s].sumR = 0.0;
    st[s].innerMu = 0.0;
}

__global__ void __launch_bounds__(kRowsPerCta) k_ref_detect(const Chunk* __restrict__ ch, Sell S,
                                                            const double* __restrict__ val,
                                                            const double* __restrict__ diag,
                                                            const int32_t* __restrict__ perm, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    VLM_ROWS(c) {
        if (perm[row] < 0) continue;
        const double d = diag[row];
        const double sum = row_accumulate<false>(S, val, [](int) { return 1.0; }, row, d);
        if (fabs(sum) > 1e-9 * fabs(d)) {
            if (atomicAdd(&st[c.sys].refCount, 1) == 0) {
                st[c.sys].refRow = row;
                st[c.sys].refC = sum;
            }
        }
    }
}

__global__ void k_ref_finish(int nsys, SysState* st) {
    pdl_entry();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    if (st[s].refCount != 1) st[s].refRow = -1;
}

// FP32 diagonal of the inner operator: A's, with refC taken off the reference row (L)
__global__ void __launch_bounds__(kRowsPerCta) k_ref_diag32(const Chunk* __restrict__ ch,
                                                            const double* __restrict__ diag, float* __restrict__ dL,
                                                            const SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    const int ref = st[c.sys].refRow;
    const double rc = st[c.sys].refC;
    VLM_ROWS(c) dL[row] = (float)(row == ref ? diag[row] - rc : diag[row]);
}

// sumR = sum of the initial residual
__global__ void __launch_bounds__(kRowsPerCta) k_ref_sum_r(const Chunk* __restrict__ ch, const double* __restrict__ r,
                                                           RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    BlockSum<1, false> acc;
    acc.begin();
    VLM_ROWS(c) acc.add(0, r[row]);
    double out[1];
    if (acc.finish(c, R, out)) st[c.sys].sumR = out[0];
}

// the inner right-hand side r - (sum r) e_ref: only the reference row's FP32 value changes
__global__ void k_ref_rhs(int nsys, const double* __restrict__ r, float* __restrict__ r32, const SysState* st) {
    pdl_entry();
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const SysState& q = st[s];
    if (q.refRow >= 0 && !q.done) r32[q.refRow] = (float)(r[q.refRow] - q.sumR);
}

// wArA = (z - mu) . r, mu = the mean of z over the system's cells (with a reference row), and beta
// for the inner recurrence; padding rows are left out of the sums
__global__ void __launch_bounds__(kRowsPerCta) k_inner_dot_wr(const Chunk* __restrict__ ch, const float* __restrict__ z,
                                                              const float* __restrict__ r,
                                                              const int32_t* __restrict__ perm,
                                                              const int* __restrict__ sysCells, RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (sys_idle(st[c.sys], kFlagInner)) return;
    BlockSum<3, false> acc;
    acc.begin();
    VLM_ROWS(c) {
        if (perm[row] < 0) continue;
        const double zv = (double)z[row], rv = (double)r[row];
        acc.add(0, zv * rv);
        acc.add(1, zv);
        acc.add(2, rv);
    }
    double out[3];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        const double mu = s.refRow >= 0 ? out[1] / double(sysCells[c.sys]) : 0.0;
        s.innerMu = mu;
        pcg_dot_wr_done<kFlagInner>(s, out[0] - mu * out[2]);
    }
}

// p = (z - mu) or (z - mu) + beta p on the system's cells
__global__ void __launch_bounds__(kRowsPerCta) k_inner_p(const Chunk* __restrict__ ch, const float* __restrict__ z,
                                                         float* __restrict__ p, const int32_t* __restrict__ perm,
                                                         const SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    const SysState& s = st[c.sys];
    if (sys_idle(s, kFlagInner)) return;
    const float mu = (float)s.innerMu, beta = (float)s.beta;
    const bool first = s.innerIterations == 0;
    VLM_ROWS(c) {
        if (perm[row] < 0) continue;
        const float v = z[row] - mu;
        p[row] = first ? v : v + beta * p[row];
    }
}

// x64 += e32 (+ the constant that restores A e = r around a reference row) ; then r64 = b - A x64
// in a second kernel (neighbours must be updated first)
__global__ void __launch_bounds__(kRowsPerCta) k_mixed_correct(const Chunk* __restrict__ ch, double* __restrict__ x,
                                                               const float* __restrict__ e,
                                                               const int32_t* __restrict__ perm, const SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    const SysState& s = st[c.sys];
    if (s.done) return;
    const double a = s.refRow >= 0 ? s.sumR / s.refC - (double)e[s.refRow] : 0.0;
    VLM_ROWS(c) {
        if (perm[row] < 0) continue;
        x[row] += (double)e[row] + a;
    }
}

// FP64 defect: r = b - A x (exact FP64 matrix), r32 = (float) r, finalResidual = Σ|r| / nf, sumR = Σ r
__global__ void __launch_bounds__(kRowsPerCta) k_mixed_residual(const Chunk* __restrict__ ch, Sell S,
                                                                const double* __restrict__ val,
                                                                const double* __restrict__ diag,
                                                                const double* __restrict__ x,
                                                                const double* __restrict__ b, double* __restrict__ r,
                                                                float* __restrict__ r32, RedCtx R, SysState* st,
                                                                const DevCtrl* __restrict__ ctrlp) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (st[c.sys].done) return;
    BlockSum<2, false> acc;
    acc.begin();
    VLM_ROWS(c) {
        const double wA = row_plus(S, val, x, row, diag[row] * x[row]);
        const double rr = b[row] - wA;
        r[row] = rr;
        r32[row] = (float)rr;
        acc.add(0, fabs(rr));
        acc.add(1, rr);
    }
    double out[2];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        s.sumR = out[1];
        s.finalResidual = out[0] / s.normFactor;
        s.innerInit = out[0];
        s.outer += 1;
        if (!isfinite(s.finalResidual)) {
            s.status = VLM_ERR_NONFINITE;
            s.done = 1;
        } else if (s.iterations >= ctrlp->maxIter || s.outer >= ctrlp->maxIter || s.s1 != 0.0 ||
                   dev_converged(*ctrlp, s.iterations, s.finalResidual, s.initialResidual)) {
            s.done = 1;
        }
    }
}

// ------------------------------------------------------------------ PBiCGStab (LinearSolver.cpp:202-237)
// rho = Σ r0·r ; beta = (rho/rhoOld)(alpha/omega), break on |rhoOld| or |omega| < VSMALL
template <bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_bicg_rho(const Chunk* __restrict__ ch, const double* __restrict__ r0,
                                                          const double* __restrict__ r, RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (st[c.sys].done) return;
    BlockSum<1, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) acc.add(0, r0[row] * r[row]);
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        s.rhoOld = s.rho;
        s.rho = out[0];
        if (s.iterations > 0) {
            if (fabs(s.rhoOld) < kVSMALL || fabs(s.omega) < kVSMALL)
                s.done = 1;
            else
                s.beta = (s.rho / s.rhoOld) * (s.alpha / s.omega);
        }
    }
}

// p = r (first) or r + beta (p - omega Ay)
__global__ void __launch_bounds__(kRowsPerCta) k_bicg_p(const Chunk* __restrict__ ch, const double* __restrict__ r,
                                                        const double* __restrict__ Ay, double* __restrict__ p,
                                                        const SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    const SysState& s = st[c.sys];
    if (s.done) return;
    if (s.iterations == 0) {
        VLM_ROWS(c) p[row] = r[row];
    } else {
        const double beta = s.beta, omega = s.omega;
        VLM_ROWS(c) p[row] = r[row] + beta * (p[row] - omega * Ay[row]);
    }
}

// Ay = A y ; alpha = rho / Σ r0·Ay (break when < VSMALL)
template <bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_bicg_spmv_alpha(const Chunk* __restrict__ ch, Sell S,
                                                                 const double* __restrict__ val,
                                                                 const double* __restrict__ diag,
                                                                 const double* __restrict__ y, double* __restrict__ Ay,
                                                                 const double* __restrict__ r0, RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (st[c.sys].done) return;
    BlockSum<1, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) {
        const double a = row_plus(S, val, y, row, diag[row] * y[row]);
        Ay[row] = a;
        acc.add(0, r0[row] * a);
    }
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        if (fabs(out[0]) < kVSMALL)
            s.done = 1;
        else
            s.alpha = s.rho / out[0];
    }
}

// s = r - alpha Ay ; iterations++ ; finalResidual = Σ|s|/nf ; converged -> early exit flag (s1 = 1)
template <bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_bicg_s(const Chunk* __restrict__ ch, const double* __restrict__ r,
                                                        const double* __restrict__ Ay, double* __restrict__ sv, RedCtx R,
                                                        SysState* st, const DevCtrl* __restrict__ ctrlp) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (st[c.sys].done) return;
    const double alpha = st[c.sys].alpha;
    BlockSum<1, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) {
        const double s = r[row] - alpha * Ay[row];
        sv[row] = s;
        acc.add(0, fabs(s));
    }
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        s.iterations += 1;
        s.finalResidual = out[0] / s.normFactor;
        s.s1 = 0.0;
        if (!isfinite(s.finalResidual)) {
            s.status = VLM_ERR_NONFINITE;
            s.done = 1;
        } else if (dev_converged(*ctrlp, s.iterations, s.finalResidual, s.initialResidual)) {
            s.s1 = 1.0;  // early exit: x += alpha y, then stop
        }
    }
}

// early exit of LinearSolver.cpp:224-227
__global__ void __launch_bounds__(kRowsPerCta) k_bicg_early(const Chunk* __restrict__ ch, double* __restrict__ x,
                                                            const double* __restrict__ y, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    SysState& s = st[c.sys];
    if (s.done || s.s1 == 0.0) return;
    const double alpha = s.alpha;
    VLM_ROWS(c) x[row] += alpha * y[row];
}

// closes the early exit (separate launch so every CTA above saw s1 before done is set)
__global__ void k_bicg_early_close(int nsys, SysState* st) {
    pdl_entry();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nsys && !st[i].done && st[i].s1 != 0.0) {
        st[i].converged = 1;
        st[i].done = 1;
    }
}

// t = A z ; tAtA = Σ t·t ; tAsA = Σ t·s ; omega = tAtA > VSMALL ? tAsA/tAtA : 0
template <bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_bicg_spmv_omega(const Chunk* __restrict__ ch, Sell S,
                                                                 const double* __restrict__ val,
                                                                 const double* __restrict__ diag,
                                                                 const double* __restrict__ z, double* __restrict__ t,
                                                                 const double* __restrict__ sv, RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (st[c.sys].done) return;
    BlockSum<2, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) {
        const double a = row_plus(S, val, z, row, diag[row] * z[row]);
        t[row] = a;
        acc.add(0, a * a);
        acc.add(1, a * sv[row]);
    }
    double out[2];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        s.omega = out[0] > kVSMALL ? out[1] / out[0] : 0.0;
    }
}

// x += alpha y + omega z ; r = s - omega t ; finalResidual = Σ|r| / nf
template <bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_bicg_update(const Chunk* __restrict__ ch, double* __restrict__ x,
                                                             double* __restrict__ r, const double* __restrict__ y,
                                                             const double* __restrict__ z, const double* __restrict__ sv,
                                                             const double* __restrict__ t, RedCtx R, SysState* st,
                                                             const DevCtrl* __restrict__ ctrlp) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    if (st[c.sys].done) return;
    const double alpha = st[c.sys].alpha, omega = st[c.sys].omega;
    BlockSum<1, EXACT> acc;
    acc.begin();
    VLM_ROWS(c) {
        x[row] += alpha * y[row] + omega * z[row];
        const double rr = sv[row] - omega * t[row];
        r[row] = rr;
        acc.add(0, fabs(rr));
    }
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
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

// ------------------------------------------------------------------ plain SpMV (amul)
__global__ void __launch_bounds__(kRowsPerCta) k_amul(const Chunk* __restrict__ ch, Sell S, const double* __restrict__ val,
                                                      const double* __restrict__ diag, const double* __restrict__ x,
                                                      double* __restrict__ y) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    pdl_wait();
    VLM_ROWS(c) y[row] = row_plus(S, val, x, row, diag[row] * x[row]);
}

}  // namespace vlm
