// Level-0 row kernels of box meshes (layout in box.h): the Gauss-Seidel colour step, the residual
// and the PCG matrix product with its fused dot.  A row finds its (at most six) neighbours by index
// arithmetic and reads the face coefficients from three per-direction arrays, each face stored once
// at the cell on its minus side: per row 3 coefficients and no column indices, against 6
// coefficients + 6 indices of a SELL row, and no dependent index load before the gathers.
//
// Every row sum runs over the cell's faces in ascending face order, which on a box is
//   -z, -y, -x (internal faces the cell neighbours), +x, +y, +z (faces it owns), then the cyclic
//   faces of x, y, z,
// the order of the SELL rows and of the reference's face loops, so results are those of the SELL
// kernels bit for bit.
#pragma once

#include "box.h"
#include "kernels.cuh"

namespace vlm {

// Loads of the arrays that stay fixed for a whole solve (face coefficients, diagonal), marked
// evict-last in L2: a level-0 sweep re-reads them in each colour step, and the FP32 set of a
// 128^3 box (coefficients 25 MB, diagonal 8 MB) fits in the 126 MB L2 beside the vectors.
__device__ __forceinline__ uint64_t l2_keep() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float ld_keep(const float* p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_keep(const double* p, uint64_t pol) {
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
    return v;
}

__device__ __forceinline__ int fast_div(int n, FastDiv d) {
    return d.shift < 0 ? n : int(__umulhi(unsigned(n), d.m) >> d.shift);
}

// Cell of a level-0 row: false for padding rows.  C: colour, q: x-row index j + ny k.
__device__ __forceinline__ bool box_locate(const BoxSys& B, int row, int& C, int& i, int& j, int& k, int& q) {
    C = row >= B.base1 ? 1 : 0;
    const int s = row - (C ? B.base1 : B.base0);
    if (s >= B.slots) return false;
    q = fast_div(s, B.divH);
    const int m = s - q * B.H;
    k = fast_div(q, B.divNy);
    j = q - k * B.ny;
    i = 2 * m + ((j + k + C) & 1);
    return i < B.nx;
}

__device__ __forceinline__ BoxSys box_load(const BoxSys* __restrict__ boxes, int sys) {
    static_assert(sizeof(BoxSys) == 48, "BoxSys is read as three int4");
    const int4* p = reinterpret_cast<const int4*>(boxes + sys);
    const int4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    return BoxSys{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, FastDiv{unsigned(c.x), c.y}, FastDiv{unsigned(c.z), c.w}};
}

// One row's neighbours (rows and face coefficients, in the six directions) loaded ahead of the
// gathers, before the kernel waits for its predecessor; accumulate() gathers X and sums the terms
// s -= (MINUS) or += a_f X(nbr) in the cell's face order.  xf(row) reads a neighbour's value.
template <class T>
struct BoxRowPre {
    bool valid = false;
    int i, j, k, nx, ny, nz, per;
    int rmx, rpx, rmy, rpy, rmz, rpz;
    T amx, apx, amy, apy, amz, apz;
    __device__ __forceinline__ void load(const BoxSys& B, int row, const T* __restrict__ cx, const T* __restrict__ cy,
                                         const T* __restrict__ cz) {
        int C, q;
        valid = box_locate(B, row, C, i, j, k, q);
        if (!valid) return;
        const int H = B.H;
        nx = B.nx;
        ny = B.ny;
        nz = B.nz;
        per = B.per;
        const int o = C ? B.base0 : B.base1;  // the other colour's group: every face neighbour is there
        const int ih = i >> 1;
        const int xr = o + q * H;
        const bool px = per & 1, py = per & 2, pz = per & 4;
        rmx = xr + (i > 0 ? (i - 1) >> 1 : (nx - 1) >> 1);
        rpx = xr + (i < nx - 1 ? (i + 1) >> 1 : 0);
        rmy = o + (j > 0 ? q - 1 : q + ny - 1) * H + ih;
        rpy = o + (j < ny - 1 ? q + 1 : q - (ny - 1)) * H + ih;
        rmz = o + (k > 0 ? q - ny : q + (nz - 1) * ny) * H + ih;
        rpz = o + (k < nz - 1 ? q + ny : q - (nz - 1) * ny) * H + ih;
        const uint64_t pol = l2_keep();
        amx = apx = amy = apy = amz = apz = T(0);
        if (k > 0 || pz) amz = ld_keep(cz + rmz, pol);
        if (j > 0 || py) amy = ld_keep(cy + rmy, pol);
        if (i > 0 || px) amx = ld_keep(cx + rmx, pol);
        if (i < nx - 1 || px) apx = ld_keep(cx + row, pol);
        if (j < ny - 1 || py) apy = ld_keep(cy + row, pol);
        if (k < nz - 1 || pz) apz = ld_keep(cz + row, pol);
    }
    template <bool MINUS, class XF>
    __device__ __forceinline__ T accumulate(XF xf, T s) const {
        if (!valid) return s;
        const bool px = per & 1, py = per & 2, pz = per & 4;
        const bool hmx = i > 0 || px, hpx = i < nx - 1 || px;
        const bool hmy = j > 0 || py, hpy = j < ny - 1 || py;
        const bool hmz = k > 0 || pz, hpz = k < nz - 1 || pz;
        T vmx = T(0), vpx = T(0), vmy = T(0), vpy = T(0), vmz = T(0), vpz = T(0);
        if (hmz) vmz = xf(rmz);
        if (hmy) vmy = xf(rmy);
        if (hmx) vmx = xf(rmx);
        if (hpx) vpx = xf(rpx);
        if (hpy) vpy = xf(rpy);
        if (hpz) vpz = xf(rpz);
        auto term = [&](T a, T v) {
            if (MINUS)
                s -= a * v;
            else
                s += a * v;
        };
        if (k > 0) term(amz, vmz);
        if (j > 0) term(amy, vmy);
        if (i > 0) term(amx, vmx);
        if (i < nx - 1) term(apx, vpx);
        if (j < ny - 1) term(apy, vpy);
        if (k < nz - 1) term(apz, vpz);
        if (px) {
            if (i == 0)
                term(amx, vmx);
            else if (i == nx - 1)
                term(apx, vpx);
        }
        if (py) {
            if (j == 0)
                term(amy, vmy);
            else if (j == ny - 1)
                term(apy, vpy);
        }
        if (pz) {
            if (k == 0)
                term(amz, vmz);
            else if (k == nz - 1)
                term(apz, vpz);
        }
        return s;
    }
};

// Coefficients of the box level 0 from the LDU face coefficients (symmetric: upper == lower):
// coef[d * nrows + row] = upper[boxFace[...]] (0 where the cell has no +d face).
__global__ void k_box_coef(int n3, const int32_t* __restrict__ face, const double* __restrict__ upper,
                           double* __restrict__ c64, float* __restrict__ c32) {
    pdl_entry();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n3) return;
    const int f = face[t];
    const double v = f >= 0 ? upper[f] : 0.0;
    c64[t] = v;
    if (c32) c32[t] = (float)v;
}

// Gauss-Seidel colour step (GAMG.cpp:368-380) on the rows of one colour; MODE as k_smooth_gs:
// 0 plain, 1 first colour from x = 0 (x = r / D), 2 first colour of the first post-sweep with the
// coarse-grid correction x + xc[agg] applied to the neighbours it reads.
__device__ __forceinline__ bool box_rows(const BoxRows& R, const SysState* st, int flag, int& row, BoxSys& B,
                                         bool& idle, int& sys) {
    if (R.ch == nullptr) {
        row = R.begin + int(blockIdx.x) * kRowsPerCta + int(threadIdx.x);
        B = R.one;
        idle = false;
        sys = 0;
        return row < R.end;
    }
    const Chunk c = R.ch[blockIdx.x];
    row = c.start + int(threadIdx.x);
    sys = c.sys;
    if ((int)threadIdx.x >= c.count) return false;
    B = box_load(R.boxes, c.sys);
    idle = false;
    return true;
}

// Gauss-Seidel colour step (GAMG.cpp:368-380) on the rows of one colour; MODE as k_smooth_gs:
// 0 plain, 1 first colour from x = 0 (x = r / D), 2 first colour of the first post-sweep with the
// coarse-grid correction x + xc[agg] applied to the neighbours it reads.
template <class T, int MODE = 0>
__global__ void __launch_bounds__(kRowsPerCta) k_box_gs(BoxRows R, const T* __restrict__ coef, int nrows,
                                                        const T* __restrict__ diag, const T* __restrict__ r, T* x,
                                                        const int32_t* __restrict__ agg, const T* __restrict__ xc,
                                                        const SysState* st, int flag) {
    pdl_launch();
    int row, sys;
    BoxSys B;
    bool idle;
    if (!box_rows(R, st, flag, row, B, idle, sys)) return;
    const T dg = ld_keep(diag + row, l2_keep());
    BoxRowPre<T> pre;
    if (MODE != 1) pre.load(B, row, coef, coef + nrows, coef + 2 * size_t(nrows));
    pdl_wait();
    if (R.ch != nullptr && sys_idle(st[sys], flag)) return;
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
    x[row] = pre.template accumulate<true>(xf, r[row]) / dg;
}

// res = r - A x (GAMG.cpp:387-401: diagonal first, then the faces in order)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_box_residual(BoxRows R, const T* __restrict__ coef, int nrows,
                                                              const T* __restrict__ diag, const T* __restrict__ r,
                                                              const T* __restrict__ x, T* __restrict__ res,
                                                              const SysState* st, int flag) {
    pdl_launch();
    int row, sys;
    BoxSys B;
    bool idle;
    if (!box_rows(R, st, flag, row, B, idle, sys)) return;
    const T dg = ld_keep(diag + row, l2_keep());
    BoxRowPre<T> pre;
    pre.load(B, row, coef, coef + nrows, coef + 2 * size_t(nrows));
    pdl_wait();
    if (R.ch != nullptr && sys_idle(st[sys], flag)) return;
    res[row] = pre.template accumulate<true>([&](int j) { return __ldg(x + j); }, r[row] - dg * x[row]);
}

// Ap = A p ; wApA = sum Ap.p ; alpha = wArA / wApA (k_pcg_spmv on the box layout)
template <class T, int FLAG, bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_box_pcg_spmv(const Chunk* __restrict__ ch,
                                                              const BoxSys* __restrict__ boxes,
                                                              const T* __restrict__ coef, int nrows,
                                                              const T* __restrict__ diag, const T* __restrict__ p,
                                                              T* __restrict__ Ap, RedCtx R, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    const BoxSys B = box_load(boxes, c.sys);
    pdl_wait();
    if (sys_idle(st[c.sys], FLAG)) return;
    auto xf = [&](int j) -> T { return __ldg(p + j); };
    BlockSum<1, EXACT> acc;
    acc.begin();
    for (int row = c.start + (int)threadIdx.x; row < c.start + c.count; row += kRowsPerCta) {
        const T pr = p[row];
        BoxRowPre<T> pre;
        pre.load(B, row, coef, coef + nrows, coef + 2 * size_t(nrows));
        const T y = pre.template accumulate<false>(xf, ld_keep(diag + row, l2_keep()) * pr);
        Ap[row] = y;
        acc.add(0, (double)y * (double)pr);
    }
    double out[1];
    if (acc.finish(c, R, out)) {
        SysState& s = st[c.sys];
        if (fabs(out[0]) < kVSMALL) {
            if (FLAG == kFlagDone) {
                s.done = 1;
            } else {
                s.innerDone = 1;
                s.s1 = 1.0;
            }
        } else {
            s.alpha = s.wArA / out[0];
        }
    }
}

}  // namespace vlm
