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

// ------------------------------------------------------------------ four slots per thread
// Range form with H % 4 == 0: thread g takes the four consecutive slots 4g..4g+3 of its colour
// group, which lie in one x-row (same j, k, colour) at x = i0, i0+2, i0+4, i0+6.  Their own arrays
// (r, diagonal, +x/+y/+z coefficients) and their +-y and +-z neighbours in the other colour are
// four consecutive, 16-byte aligned rows each (one vector load); the +-x neighbours are the other
// colour's slots m0-1+p .. m0+4+p of the same x-row (one vector load and one scalar).  Index
// arithmetic is paid once per four rows, and every row still sums its faces in its own face order.
template <class T> struct V4 { T v[4]; };

__device__ __forceinline__ V4<float> ld4(const float* p) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    return V4<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ V4<double> ld4(const double* p) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    return V4<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ V4<float> ld4_keep(const float* p, uint64_t pol) {
    float4 a;
    asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w) : "l"(p), "l"(pol));
    return V4<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ V4<double> ld4_keep(const double* p, uint64_t pol) {
    double2 a, b;
    asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(a.x), "=d"(a.y) : "l"(p), "l"(pol));
    asm("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(b.x), "=d"(b.y) : "l"(p + 2), "l"(pol));
    return V4<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double* p, const double (&v)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

// A four-slot group's geometry and fixed operands (coefficients, diagonal), loaded ahead of the wait.
// Every neighbour row is formed with the periodic wrap (always a row of the other colour's group),
// and per-row predicates say which faces the cell has and whether each is internal or cyclic, so
// walls, cyclic faces and padding slots of odd x extents take the same instruction stream.
template <class T>
struct BoxGroup4 {
    bool valid;     // not a padding group (slots past the colour group's cells)
    int p;          // parity offset of the group's x-row: cell x = 2 (m0 + v) + p
    int xr, xe, rmy, rpy, rmz, rpz;  // other colour: x-row at slot m0, the slot just outside, +-y, +-z
    // per-row faces: bit 0..5 internal -z,-y,-x,+x,+y,+z; bit 6..11 cyclic -z,-y,-x,+x,+y,+z
    int faces[4];
    V4<T> dg, cpx, cpy, cpz, cmy, cmz, cmx;  // diagonal, own +d coefficients, neighbours' -d ones
    T cme;          // the -x coefficient at slot xe (p == 0)

    // faces[] of the group's rows (x-row j, plane k, slots m0.., parity p already set)
    __device__ __forceinline__ void set_faces(const BoxSys& B, int j, int k, int m0) {
        const int nx = B.nx, ny = B.ny, nz = B.nz;
        const bool px = B.per & 1, py = B.per & 2, pz = B.per & 4;
        const int fy = (j > 0 ? 2 : (py ? 2 << 6 : 0)) | (j < ny - 1 ? 16 : (py ? 16 << 6 : 0));
        const int fz = (k > 0 ? 1 : (pz ? 1 << 6 : 0)) | (k < nz - 1 ? 32 : (pz ? 32 << 6 : 0));
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int i = 2 * (m0 + v) + p;
            const int fx = (i > 0 ? 4 : (px ? 4 << 6 : 0)) | (i < nx - 1 ? 8 : (px ? 8 << 6 : 0));
            faces[v] = i < nx ? (fx | fy | fz) : 0;  // i >= nx: a padding slot (odd nx)
        }
    }

    __device__ __forceinline__ void load(const BoxSys& B, int row, const T* __restrict__ cx,
                                         const T* __restrict__ cy, const T* __restrict__ cz,
                                         const T* __restrict__ diag) {
        const int C = row >= B.base1 ? 1 : 0;
        const int s = row - (C ? B.base1 : B.base0);
        valid = s < B.slots;
        if (!valid) return;
        const int H = B.H, ny = B.ny, nz = B.nz;
        const int q = fast_div(s, B.divH);
        const int m0 = s - q * H;
        const int k = fast_div(q, B.divNy);
        const int j = q - k * ny;
        p = (j + k + C) & 1;
        const int o = C ? B.base0 : B.base1;
        const int x0 = o + q * H;  // the other colour's x-row
        xr = x0 + m0;
        // the slot just outside the vector: p == 0 -> m0 - 1 (wrapping to H - 1), p == 1 -> m0 + 4 (to 0)
        xe = p == 0 ? (m0 > 0 ? xr - 1 : x0 + H - 1) : (m0 + 4 < H ? xr + 4 : x0);
        rmy = o + (j > 0 ? q - 1 : q + ny - 1) * H + m0;
        rpy = o + (j < ny - 1 ? q + 1 : q - (ny - 1)) * H + m0;
        rmz = o + (k > 0 ? q - ny : q + (nz - 1) * ny) * H + m0;
        rpz = o + (k < nz - 1 ? q + ny : q - (nz - 1) * ny) * H + m0;
        set_faces(B, j, k, m0);
        const uint64_t pol = l2_keep();
        dg = ld4_keep(diag + row, pol);
        cpx = ld4_keep(cx + row, pol);
        cpy = ld4_keep(cy + row, pol);
        cmy = ld4_keep(cy + rmy, pol);
        if (nz > 1) {
            cpz = ld4_keep(cz + row, pol);
            cmz = ld4_keep(cz + rmz, pol);
        }
        cmx = ld4_keep(cx + xr, pol);  // p == 1: the -x neighbours are slots m0..m0+3
        cme = p == 0 ? ld_keep(cx + xe, pol) : T(0);
    }

    // s[v] (op)= a_f X(neighbour) over the faces of row v in face order: internal -z, -y, -x, +x, +y,
    // +z, then the cyclic faces of x, y, z.  xv4(row): four neighbour values; xv1(row): one.
    template <bool MINUS, bool Z, class XV4, class XV1>
    __device__ __forceinline__ void accumulate(XV4 xv4, XV1 xv1, T (&s)[4]) const {
        const V4<T> xmy = xv4(rmy), xpy = xv4(rpy), xrow = xv4(xr);
        V4<T> xmz, xpz;
        if (Z) {
            xmz = xv4(rmz);
            xpz = xv4(rpz);
        }
        const T vx = xv1(xe);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            // p == 0: -x is slot m0+v-1, +x slot m0+v; p == 1: -x slot m0+v, +x slot m0+v+1
            const T am = p == 0 ? (v == 0 ? cme : cmx.v[v - 1]) : cmx.v[v];
            const T vm = p == 0 ? (v == 0 ? vx : xrow.v[v - 1]) : xrow.v[v];
            const T vp = p == 0 ? xrow.v[v] : (v == 3 ? vx : xrow.v[v + 1]);
            const int f = faces[v];
            T a = s[v];
            auto term = [&](int bit, T c, T x) {
                if (f & bit) {
                    if (MINUS)
                        a -= c * x;
                    else
                        a += c * x;
                }
            };
            if (Z) term(1, cmz.v[v], xmz.v[v]);
            term(2, cmy.v[v], xmy.v[v]);
            term(4, am, vm);
            term(8, cpx.v[v], vp);
            term(16, cpy.v[v], xpy.v[v]);
            if (Z) term(32, cpz.v[v], xpz.v[v]);
            term(4 << 6, am, vm);
            term(8 << 6, cpx.v[v], vp);
            term(2 << 6, cmy.v[v], xmy.v[v]);
            term(16 << 6, cpy.v[v], xpy.v[v]);
            if (Z) {
                term(1 << 6, cmz.v[v], xmz.v[v]);
                term(32 << 6, cpz.v[v], xpz.v[v]);
            }
            s[v] = a;
        }
    }
};

// Coherent (L2) vector loads: values that other CTAs of the same launch write (the fused sweep).
__device__ __forceinline__ V4<float> ld4_cg(const float* p) {
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    return V4<float>{{a.x, a.y, a.z, a.w}};
}
__device__ __forceinline__ V4<double> ld4_cg(const double* p) {
    const double2 a = __ldcg(reinterpret_cast<const double2*>(p)), b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
    return V4<double>{{a.x, a.y, b.x, b.y}};
}

// One four-slot group of a Gauss-Seidel colour step after its fixed operands are loaded (G.load):
// MODE 0 plain, 1 from a zero iterate (x = r / D), 2 with the coarse-grid correction x + xc[agg] of the
// neighbours read (the prolongation fused into the first post-smoothing step).  COH: the other colour
// was written by this launch (coherent loads) instead of by an earlier one.
template <class T, int MODE, bool COH>
__device__ __forceinline__ void box_gs4_group(const BoxGroup4<T>& G, const BoxSys& B, int row0,
                                              const T* __restrict__ diag, const T* __restrict__ r, T* x,
                                              const int32_t* __restrict__ agg, const T* __restrict__ xc) {
    if (MODE == 1) {
        const V4<T> rv = ld4(r + row0);
        T out[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) out[v] = rv.v[v] / G.dg.v[v];
        st4(x + row0, out);
        return;
    }
    if (!G.valid) {
        // padding slots past the colour group's cells: x = r / D as for any padding row
        for (int v = 0; v < 4; ++v) x[row0 + v] = r[row0 + v] / diag[row0 + v];
        return;
    }
    // the other colour's values (x, plus the coarse-grid correction for MODE 2)
    auto xv4 = [&](int j) -> V4<T> {
        V4<T> a = COH ? ld4_cg(x + j) : ld4(x + j);
        if (MODE == 2) {
            const int4 g = __ldg(reinterpret_cast<const int4*>(agg + j));
            const int gi[4] = {g.x, g.y, g.z, g.w};
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (gi[v] >= 0) a.v[v] += __ldg(xc + gi[v]);
        }
        return a;
    };
    auto xv1 = [&](int j) -> T {
        T a = COH ? __ldcg(x + j) : __ldg(x + j);
        if (MODE == 2) {
            const int g = __ldg(agg + j);
            if (g >= 0) a += __ldg(xc + g);
        }
        return a;
    };
    const V4<T> rv = ld4(r + row0);
    T s[4] = {rv.v[0], rv.v[1], rv.v[2], rv.v[3]};
    if (B.nz > 1)
        G.template accumulate<true, true>(xv4, xv1, s);
    else
        G.template accumulate<true, false>(xv4, xv1, s);
    T out[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) out[v] = s[v] / G.dg.v[v];
    st4(x + row0, out);
}

// Gauss-Seidel colour step, four slots per thread (range form, H % 4 == 0); MODE as k_box_gs.
template <class T, int MODE = 0>
__global__ void __launch_bounds__(kRowsPerCta) k_box_gs4(BoxRows R, const T* __restrict__ coef, int nrows,
                                                         const T* __restrict__ diag, const T* __restrict__ r, T* x,
                                                         const int32_t* __restrict__ agg, const T* __restrict__ xc) {
    pdl_launch();
    const int row0 = R.begin + 4 * (int(blockIdx.x) * kRowsPerCta + int(threadIdx.x));
    if (row0 >= R.end) return;
    const BoxSys& B = R.one;
    BoxGroup4<T> G;
    if (MODE == 1)
        G.dg = ld4_keep(diag + row0, l2_keep());
    else
        G.load(B, row0, coef, coef + nrows, coef + 2 * size_t(nrows), diag);
    pdl_wait();
    box_gs4_group<T, MODE, false>(G, B, row0, diag, r, x, agg, xc);
}

// ---------------------------------------------------------------- fused two-colour sweep
// Both colour steps of a red-black sweep in one launch.  Pieces of kSweepPiece slots are taken in
// ticket order from a device counter: first every piece of the first colour, then every piece of the
// second; a second-colour piece starts once the first-colour pieces it reads (its z-planes and the two
// next to them, across the periodic wrap) carry this launch's done stamp.  A piece only waits for
// lower tickets, which CTAs that are already running hold, so the waits end without any guarantee
// of co-residency; each is still bounded (spin limit, then an error word and no wait).  The last CTA
// resets the counters and advances the launch epoch that the stamps compare against.
constexpr int kSweepPiece = 4 * kRowsPerCta;
constexpr long long kSweepSpinLimit = 1ll << 22;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Lanes of one warp wait until stamps[lo..hi] all equal `want` (bounded).
__device__ __forceinline__ void sweep_wait_range(const unsigned* stamps, int lo, int hi, unsigned want,
                                                 SweepSync* sync) {
    for (int i = lo + int(threadIdx.x & 31); i <= hi; i += 32) {
        long long n = 0;
        while (ld_acquire_u32(stamps + i) != want) {
            if (++n > kSweepSpinLimit) {
                atomicOr(&sync->err, 1u);
                break;
            }
            __nanosleep(64);
        }
    }
}

// Launch bounds: the colour step's register budget (4 resident CTAs per SM in FP32, 2 in FP64).
template <class T, int MODE1>
__global__ void __launch_bounds__(kRowsPerCta, sizeof(T) == 4 ? 4 : 2) k_box_sweep4(BoxSys B, int beginA, int endA, int beginB, int endB,
                                                            const T* __restrict__ coef, int nrows,
                                                            const T* __restrict__ diag, const T* __restrict__ r, T* x,
                                                            const int32_t* __restrict__ agg, const T* __restrict__ xc,
                                                            SweepSync* sync, unsigned* done) {
    pdl_launch();
    pdl_wait();
    __shared__ int sTicket;
    __shared__ unsigned sEpoch;
    if (threadIdx.x == 0) sEpoch = ld_acquire_u32(&sync->epoch);
    const T* cx = coef;
    const T* cy = coef + nrows;
    const T* cz = coef + 2 * size_t(nrows);
    const int nA = (endA - beginA + kSweepPiece - 1) / kSweepPiece;
    const int nB = (endB - beginB + kSweepPiece - 1) / kSweepPiece;
    const int plane = B.H * B.ny;  // slots of one colour in one z-plane
    const bool perZ = (B.per & 4) != 0;
    __syncthreads();
    const unsigned stamp = sEpoch + 1u;
    for (;;) {
        if (threadIdx.x == 0) sTicket = int(atomicAdd(&sync->ticket, 1u));
        __syncthreads();
        const int t = sTicket;
        __syncthreads();
        if (t >= nA + nB) break;
        const bool first = t < nA;
        const int q = first ? t : t - nA;
        if (!first && threadIdx.x < 32) {
            // the first colour's slots this piece reads: its z-planes and one more on each side
            const int s0 = q * kSweepPiece, s1 = min((q + 1) * kSweepPiece, endB - beginB);
            const int k0 = s0 / plane, k1 = (s1 - 1) / plane;
            const int lo = max(k0 - 1, 0) * plane, hi = min(k1 + 2, B.nz) * plane;
            sweep_wait_range(done, lo / kSweepPiece, min((hi - 1) / kSweepPiece, nA - 1), stamp, sync);
            if (perZ && k0 == 0) sweep_wait_range(done, ((B.nz - 1) * plane) / kSweepPiece, nA - 1, stamp, sync);
            if (perZ && k1 == B.nz - 1) sweep_wait_range(done, 0, min((plane - 1) / kSweepPiece, nA - 1), stamp, sync);
        }
        if (!first) __syncthreads();
        const int row0 = (first ? beginA : beginB) + q * kSweepPiece + 4 * int(threadIdx.x);
        if (row0 < (first ? endA : endB)) {
            BoxGroup4<T> G;
            if (MODE1 != 0 && first) {
                if (MODE1 == 1)
                    G.dg = ld4_keep(diag + row0, l2_keep());
                else
                    G.load(B, row0, cx, cy, cz, diag);
                box_gs4_group<T, MODE1, false>(G, B, row0, diag, r, x, agg, xc);
            } else {
                // the other colour: written by an earlier launch (first colour) or by this one
                G.load(B, row0, cx, cy, cz, diag);
                box_gs4_group<T, 0, true>(G, B, row0, diag, r, x, agg, xc);
            }
        }
        if (first) {
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                st_release_u32(done + t, stamp);
            }
        }
    }
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&sync->finished, 1u) == gridDim.x - 1) {
            sync->ticket = 0u;
            sync->finished = 0u;
            __threadfence();
            st_release_u32(&sync->epoch, stamp);
        }
    }
}

// res = r - A x, four slots per thread (range form, H % 4 == 0)
template <class T>
__global__ void __launch_bounds__(kRowsPerCta) k_box_residual4(BoxRows R, const T* __restrict__ coef, int nrows,
                                                               const T* __restrict__ diag, const T* __restrict__ r,
                                                               const T* __restrict__ x, T* __restrict__ res) {
    pdl_launch();
    const int row0 = R.begin + 4 * (int(blockIdx.x) * kRowsPerCta + int(threadIdx.x));
    if (row0 >= R.end) return;
    const BoxSys& B = R.one;
    const T* cx = coef;
    const T* cy = coef + nrows;
    const T* cz = coef + 2 * size_t(nrows);
    BoxGroup4<T> G;
    G.load(B, row0, cx, cy, cz, diag);
    auto xf = [&](int j) -> T { return __ldg(x + j); };
    if (!G.valid) {
        pdl_wait();
        for (int v = 0; v < 4; ++v) res[row0 + v] = r[row0 + v] - diag[row0 + v] * x[row0 + v];
        return;
    }
    pdl_wait();
    const V4<T> rv = ld4(r + row0), xo = ld4(x + row0);
    T s[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) s[v] = rv.v[v] - G.dg.v[v] * xo.v[v];
    auto xv4 = [&](int j) { return ld4(x + j); };
    if (B.nz > 1)
        G.template accumulate<true, true>(xv4, xf, s);
    else
        G.template accumulate<true, false>(xv4, xf, s);
    st4(res + row0, s);
}

// Ap = A p ; wApA = sum Ap.p ; alpha = wArA / wApA (k_pcg_spmv on the box layout).  Rows of a chunk
// are taken four consecutive rows per thread (the mapping of k_pcg_spmv, so both products add the
// same partial sums); with the range form and H % 4 == 0 interior groups take the vector path.
template <class T, int FLAG, bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta) k_box_pcg_spmv(const Chunk* __restrict__ ch, BoxRows R,
                                                              const T* __restrict__ coef, int nrows,
                                                              const T* __restrict__ diag, const T* __restrict__ p,
                                                              T* __restrict__ Ap, RedCtx Rc, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    const BoxSys B = R.ch == nullptr ? R.one : box_load(R.boxes, c.sys);
    const T* cx = coef;
    const T* cy = coef + nrows;
    const T* cz = coef + 2 * size_t(nrows);
    const int row0 = c.start + 4 * int(threadIdx.x);
    const bool vec = R.ch == nullptr && B.H % 4 == 0 && row0 + 3 < c.start + c.count;
    BoxGroup4<T> G;
    G.valid = false;
    if (vec) G.load(B, row0, cx, cy, cz, diag);
    pdl_wait();
    if (sys_idle(st[c.sys], FLAG)) return;
    auto xf = [&](int j) -> T { return __ldg(p + j); };
    BlockSum<1, EXACT> acc;
    acc.begin();
    if (G.valid) {
        const V4<T> pv = ld4(p + row0);
        T s[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) s[v] = G.dg.v[v] * pv.v[v];
        auto xv4 = [&](int j) { return ld4(p + j); };
        if (B.nz > 1)
            G.template accumulate<false, true>(xv4, xf, s);
        else
            G.template accumulate<false, false>(xv4, xf, s);
        st4(Ap + row0, s);
#pragma unroll
        for (int v = 0; v < 4; ++v) acc.add(0, (double)s[v] * (double)pv.v[v]);
    } else {
        for (int v = 0; v < 4; ++v) {
            const int row = row0 + v;
            if (row >= c.start + c.count) break;
            const T pr = p[row];
            BoxRowPre<T> pre;
            pre.load(B, row, cx, cy, cz);
            const T y = pre.template accumulate<false>(xf, ld_keep(diag + row, l2_keep()) * pr);
            Ap[row] = y;
            acc.add(0, (double)y * (double)pr);
        }
    }
    double out[1];
    if (acc.finish(c, Rc, out)) {
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

// k_box_pcg_spmv for a single box system with H % 4 == 0 (every group of four slots takes the
// vector path): no per-row fallback, so FP64 fits three resident CTAs per SM instead of two (the
// exact-sum form, with its larger accumulator, keeps two).
template <class T, int FLAG, bool EXACT>
__global__ void __launch_bounds__(kRowsPerCta, sizeof(T) == 8 ? (EXACT ? 2 : 3) : 4) k_box_pcg_spmv4(
    const Chunk* __restrict__ ch, BoxSys B, const T* __restrict__ coef, int nrows, const T* __restrict__ diag,
    const T* __restrict__ p, T* __restrict__ Ap, RedCtx Rc, SysState* st) {
    pdl_launch();
    const Chunk c = ch[blockIdx.x];
    const int row0 = c.start + 4 * int(threadIdx.x);
    const bool has = row0 < c.start + c.count;
    BoxGroup4<T> G;
    G.valid = false;
    if (has) G.load(B, row0, coef, coef + nrows, coef + 2 * size_t(nrows), diag);
    pdl_wait();
    if (sys_idle(st[c.sys], FLAG)) return;
    BlockSum<1, EXACT> acc;
    acc.begin();
    if (has) {
        const V4<T> pv = ld4(p + row0);
        T s[4];
        if (G.valid) {
#pragma unroll
            for (int v = 0; v < 4; ++v) s[v] = G.dg.v[v] * pv.v[v];
            auto xv4 = [&](int j) { return ld4(p + j); };
            auto xf = [&](int j) -> T { return __ldg(p + j); };
            if (B.nz > 1)
                G.template accumulate<false, true>(xv4, xf, s);
            else
                G.template accumulate<false, false>(xv4, xf, s);
        } else {
            // padding slots past the colour group's cells: a diagonal-only row
            const V4<T> dg = ld4(diag + row0);
#pragma unroll
            for (int v = 0; v < 4; ++v) s[v] = dg.v[v] * pv.v[v];
        }
        st4(Ap + row0, s);
#pragma unroll
        for (int v = 0; v < 4; ++v) acc.add(0, (double)s[v] * (double)pv.v[v]);
    }
    double out[1];
    if (acc.finish(c, Rc, out)) {
        SysState& q = st[c.sys];
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
