// Finite-volume assembly of the pressure equation on the device.
//
// Every kernel is a gather: one thread per cell walks the cell's faces in ascending face order
// (the order in which the reference's face loops update that cell), or one thread per face.
// With -fmad=false the results equal the reference's face-loop scatters bit for bit; nothing
// is accumulated with atomics.
#include <algorithm>
#include <cmath>

#include "assembly.h"

namespace vlm {

namespace {

inline int nblk(int n, int t = 256) { return (n + t - 1) / t; }

struct V3 {
    double x, y, z;
};

__device__ __forceinline__ V3 ld3(const double* soa, int n, int i) { return V3{soa[i], soa[n + i], soa[2 * n + i]}; }
__device__ __forceinline__ double dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Boundary constraint of the least-squares gradient (Fvc.h:267-287): value BCs use d and
// phi_b - phi_P, gradient BCs n (n.d) and g_b (n.d) with n.d >= 0.05|d|.
struct BFace {
    V3 de;
    bool value;
    double nd;  // max(n.d, 0.05|d|) of a gradient constraint
};

__device__ __forceinline__ BFace lsBoundary(const double* Sf, const double* magSf, const double* d, int nF, int f,
                                            bool value) {
    const V3 dd = ld3(d, nF, f);
    if (value) return BFace{dd, true, 0.0};
    const double inv = 1.0 / magSf[f];
    const V3 n{Sf[f] * inv, Sf[nF + f] * inv, Sf[2 * nF + f] * inv};
    const double nd = fmax(dot3(n, dd), 0.05 * sqrt(dot3(dd, dd)));
    return BFace{V3{n.x * nd, n.y * nd, n.z * nd}, false, nd};
}

// The least-squares constraint kind of a boundary face: a value constraint where the patch's
// condition fixes the value (lsFix per patch when given, else fixedValue), else a normal-gradient one
__device__ __forceinline__ bool lsValue(const int32_t* bcType, const int32_t* lsFix, const double* robin, int p) {
    return lsFix ? lsFix[p] != 0 : (bcType[p] == 1 || (bcType[p] == 8 && robin[2 * p] != 0.0));
}

// Robin a phi + b dphi/dn = c (RobinBC, BoundaryCondition.h:166-192): the gradient coefficients
// gic = dc (b dc / (a + b dc) - 1), gbc = dc (c / (a + b dc)), the face value (c + b dc phi_P) / (a + b dc)
__device__ __forceinline__ void robinGradient(const double* ab, double c, double dc, double& gic, double& gbc) {
    const double a = ab[0], b = ab[1];
    gic = dc * (b * dc / (a + b * dc) - 1.0);
    gbc = dc * (c / (a + b * dc));
}
__device__ __forceinline__ double robinValue(const double* ab, double c, double dc, double psiP) {
    const double bd = ab[1] * dc;
    return (c + bd * psiP) / (ab[0] + bd);
}

// (gic psi_P + gbc) of a gradient-constrained face (Fvc.h:283-284): zeroGradient / symmetry 0, 0;
// mixed -w dc, w dc v (refGrad 0); fixedGradient 0, g; Robin (rob = the patch's {a, b})
__device__ __forceinline__ double lsBoundaryGradient(int t, double psiP, double v, double w, double dc,
                                                     const double* rob) {
    double gic = 0.0, gbc = 0.0;
    if (t == 4) {
        gic = -w * dc;
        gbc = w * dc * v + (1.0 - w) * 0.0;
    } else if (t == 5) {
        gbc = v;
    } else if (t == 8) {
        robinGradient(rob, v, dc, gic, gbc);
    }
    return gic * psiP + gbc;
}

// ---------------------------------------------------------------- kernels
// gs = gamma |S|; upper = gamma |S| ndc  (Fvm.h:150, :176)
__global__ void k_face_gs(int nF, int nI, const double* __restrict__ gamma, const double* __restrict__ magSf,
                          const double* __restrict__ ndc, double* __restrict__ gs, double* __restrict__ upper) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const double g = gamma[f] * magSf[f];
    gs[f] = g;
    if (f < nI) upper[f] = g * ndc[f];
}

// boundary coefficients of the laplacian (Fvm.h:171-180): fixedValue (gic -dc, gbc dc v), mixed
// (MixedBC, BoundaryCondition.h:240-243: -w dc, w dc v + (1 - w) g with g = 0), fixedGradient
// (BoundaryCondition.h:147-148: 0, g), zeroGradient (0, 0)
__global__ void k_lap_boundary(int nB, int nI, const double* __restrict__ gs, const double* __restrict__ ndc,
                               const int32_t* __restrict__ bPatch, const int32_t* __restrict__ bcType,
                               const double* __restrict__ bcValue, const double* __restrict__ frac, const double* __restrict__ robin,
                               double* __restrict__ ic, double* __restrict__ bs) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB) return;
    const int f = nI + b;
    double gic = 0.0, gbc = 0.0;
    const int t = bcType[bPatch[b]];
    const double v = bcValue ? bcValue[b] : 0.0;
    if (t == 1) {
        gic = -ndc[f];
        gbc = ndc[f] * v;
    } else if (t == 4) {
        const double w = frac[b], dc = ndc[f];
        gic = -w * dc;
        gbc = w * dc * v + (1.0 - w) * 0.0;
    } else if (t == 5) {
        gbc = v;
    } else if (t == 8) {
        robinGradient(robin + 2 * bPatch[b], v, ndc[f], gic, gbc);
    }
    ic[b] = 0.0 + gs[f] * gic;
    bs[b] = 0.0 - gs[f] * gbc;
}

// GaussSkew gradient (Fvc.h:233-262): Gauss with the face values w psi_P + (1-w) psi_N + (x_f - x'_f).
// (w gls_P + (1-w) gls_N) on internal faces; on boundary faces the boundary value where the condition
// fixes it, else psi_P + dt.gls_P + gb (n.d) with n.d unclipped, dt = d - n (n.d), gb = gic psi_P + gbc;
// gls: the least-squares gradient (3 per cell)
__global__ void k_grad_gauss_skew(int nC, int nI, int nF, const int32_t* __restrict__ cfOff,
                                  const int32_t* __restrict__ cf, const int32_t* __restrict__ own,
                                  const int32_t* __restrict__ nei, const double* __restrict__ w,
                                  const double* __restrict__ Sf, const double* __restrict__ magSf,
                                  const double* __restrict__ d, const double* __restrict__ V,
                                  const double* __restrict__ skew, const double* __restrict__ ndc,
                                  const double* __restrict__ psi, const double* __restrict__ psiB,
                                  const double* __restrict__ gls, const int32_t* __restrict__ bPatch,
                                  const int32_t* __restrict__ bcType, const int32_t* __restrict__ lsFix,
                                  const double* __restrict__ bcValue, const double* __restrict__ frac, const double* __restrict__ robin, int twoD,
                                  int emptyDir, double* __restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = (int)(e & 0x7fffffffu);
        double phif;
        if (f < nI) {
            const int o = own[f], n = nei[f];
            const double wf = w[f], wn = 1.0 - wf;
            double gf[3];
            for (int q = 0; q < 3; ++q) gf[q] = wf * gls[3 * o + q] + wn * gls[3 * n + q];
            const double sk = skew[f] * gf[0] + skew[nF + f] * gf[1] + skew[2 * nF + f] * gf[2];
            phif = (wf * psi[o] + wn * psi[n]) + sk;
        } else {
            const int b = f - nI, p = bPatch[b], o = own[f];
            if (lsValue(bcType, lsFix, robin, p)) {
                phif = psiB[b];
            } else {
                const double inv = 1.0 / magSf[f];
                const V3 n{Sf[f] * inv, Sf[nF + f] * inv, Sf[2 * nF + f] * inv};
                const V3 dd = ld3(d, nF, f);
                const double nd = dot3(n, dd);
                const V3 dt{dd.x - n.x * nd, dd.y - n.y * nd, dd.z - n.z * nd};
                const int t = bcType[p];
                const double gb =
                    lsBoundaryGradient(t, psi[o], bcValue ? bcValue[b] : 0.0, t == 4 ? frac[b] : 0.0, ndc[f],
                                       robin ? robin + 2 * p : nullptr);
                const double tg = dt.x * gls[3 * o] + dt.y * gls[3 * o + 1] + dt.z * gls[3 * o + 2];
                phif = (psi[o] + tg) + gb * nd;
            }
        }
        const double cx = Sf[f] * phif, cy = Sf[nF + f] * phif, cz = Sf[2 * nF + f] * phif;
        if (e >> 31) {
            gx -= cx;
            gy -= cy;
            gz -= cz;
        } else {
            gx += cx;
            gy += cy;
            gz += cz;
        }
    }
    const double iv = 1.0 / V[c];
    gx = gx * iv;
    gy = gy * iv;
    gz = gz * iv;
    if (twoD) {
        if (emptyDir == 0) gx = 0.0;
        if (emptyDir == 1) gy = 0.0;
        if (emptyDir == 2) gz = 0.0;
    }
    g[3 * c] = gx;
    g[3 * c + 1] = gy;
    g[3 * c + 2] = gz;
}

// diag[c] = -Σ upper; source[c] = Σ ∓ffc (Fvm.h:149-168), cell faces in ascending order
__global__ void k_lap_cells(int nC, int nI, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                            const double* __restrict__ upper, const double* __restrict__ ffc, double* __restrict__ diag,
                            double* __restrict__ source) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double dg = 0.0, src = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = (int)(e & 0x7fffffffu);
        if (f >= nI) continue;
        dg -= upper[f];
        if (ffc) {
            if (e >> 31)
                src += ffc[f];
            else
                src -= ffc[f];
        }
    }
    diag[c] = dg;
    source[c] = src;
}

// Gauss linear gradient (Fvc.h:216-225)
__global__ void k_grad_gauss(int nC, int nI, int nF, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                             const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                             const double* __restrict__ w, const double* __restrict__ Sf, const double* __restrict__ V,
                             const double* __restrict__ psi, const double* __restrict__ psiB, int twoD, int emptyDir,
                             double* __restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = (int)(e & 0x7fffffffu);
        double phif;
        if (f < nI)
            phif = w[f] * psi[own[f]] + (1.0 - w[f]) * psi[nei[f]];
        else
            phif = psiB[f - nI];
        const double cx = Sf[f] * phif, cy = Sf[nF + f] * phif, cz = Sf[2 * nF + f] * phif;
        if (e >> 31) {
            gx -= cx;
            gy -= cy;
            gz -= cz;
        } else {
            gx += cx;
            gy += cy;
            gz += cz;
        }
    }
    const double iv = 1.0 / V[c];
    gx = gx * iv;
    gy = gy * iv;
    gz = gz * iv;
    if (twoD) {  // finishGrad (Fvc.h:169-181)
        if (emptyDir == 0) gx = 0.0;
        if (emptyDir == 1) gy = 0.0;
        if (emptyDir == 2) gz = 0.0;
    }
    g[3 * c] = gx;
    g[3 * c + 1] = gy;
    g[3 * c + 2] = gz;
}

// weighted least-squares gradient (Fvc.h:135-167 with the field boundary constraints :267-287)
__global__ void k_grad_ls(int nC, int nI, int nF, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                          const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                          const double* __restrict__ Sf, const double* __restrict__ magSf, const double* __restrict__ d,
                          const double* __restrict__ ndc, const double* __restrict__ psi,
                          const double* __restrict__ psiB, const int32_t* __restrict__ bPatch,
                          const int32_t* __restrict__ bcType, const int32_t* __restrict__ lsFix,
                          const double* __restrict__ bcValue, const double* __restrict__ frac, const double* __restrict__ robin, int twoD,
                          int emptyDir, double* __restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = (int)((uint32_t)cf[k] & 0x7fffffffu);
        V3 v;
        if (f < nI)
            v = ld3(d, nF, f);
        else
            v = lsBoundary(Sf, magSf, d, nF, f, lsValue(bcType, lsFix, robin, bPatch[f - nI])).de;
        const double s = 1.0 / dot3(v, v);
        const double o[9] = {v.x * v.x, v.x * v.y, v.x * v.z, v.y * v.x, v.y * v.y, v.y * v.z,
                             v.z * v.x, v.z * v.y, v.z * v.z};
#pragma unroll
        for (int q = 0; q < 9; ++q) a[q] += o[q] * s;
    }
    if (twoD) a[4 * emptyDir] += 1.0;
    // detail::inv (Fvc.h:112-126)
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    double G[9];
    G[0] = (a[4] * a[8] - a[5] * a[7]) / det;
    G[1] = (a[2] * a[7] - a[1] * a[8]) / det;
    G[2] = (a[1] * a[5] - a[2] * a[4]) / det;
    G[3] = (a[5] * a[6] - a[3] * a[8]) / det;
    G[4] = (a[0] * a[8] - a[2] * a[6]) / det;
    G[5] = (a[2] * a[3] - a[0] * a[5]) / det;
    G[6] = (a[3] * a[7] - a[4] * a[6]) / det;
    G[7] = (a[1] * a[6] - a[0] * a[7]) / det;
    G[8] = (a[0] * a[4] - a[1] * a[3]) / det;
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = (int)((uint32_t)cf[k] & 0x7fffffffu);
        V3 v;
        double dp;
        if (f < nI) {
            v = ld3(d, nF, f);
            dp = psi[nei[f]] - psi[own[f]];
        } else {
            const int b = f - nI, p = bPatch[b];
            const bool value = lsValue(bcType, lsFix, robin, p);
            const BFace bfc = lsBoundary(Sf, magSf, d, nF, f, value);
            v = bfc.de;
            if (value) {
                dp = psiB[b] - psi[own[f]];
            } else {
                const int t = bcType[p];
                dp = lsBoundaryGradient(t, psi[own[f]], bcValue ? bcValue[b] : 0.0, t == 4 ? frac[b] : 0.0, ndc[f],
                                        robin ? robin + 2 * p : nullptr) *
                     bfc.nd;
            }
        }
        const double wgt = 1.0 / dot3(v, v);
        const V3 dw{v.x * wgt, v.y * wgt, v.z * wgt};
        const V3 Gd{G[0] * dw.x + G[1] * dw.y + G[2] * dw.z, G[3] * dw.x + G[4] * dw.y + G[5] * dw.z,
                    G[6] * dw.x + G[7] * dw.y + G[8] * dw.z};
        gx += Gd.x * dp;
        gy += Gd.y * dp;
        gz += Gd.z * dp;
    }
    if (twoD) {
        if (emptyDir == 0) gx = 0.0;
        if (emptyDir == 1) gy = 0.0;
        if (emptyDir == 2) gz = 0.0;
    }
    g[3 * c] = gx;
    g[3 * c + 1] = gy;
    g[3 * c + 2] = gz;
}

// explicit non-orthogonal correction flux (Fvm.h:162-165)
__global__ void k_lap_ffc(int nI, int nF, const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                          const double* __restrict__ w, const double* __restrict__ corr, const double* __restrict__ gs,
                          const double* __restrict__ g, double* __restrict__ ffc) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    if (f >= nI) {
        ffc[f] = 0.0;
        return;
    }
    const int o = own[f], n = nei[f];
    const double wf = w[f], wn = 1.0 - wf;
    const double gx = wf * g[3 * o] + wn * g[3 * n];
    const double gy = wf * g[3 * o + 1] + wn * g[3 * n + 1];
    const double gz = wf * g[3 * o + 2] + wn * g[3 * n + 2];
    ffc[f] = gs[f] * (corr[f] * gx + corr[nF + f] * gy + corr[2 * nF + f] * gz);
}

__global__ void k_fold(int nC, int nI, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                       const double* __restrict__ diag, const double* __restrict__ source, const double* __restrict__ ic,
                       const double* __restrict__ bs, double* __restrict__ d, double* __restrict__ b) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double dd = diag[c], bb = source[c];
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = (int)((uint32_t)cf[k] & 0x7fffffffu);
        if (f < nI) continue;
        dd += ic[f - nI];
        bb += bs[f - nI];
    }
    d[c] = dd;
    b[c] = bb;
}

__global__ void k_flux(int nF, int nI, const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                       const double* __restrict__ upper, const double* __restrict__ psi, const double* __restrict__ ic,
                       const double* __restrict__ bs, const double* __restrict__ ffc, double* __restrict__ F) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    double v;
    if (f < nI)
        v = upper[f] * psi[nei[f]] - upper[f] * psi[own[f]];
    else
        v = ic[f - nI] * psi[own[f]] - bs[f - nI];
    if (ffc) v += ffc[f];
    F[f] = v;
}

__global__ void k_add_vol_source(int nC, double* __restrict__ source, const double* __restrict__ su,
                                 const double* __restrict__ V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nC) source[c] += su[c] * V[c];
}

__global__ void k_div(int nC, int nI, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                      const double* __restrict__ F, const double* __restrict__ V, double* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double r = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = (int)(e & 0x7fffffffu);
        if (f < nI && (e >> 31))
            r -= F[f];
        else
            r += F[f];
    }
    out[c] = r / V[c];
}

__global__ void k_set_reference(int cell, double value, double* diag, double* source) {
    source[cell] += diag[cell] * value;
    diag[cell] += diag[cell];
}

__global__ void k_set_references(const int32_t* __restrict__ cells, int n, double value, double* diag,
                                 double* source) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int c = cells[q];
    source[c] += diag[c] * value;
    diag[c] += diag[c];
}

__global__ void k_correct_bc(int nB, int nI, const int32_t* __restrict__ own, const int32_t* __restrict__ bPatch,
                             const int32_t* __restrict__ bcType, const double* __restrict__ bcValue,
                             const double* __restrict__ frac, const double* __restrict__ robin, const double* __restrict__ ndc,
                             const double* __restrict__ psi, double* __restrict__ psiB) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB) return;
    const int t = bcType[bPatch[b]];
    const double v = bcValue ? bcValue[b] : 0.0;
    const double pP = psi[own[nI + b]];
    if (t == 1)
        psiB[b] = v;
    else if (t == 4)  // MixedBC::evaluate (BoundaryCondition.h:232-235), refGrad 0
        psiB[b] = frac[b] * v + (1.0 - frac[b]) * (pP + 0.0 / ndc[nI + b]);
    else if (t == 5)  // FixedGradientBC::evaluate (VolField.h:144-146)
        psiB[b] = pP + v / ndc[nI + b];
    else if (t == 8)  // RobinBC::evaluate (VolField.h:148-153)
        psiB[b] = robinValue(robin + 2 * bPatch[b], v, ndc[nI + b], pP);
    else
        psiB[b] = pP;
}

}  // namespace

// ---------------------------------------------------------------- DeviceGeom
DeviceGeom::DeviceGeom(int nCells, int nInternal, int nFaces, const int32_t* own, const int32_t* nei,
                       const double* magSf, const double* ndc, const double* V, const double* Sf, const double* d,
                       const double* w, const double* corrVecs, int twoD, int emptyDir, int nPatches,
                       const int32_t* patchStart, const int32_t* patchSize, const double* C, const double* Cf,
                       const double* skewVecs, cudaStream_t s)
    : nC_(nCells), nI_(nInternal), nF_(nFaces), twoD_(twoD), emptyDir_(emptyDir) {
    VLM_REQUIRE(V && Sf && d && w && corrVecs, VLM_ERR_BAD_ARG, "mesh geometry (V, Sf, d, w, corrVecs) is required");
    const int nB = nF_ - nI_;
    // cell -> face list in ascending face order (the order of every reference face loop)
    std::vector<int32_t> off(size_t(nC_) + 1, 0), list;
    for (int f = 0; f < nF_; ++f) {
        off[own[f] + 1]++;
        if (f < nI_) off[nei[f] + 1]++;
    }
    for (int c = 0; c < nC_; ++c) off[c + 1] += off[c];
    list.resize(size_t(off[nC_]));
    std::vector<int32_t> pos(off.begin(), off.end() - 1);
    for (int f = 0; f < nF_; ++f) {
        list[pos[own[f]]++] = f;
        if (f < nI_) list[pos[nei[f]]++] = int32_t(uint32_t(f) | 0x80000000u);
    }
    cfOff_.upload(off, s);
    cfList_.upload(list, s);
    // boundary face -> patch
    bPatchHost_.assign(size_t(std::max(nB, 1)), 0);
    for (int p = 0; p < nPatches; ++p) {
        patchStart_.push_back(patchStart[p]);
        patchSize_.push_back(patchSize[p]);
        for (int i = 0; i < patchSize[p]; ++i) {
            const int b = patchStart[p] + i - nI_;
            VLM_REQUIRE(b >= 0 && b < nB, VLM_ERR_BAD_ARG, "patch face range outside the boundary faces");
            bPatchHost_[b] = p;
        }
    }
    bPatch_.upload(bPatchHost_, s);
    own_.upload(own, size_t(nF_), s);
    nei_.upload(nei, size_t(std::max(nI_, 1)) * (nI_ > 0), s);
    if (nI_ == 0) nei_.resize(1);
    magSf_.upload(magSf, size_t(nF_), s);
    ndc_.upload(ndc, size_t(nF_), s);
    V_.upload(V, size_t(nC_), s);
    w_.upload(w, size_t(nF_), s);
    auto soa = [&](const double* aos, DBuf<double>& out) {
        std::vector<double> v(size_t(3) * nF_);
        for (int f = 0; f < nF_; ++f)
            for (int q = 0; q < 3; ++q) v[size_t(q) * nF_ + f] = aos[3 * size_t(f) + q];
        out.upload(v, s);
    };
    soa(Sf, Sf_);
    soa(d, d_);
    soa(corrVecs, corr_);
    if (C && Cf) {
        soa(Cf, Cf_);
        std::vector<double> v(size_t(3) * nC_);
        for (int c = 0; c < nC_; ++c)
            for (int q = 0; q < 3; ++q) v[size_t(q) * nC_ + c] = C[3 * size_t(c) + q];
        C_.upload(v, s);
    }
    // Mesh::skewed (Mesh.cpp:596, 617-621): max |x_f - x'_f| / |d| over internal faces above 1e-8
    if (skewVecs) {
        double skewMax = 0.0;
        for (int f = 0; f < nI_; ++f) {
            const double* k = skewVecs + 3 * size_t(f);
            const double* dd = d + 3 * size_t(f);
            const double sk = std::sqrt(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]) /
                              std::sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
            skewMax = std::max(skewMax, sk);
        }
        skewed_ = skewMax > 1e-8;
        soa(skewVecs, skew_);  // kept on unskewed meshes too: the GaussSkew gradient reads them
    }
    // the correction is applied when any internal corrVec is non-zero (Fvm.h:156-158)
    for (int f = 0; f < nI_ && !nonOrth_; ++f) {
        const double* c = corrVecs + 3 * size_t(f);
        nonOrth_ = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] > 1e-20;
    }
    scratchG_.resize(size_t(3) * nC_);
    scratchGS_.resize(size_t(nF_));
    bcType_.resize(size_t(std::max(nPatches, 1)));
    VLM_CUDA(cudaStreamSynchronize(s));
}

// The device copy of the patch types is refreshed only when they change (a host-to-device copy
// from pageable memory waits for the stream, which would stall every assembly call).
void DeviceGeom::uploadBCType(const ScalarBC& bc, cudaStream_t s) {
    std::vector<int32_t> t(bcType_.size(), 0);
    for (size_t p = 0; p < patchStart_.size(); ++p) {
        t[p] = bc.type ? bc.type[p] : 0;
        VLM_REQUIRE(t[p] == 0 || t[p] == 1 || t[p] == 2 || t[p] == 4 || t[p] == 5 || (t[p] == 8 && bc.robin),
                    VLM_ERR_BAD_ARG,
                    "scalar boundary type must be 0 zeroGradient, 1 fixedValue, 2 symmetry, 4 mixed or 5 fixedGradient "
                    "(8 Robin inside a flow, which carries its coefficients)");
        VLM_REQUIRE(t[p] != 4 || bc.frac != nullptr, VLM_ERR_BAD_ARG, "a mixed boundary needs its value fractions");
    }
    if (t == bcTypeHost_) return;
    VLM_CUDA(cudaMemcpyAsync(bcType_.get(), t.data(), sizeof(int32_t) * t.size(), cudaMemcpyHostToDevice, s));
    VLM_CUDA(cudaStreamSynchronize(s));  // t is a local
    bcTypeHost_ = std::move(t);
}

void DeviceGeom::correctBoundary(const double* psi, const ScalarBC& bc, double* psiB, cudaStream_t s) {
    uploadBCType(bc, s);
    const int nB = nBoundary();
    if (nB > 0)
        k_correct_bc<<<nblk(nB), 256, 0, s>>>(nB, nI_, own_.get(), bPatch_.get(), bcType_.get(), bc.value, bc.frac, bc.robin,
                                              ndc_.get(), psi, psiB), ++launches_;
}

void DeviceGeom::grad(const double* psi, const double* psiB, const ScalarBC& bc, int scheme, double* out,
                      cudaStream_t s) {
    uploadBCType(bc, s);
    if (scheme == 2) {
        VLM_REQUIRE(skew_.size() > 0, VLM_ERR_BAD_ARG, "the GaussSkew gradient needs the mesh's skew vectors");
        scratchGls_.resize(size_t(3) * nC_);
        k_grad_ls<<<nblk(nC_), 256, 0, s>>>(nC_, nI_, nF_, cfOff_.get(), cfList_.get(), own_.get(), nei_.get(),
                                            Sf_.get(), magSf_.get(), d_.get(), ndc_.get(), psi, psiB, bPatch_.get(),
                                            bcType_.get(), bc.lsFix, bc.value, bc.frac, bc.robin, twoD_, emptyDir_,
                                            scratchGls_.get()), ++launches_;
        k_grad_gauss_skew<<<nblk(nC_), 256, 0, s>>>(nC_, nI_, nF_, cfOff_.get(), cfList_.get(), own_.get(), nei_.get(),
                                                    w_.get(), Sf_.get(), magSf_.get(), d_.get(), V_.get(), skew_.get(),
                                                    ndc_.get(), psi, psiB, scratchGls_.get(), bPatch_.get(),
                                                    bcType_.get(), bc.lsFix, bc.value, bc.frac, bc.robin, twoD_, emptyDir_, out),
            ++launches_;
    } else if (scheme == 1)
        k_grad_ls<<<nblk(nC_), 256, 0, s>>>(nC_, nI_, nF_, cfOff_.get(), cfList_.get(), own_.get(), nei_.get(),
                                            Sf_.get(), magSf_.get(), d_.get(), ndc_.get(), psi, psiB, bPatch_.get(),
                                            bcType_.get(), bc.lsFix, bc.value, bc.frac, bc.robin, twoD_, emptyDir_, out),
            ++launches_;
    else
        k_grad_gauss<<<nblk(nC_), 256, 0, s>>>(nC_, nI_, nF_, cfOff_.get(), cfList_.get(), own_.get(), nei_.get(),
                                               w_.get(), Sf_.get(), V_.get(), psi, psiB, twoD_, emptyDir_, out), ++launches_;
}

void DeviceGeom::laplacian(const double* gamma, const double* psi, const double* psiB, const ScalarBC& bc,
                           bool nonOrthCorr, int gradScheme, double* diag, double* upper, double* source, double* ic,
                           double* bs, double* ffc, bool* hasFfc, cudaStream_t s) {
    uploadBCType(bc, s);
    double* gs = scratchGS_.get();
    k_face_gs<<<nblk(nF_), 256, 0, s>>>(nF_, nI_, gamma, magSf_.get(), ndc_.get(), gs, upper), ++launches_;
    const bool corr = nonOrthCorr && nonOrth_;
    if (corr) {
        grad(psi, psiB, bc, gradScheme, scratchG_.get(), s);
        k_lap_ffc<<<nblk(nF_), 256, 0, s>>>(nI_, nF_, own_.get(), nei_.get(), w_.get(), corr_.get(), gs,
                                            scratchG_.get(), ffc), ++launches_;
    }
    k_lap_cells<<<nblk(nC_), 256, 0, s>>>(nC_, nI_, cfOff_.get(), cfList_.get(), upper, corr ? ffc : nullptr, diag,
                                          source), ++launches_;
    const int nB = nBoundary();
    if (nB > 0)
        k_lap_boundary<<<nblk(nB), 256, 0, s>>>(nB, nI_, gs, ndc_.get(), bPatch_.get(), bcType_.get(), bc.value,
                                                bc.frac, bc.robin, ic, bs), ++launches_;
    if (hasFfc) *hasFfc = corr;
}

void DeviceGeom::fold(const double* diag, const double* source, const double* ic, const double* bs, double* d,
                      double* b, cudaStream_t s) {
    k_fold<<<nblk(nC_), 256, 0, s>>>(nC_, nI_, cfOff_.get(), cfList_.get(), diag, source, ic, bs, d, b), ++launches_;
}

void DeviceGeom::flux(const double* upper, const double* psi, const double* ic, const double* bs, const double* ffc,
                      double* F, cudaStream_t s) {
    k_flux<<<nblk(nF_), 256, 0, s>>>(nF_, nI_, own_.get(), nei_.get(), upper, psi, ic, bs, ffc, F), ++launches_;
}

void DeviceGeom::addVolumeSource(double* source, const double* su, cudaStream_t s) {
    k_add_vol_source<<<nblk(nC_), 256, 0, s>>>(nC_, source, su, V_.get()), ++launches_;
}

void DeviceGeom::div(const double* F, double* out, cudaStream_t s) {
    k_div<<<nblk(nC_), 256, 0, s>>>(nC_, nI_, cfOff_.get(), cfList_.get(), F, V_.get(), out), ++launches_;
}

void DeviceGeom::setReference(int cell, double value, double* diag, double* source, cudaStream_t s) {
    VLM_REQUIRE(cell >= 0 && cell < nC_, VLM_ERR_BAD_ARG, "reference cell out of range");
    k_set_reference<<<1, 1, 0, s>>>(cell, value, diag, source), ++launches_;
}

void DeviceGeom::setReferences(const int32_t* cells, int n, double value, double* diag, double* source,
                               cudaStream_t s) {
    if (n > 0) k_set_references<<<nblk(n), 256, 0, s>>>(cells, n, value, diag, source), ++launches_;
}

}  // namespace vlm
