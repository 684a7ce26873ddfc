// Device incompressible step (see flow.h).  Every kernel names the reference loop it restates;
// floating-point expressions keep the reference's operand order (the library is built with
// -fmad=false, so a*b+c rounds twice, as in the reference's -ffp-contract=off build).
#include "flow.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <map>
#include <string>

namespace vlm {
namespace {

inline int nblk(int64_t n, int b = 256) { return int((n + b - 1) / b); }

enum : int { kUpwind = 0, kLinear = 1, kLinearUpwind = 2, kLUST = 3, kLimitedLinear = 4, kVanLeer = 5, kMUSCL = 6,
             kMinmod = 7 };

// the TVD limiters of detail::limiter (Fvm.h:63-72); std::min / std::max as the reference evaluates them
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double tvd_limiter(int scheme, double k, double r) {
    switch (scheme) {
    case kVanLeer: return (r + fabs(r)) / (1.0 + fabs(r));
    case kMinmod: return dmax(dmin(r, 1.0), 0.0);
    case kMUSCL: return dmax(dmin(dmin(2.0 * r, 0.5 * r + 0.5), 2.0), 0.0);
    case kLimitedLinear: return dmax(dmin(2.0 / dmax(k, 1.0e-15) * r, 1.0), 0.0);
    default: return 1.0;
    }
}

// ---------------------------------------------------------------- boundary values of U
// correctBoundaryConditions (VolField.h:96-103) for fixedValue (value) and zeroGradient (cell value)
// U boundary values (VolField::correctBoundaryConditions): fixedValue the value; zeroGradient the
// owner's; symmetry u - (n.u) n with n = S_f / |S_f| (SymmetryBC<Vec3>::evaluate, VolField.h:164-170)
__global__ void k_u_boundary(int nB, int nI, int nC, int nF, const int32_t* __restrict__ own,
                             const int32_t* __restrict__ bPatch, const int32_t* __restrict__ uType,
                             const double* __restrict__ uValueB, const double* __restrict__ Sf,
                             const double* __restrict__ magSf, const double* __restrict__ ndc,
                             const double* __restrict__ wIO, const double* __restrict__ phi,
                             const double* __restrict__ uRobin, const double* __restrict__ U,
                             double* __restrict__ Ub) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB) return;
    const int q = bPatch[b];
    const int c = own[nI + b];
    if (uType[q] == 8) {
        // RobinBC<Vec3>::evaluate (VolField.h:148-153): (c + b dc U_P) / (a + b dc)
        const double bd = uRobin[2 * q + 1] * ndc[nI + b];
        for (int k = 0; k < 3; ++k) Ub[k * nB + b] = (uValueB[k * nB + b] + bd * U[k * nC + c]) / (uRobin[2 * q] + bd);
        return;
    }
    if (uType[q] == 3 || uType[q] == 4 || uType[q] == 9) {
        // inletOutlet / freestream / advective = mixed with refGrad 0 (MixedBC::evaluate, BoundaryCondition.h:232-235)
        const double w = wIO[b], dc = ndc[nI + b];
        for (int k = 0; k < 3; ++k)
            Ub[k * nB + b] = w * uValueB[k * nB + b] + (1.0 - w) * (U[k * nC + c] + 0.0 / dc);
        return;
    }
    if (uType[q] == 6) {
        // pressureInletOutletVelocity (VolField.h:204-212): outflow zero gradient; inflow the normal
        // component of U_P and the tangential part of Ut; the current flux decides
        double u[3];
        for (int k = 0; k < 3; ++k) u[k] = U[k * nC + c];
        if (phi[nI + b] >= 0) {
            for (int k = 0; k < 3; ++k) Ub[k * nB + b] = u[k];
            return;
        }
        const int f = nI + b;
        const double A = magSf[f];
        const double n[3] = {Sf[f] / A, Sf[nF + f] / A, Sf[2 * size_t(nF) + f] / A};
        const double ut[3] = {uValueB[b], uValueB[size_t(nB) + b], uValueB[2 * size_t(nB) + b]};
        const double nu_ = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
        const double nt = n[0] * ut[0] + n[1] * ut[1] + n[2] * ut[2];
        for (int k = 0; k < 3; ++k) Ub[k * nB + b] = nu_ * n[k] + (ut[k] - nt * n[k]);
        return;
    }
    if (uType[q] == 5) {  // fixedGradient (VolField.h:144-146): U_P + g / dc
        const double dc = ndc[nI + b];
        for (int k = 0; k < 3; ++k) Ub[k * nB + b] = U[k * nC + c] + uValueB[k * nB + b] / dc;
        return;
    }
    if (uType[q] == 2) {
        const int f = nI + b;
        const double A = magSf[f];
        const double n[3] = {Sf[f] / A, Sf[nF + f] / A, Sf[2 * size_t(nF) + f] / A};
        const double u[3] = {U[c], U[size_t(nC) + c], U[2 * size_t(nC) + c]};
        const double dnu = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
        for (int k = 0; k < 3; ++k) Ub[k * nB + b] = u[k] - dnu * n[k];
        return;
    }
    for (int k = 0; k < 3; ++k) Ub[k * nB + b] = uType[q] == 1 ? uValueB[k * nB + b] : U[k * nC + c];
}

// freestream value fractions (constant): U w = clamp(1/2 - (U_inf.n)/(2|U_inf|), 0, 1)
// (FreestreamVelocityBC, BoundaryCondition.h:291-302) and, on the same patch, p w = clamp(1/2 +
// (U_inf.n)/(2|U_inf|), 0, 1) (FreestreamPressureBC::setDirection, BoundaryCondition.h:316-320)
__global__ void k_freestream_fractions(int nB, int nI, int nF, const int32_t* __restrict__ bPatch,
                                       const int32_t* __restrict__ uType, const int32_t* __restrict__ pType,
                                       const double* __restrict__ uValueB, const double* __restrict__ Sf,
                                       const double* __restrict__ magSf, double* __restrict__ wU,
                                       double* __restrict__ wP) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB) return;
    const int q = bPatch[b];
    if (uType[q] != 4) return;
    const int f = nI + b;
    const double A = magSf[f];
    const double n[3] = {Sf[f] / A, Sf[nF + f] / A, Sf[2 * size_t(nF) + f] / A};
    const double u[3] = {uValueB[b], uValueB[size_t(nB) + b], uValueB[2 * size_t(nB) + b]};
    const double mu = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    const double un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
    auto clamp01 = [](double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); };
    wU[b] = mu > 0 ? clamp01(0.5 - 0.5 * un / mu) : 1.0;
    if (pType[q] == 4) wP[b] = mu > 0 ? clamp01(0.5 + 0.5 * un / mu) : 1.0;
}

// inletOutlet value fractions at the start of a step (InletOutletBC::update, BoundaryCondition.h:277-282):
// 1 where the face flux is inflow (phi < 0), else 0; phi == NULL (no flux yet) gives 0
__global__ void k_io_fraction(int nB, int nI, const int32_t* __restrict__ bPatch, const int32_t* __restrict__ uType,
                              const double* __restrict__ phi, double* __restrict__ wIO) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nB && uType[bPatch[b]] == 3) wIO[b] = phi && phi[nI + b] < 0 ? 1.0 : 0.0;
}

// advective outflow (AdvectiveBC::update, VolField.h:235-264).  On a new time
// index the current boundary values become the old level (and the old one the old-old level when
// shiftOldOld); fromZero takes zeros instead (a freshly constructed field, whose boundary values are 0).
// Then w = c / (c + max(phi/|S|, 0) dc) and refValue = (c0 U_b^0 - c00 U_b^00) / c with the step's ddt
// coefficients; phi == nullptr is a zero flux.  The face evaluates as a mixed condition with refGrad 0.
__global__ void k_adv_update(int nB, int nI, const int32_t* __restrict__ bPatch, const int32_t* __restrict__ uType,
                             const double* __restrict__ phi, const double* __restrict__ magSf,
                             const double* __restrict__ ndc, const double* __restrict__ Ub, double* __restrict__ old,
                             double* __restrict__ oldOld, const double* __restrict__ adv, int shift,
                             int shiftOldOld, int fromZero, double c, double c0, double c00,
                             double* __restrict__ wIO, double* __restrict__ uValueB) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB || uType[bPatch[b]] != 9) return;
    if (shift)
        for (int k = 0; k < 3; ++k) {
            const size_t e = size_t(k) * nB + b;
            if (shiftOldOld) oldOld[e] = old[e];
            old[e] = fromZero ? 0.0 : Ub[e];
        }
    const int f = nI + b;
    const double un = phi ? fmax(phi[f] / magSf[f], 0.0) : 0.0;
    const double a = un * ndc[f];
    const double* inf = adv + 4 * bPatch[b];
    if (inf[0] > 0.0) {
        // relaxation towards the far field: + (U_n / lInf)(U_b - fieldInf)
        const double kk = un / inf[0];
        for (int k = 0; k < 3; ++k) {
            const size_t e = size_t(k) * nB + b;
            uValueB[e] = ((c0 * old[e] - c00 * oldOld[e]) + kk * inf[1 + k]) / (c + kk);
        }
        wIO[b] = (c + kk) / (c + a + kk);
    } else {
        for (int k = 0; k < 3; ++k) {
            const size_t e = size_t(k) * nB + b;
            uValueB[e] = (c0 * old[e] - c00 * oldOld[e]) / c;
        }
        wIO[b] = c / (c + a);
    }
}

// steady (or no positive time step): zero gradient
__global__ void k_adv_steady(int nB, const int32_t* __restrict__ bPatch, const int32_t* __restrict__ uType,
                             double* __restrict__ wIO) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nB && uType[bPatch[b]] == 9) wIO[b] = 0.0;
}

// ---------------------------------------------------------------- fvc::grad of U (Gauss linear)
// Fvc.h:214-225 + finishGrad (Fvc.h:169-181): G_ij = sum S_i phi_j / V, row `emptyDir` zero in 2D.
// Output SoA: component (3i + j) at [(3i + j) * nC + c].
__global__ void k_grad_tensor(int nC, int nI, int nB, int nF, const int32_t* __restrict__ cfOff,
                              const int32_t* __restrict__ cf, const int32_t* __restrict__ own,
                              const int32_t* __restrict__ nei, const double* __restrict__ w,
                              const double* __restrict__ Sf, const double* __restrict__ V,
                              const double* __restrict__ U, const double* __restrict__ Ub, int twoD, int emptyDir,
                              double* __restrict__ G) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double g[9];
    for (int m = 0; m < 9; ++m) g[m] = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = int(e & 0x7fffffffu);
        double phif[3];
        if (f < nI) {
            const double wf = w[f], wn = 1.0 - wf;
            for (int j = 0; j < 3; ++j) phif[j] = U[j * nC + own[f]] * wf + U[j * nC + nei[f]] * wn;
        } else {
            for (int j = 0; j < 3; ++j) phif[j] = Ub[j * nB + (f - nI)];
        }
        const double S[3] = {Sf[f], Sf[nF + f], Sf[2 * nF + f]};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double t = S[i] * phif[j];
                if (e >> 31)
                    g[3 * i + j] -= t;
                else
                    g[3 * i + j] += t;
            }
    }
    const double iv = 1.0 / V[c];
    for (int m = 0; m < 9; ++m) g[m] = g[m] * iv;
    if (twoD)
        for (int j = 0; j < 3; ++j) g[3 * emptyDir + j] = 0.0;
    for (int m = 0; m < 9; ++m) G[size_t(m) * nC + c] = g[m];
}

// v . T (Types.h: dot(Vec3, Tensor)) with T read from the SoA gradient of cell c
__device__ __forceinline__ void vec_dot_tensor(const double v[3], const double* __restrict__ G, int nC, int c,
                                               double out[3]) {
    for (int j = 0; j < 3; ++j)
        out[j] = v[0] * G[size_t(j) * nC + c] + v[1] * G[size_t(3 + j) * nC + c] + v[2] * G[size_t(6 + j) * nC + c];
}

// ---------------------------------------------------------------- momentum operators, internal faces
// fvm::div(phi, U) (Fvm.h:74-123) and fvm::laplacian(nu, U) (Fvm.h:143-168) per internal face, and
// the combined off-diagonals of UEqn = ddt + div - laplacian (FvMatrix.h:52-79, addOffDiag).
__global__ void k_mom_faces(int nI, int nC, int nF, const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                            const double* __restrict__ w, const double* __restrict__ magSf,
                            const double* __restrict__ ndc, const double* __restrict__ d,
                            const double* __restrict__ corr, const double* __restrict__ C,
                            const double* __restrict__ Cf, const double* __restrict__ phi, double nu,
                            const double* __restrict__ nuF, int scheme, double limK, const double* __restrict__ U,
                            int nonOrth, const double* __restrict__ G, const double* __restrict__ skew,
                            double* __restrict__ loDiv, double* __restrict__ upDiv, double* __restrict__ lapUp,
                            double* __restrict__ upper, double* __restrict__ lower, double* __restrict__ cDiv,
                            double* __restrict__ cSkew, double* __restrict__ ffc) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nI) return;
    const double F = phi[f];
    const double wUp = F >= 0 ? 1.0 : 0.0;
    double wf;
    if (scheme == kUpwind || scheme == kLinearUpwind) {
        wf = wUp;
    } else if (scheme == kLinear) {
        wf = w[f];
    } else if (scheme == kLUST) {
        wf = 0.75 * w[f] + 0.25 * wUp;
    } else {
        // limiterR for a vector field (Fvm.h:55-61): r from (phiN - phiP) . (d . grad upwind)
        const int o = own[f], n = nei[f];
        double gradf[3], gradcf[3];
        for (int k = 0; k < 3; ++k) gradf[k] = U[size_t(k) * nC + n] - U[size_t(k) * nC + o];
        const double dv[3] = {d[f], d[nF + f], d[2 * size_t(nF) + f]};
        vec_dot_tensor(dv, G, nC, F > 0 ? o : n, gradcf);
        const double a = gradf[0] * gradcf[0] + gradf[1] * gradcf[1] + gradf[2] * gradcf[2];
        const double b = gradf[0] * gradf[0] + gradf[1] * gradf[1] + gradf[2] * gradf[2];
        double r;
        if (fabs(a) >= 1000.0 * b)
            r = 2.0 * 1000.0 * (a >= 0 ? 1 : -1) - 1.0;
        else
            r = 2.0 * (a / b) - 1.0;
        const double lim = tvd_limiter(scheme, limK, r);
        wf = lim * w[f] + (1.0 - lim) * wUp;
    }
    const double lo = -wf * F;
    const double up = lo + F;
    // laplacian(nu_eff, U) with the face values nuF (turbulence model) or the uniform nu
    const double gam = nuF ? nuF[f] : nu;
    const double lap = gam * magSf[f] * ndc[f];
    loDiv[f] = lo;
    upDiv[f] = up;
    lapUp[f] = lap;
    double u = 0.0, l = 0.0;
    l += 1.0 * lo;
    u += 1.0 * up;
    l += -1.0 * lap;
    u += -1.0 * lap;
    upper[f] = u;
    lower[f] = l;
    const int o = own[f], n = nei[f];
    // linearUpwind / LUST: explicit gradient correction (Fvm.h:106-116)
    double cc[3] = {0.0, 0.0, 0.0};
    if (scheme == kLinearUpwind || scheme == kLUST) {
        const double fac = scheme == kLUST ? 0.25 : 1.0;
        double v[3], corrv[3];
        if (F >= 0) {
            for (int k = 0; k < 3; ++k) v[k] = Cf[size_t(k) * nF + f] - C[size_t(k) * nC + o];
            vec_dot_tensor(v, G, nC, o, corrv);
        } else {
            for (int k = 0; k < 3; ++k) v[k] = Cf[size_t(k) * nF + f] - (C[size_t(k) * nC + o] + d[size_t(k) * nF + f]);
            vec_dot_tensor(v, G, nC, n, corrv);
        }
        const double s = fac * F;
        for (int k = 0; k < 3; ++k) cc[k] = corrv[k] * s;
    }
    for (int k = 0; k < 3; ++k) cDiv[size_t(k) * nI + f] = cc[k];
    // skewed mesh, linear / LUST: explicit skew correction of the linear part (Fvm.h:83, 119-123)
    if (skew && (scheme == kLinear || scheme == kLUST)) {
        const double fac = scheme == kLUST ? 0.75 : 1.0;
        const double wo = w[f], wn = 1.0 - wo;
        double gf[9];
        for (int m = 0; m < 9; ++m) gf[m] = G[size_t(m) * nC + o] * wo + G[size_t(m) * nC + n] * wn;
        const double sv[3] = {skew[f], skew[nF + f], skew[2 * size_t(nF) + f]};
        const double s = fac * F;
        for (int j = 0; j < 3; ++j) cSkew[size_t(j) * nI + f] = (sv[0] * gf[j] + sv[1] * gf[3 + j] + sv[2] * gf[6 + j]) * s;
    }
    // non-orthogonal correction of the laplacian (Fvm.h:155-167)
    double fc[3] = {0.0, 0.0, 0.0};
    if (nonOrth) {
        const double wo = w[f], wn = 1.0 - wo;
        double gf[9];
        for (int m = 0; m < 9; ++m) gf[m] = G[size_t(m) * nC + o] * wo + G[size_t(m) * nC + n] * wn;
        const double cv[3] = {corr[f], corr[nF + f], corr[2 * nF + f]};
        const double s = gam * magSf[f];
        for (int j = 0; j < 3; ++j) fc[j] = (cv[0] * gf[j] + cv[1] * gf[3 + j] + cv[2] * gf[6 + j]) * s;
    }
    for (int k = 0; k < 3; ++k) ffc[size_t(k) * nI + f] = fc[k];
}

// ---------------------------------------------------------------- momentum operators, boundary faces
// div: internalCoeffs += F vic, boundarySource -= F vbc (Fvm.h:117-126); laplacian: += gs gic,
// -= gs gbc (Fvm.h:169-178); fixedValue: vic 0, vbc U_b, gic -dc, gbc dc U_b; zeroGradient: vic 1,
// others 0 (BoundaryCondition.h:104-130).  UEqn = (0 + div) - laplacian.
__global__ void k_mom_bfaces(int nB, int nI, int nC, int nF, const int32_t* __restrict__ own,
                             const int32_t* __restrict__ bPatch, const int32_t* __restrict__ uType,
                             const double* __restrict__ uValueB, const double* __restrict__ wIO,
                             const double* __restrict__ uRobin, const double* __restrict__ Sf,
                             const double* __restrict__ magSf, const double* __restrict__ ndc,
                             const double* __restrict__ phi, double nu, const double* __restrict__ nuF,
                             const double* __restrict__ U, double* __restrict__ ic, double* __restrict__ bs) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB) return;
    const int f = nI + b, q = bPatch[b];
    const bool fixedValue = uType[q] == 1, symmetry = uType[q] == 2;
    const double F = phi[f], dc = ndc[f], gs = (nuF ? nuF[f] : nu) * magSf[f];
    // symmetry (SymmetryBC<Vec3>, VolField.h:174-191): vic = 1 - n^2, vbc = ub - vic u,
    // gic = -dc n^2, gbc = -dc (n.u) n - gic u, per component
    double n[3] = {0.0, 0.0, 0.0}, u[3] = {0.0, 0.0, 0.0}, dnu = 0.0;
    if (symmetry) {
        const double A = magSf[f];
        const int c = own[f];
        for (int k = 0; k < 3; ++k) {
            n[k] = Sf[size_t(k) * nF + f] / A;
            u[k] = U[size_t(k) * nC + c];
        }
        dnu = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
    }
    for (int k = 0; k < 3; ++k) {
        const double val = fixedValue ? uValueB[k * nB + b] : 0.0;
        double vic = fixedValue ? 0.0 : 1.0, vbc = fixedValue ? val : 0.0;
        double gic = fixedValue ? -dc : 0.0, gbc = fixedValue ? val * dc : 0.0;
        if (uType[q] == 6) {
            // pressureInletOutletVelocity (BoundaryCondition.h:351-360, VolField.h:204-215)
            const int c = own[f];
            const double uk = U[size_t(k) * nC + c];
            double fv;
            if (F >= 0) {
                vic = 1.0;
                fv = uk;
            } else {
                const double A = magSf[f];
                double nn[3], uu[3], ut[3];
                for (int j = 0; j < 3; ++j) {
                    nn[j] = Sf[size_t(j) * nF + f] / A;
                    uu[j] = U[size_t(j) * nC + c];
                    ut[j] = uValueB[j * nB + b];
                }
                vic = nn[k] * nn[k];
                const double nu_ = nn[0] * uu[0] + nn[1] * uu[1] + nn[2] * uu[2];
                const double nt = nn[0] * ut[0] + nn[1] * ut[1] + nn[2] * ut[2];
                fv = nu_ * nn[k] + (ut[k] - nt * nn[k]);
            }
            vbc = fv - vic * uk;
            gic = dc * (vic - 1.0);
            gbc = dc * vbc;
        }
        if (uType[q] == 5) {  // fixedGradient (BoundaryCondition.h:145-148)
            const double g = uValueB[k * nB + b];
            vic = 1.0;
            vbc = g / dc;
            gic = 0.0;
            gbc = g;
        }
        if (uType[q] == 8) {  // Robin (BoundaryCondition.h:170-184)
            const double a = uRobin[2 * q], rb = uRobin[2 * q + 1], cv = uValueB[k * nB + b];
            const double bd = rb * dc;
            vic = bd / (a + bd);
            vbc = cv / (a + rb * dc);
            gic = dc * (rb * dc / (a + rb * dc) - 1.0);
            gbc = dc * (cv / (a + rb * dc));
        }
        if (uType[q] == 3 || uType[q] == 4 || uType[q] == 9) {
            // inletOutlet / freestream / advective = mixed (MixedBC, BoundaryCondition.h:236-243) with refGrad 0
            const double w = wIO[b], rv = uValueB[k * nB + b], rg = 0.0;
            vic = 1.0 - w;
            vbc = w * rv + (1.0 - w) * (rg / dc);
            gic = -w * dc;
            gbc = w * dc * rv + (1.0 - w) * rg;
        }
        if (symmetry) {
            const double nn = n[k] * n[k];
            vic = 1.0 - nn;
            vbc = (u[k] - dnu * n[k]) - vic * u[k];
            gic = -dc * nn;
            gbc = (-dc * dnu) * n[k] - gic * u[k];
        }
        double icDiv = 0.0, bsDiv = 0.0, icLap = 0.0, bsLap = 0.0;
        icDiv += vic * F;
        bsDiv -= vbc * F;
        icLap += gic * gs;
        bsLap -= gbc * gs;
        double i = 0.0, s = 0.0;
        i += icDiv;
        s += bsDiv;
        i -= icLap;
        s -= bsLap;
        ic[size_t(k) * nB + b] = i;
        bs[size_t(k) * nB + b] = s;
    }
}

// ---------------------------------------------------------------- momentum operators, cells
// diag and source of ddt (Fvm.h:18-31), div and laplacian accumulated per operator in face order,
// then UEqn = ddt; UEqn += div; UEqn -= laplacian (FvMatrix.h:52-79)
__global__ void k_mom_cells(int nC, int nI, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                            const double* __restrict__ loDiv, const double* __restrict__ upDiv,
                            const double* __restrict__ lapUp, const double* __restrict__ cDiv,
                            const double* __restrict__ cSkew, const double* __restrict__ ffc,
                            const double* __restrict__ V, int transient, double kc,
                            double kc0, double kc00, const double* __restrict__ U0, const double* __restrict__ U00,
                            double* __restrict__ diag, double* __restrict__ src) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double dDiv = 0.0, dLap = 0.0, sDiv[3] = {0.0, 0.0, 0.0}, sLap[3] = {0.0, 0.0, 0.0};
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = int(e & 0x7fffffffu);
        if (f >= nI) continue;
        if (e >> 31) {
            dDiv -= upDiv[f];
            dLap -= lapUp[f];
            for (int q = 0; q < 3; ++q) {
                sDiv[q] += cDiv[size_t(q) * nI + f];
                if (cSkew) sDiv[q] += cSkew[size_t(q) * nI + f];
                sLap[q] += ffc[size_t(q) * nI + f];
            }
        } else {
            dDiv -= loDiv[f];
            dLap -= lapUp[f];
            for (int q = 0; q < 3; ++q) {
                sDiv[q] -= cDiv[size_t(q) * nI + f];
                if (cSkew) sDiv[q] -= cSkew[size_t(q) * nI + f];
                sLap[q] -= ffc[size_t(q) * nI + f];
            }
        }
    }
    double dg = 0.0, s[3] = {0.0, 0.0, 0.0};
    if (transient) {
        const double Vc = V[c];
        dg += kc * Vc;
        for (int q = 0; q < 3; ++q) {
            const double t = U0[size_t(q) * nC + c] * kc0 - U00[size_t(q) * nC + c] * kc00;
            s[q] += t * Vc;
        }
    }
    dg += dDiv;
    dg -= dLap;
    diag[c] = dg;
    for (int q = 0; q < 3; ++q) {
        s[q] += sDiv[q];
        s[q] -= sLap[q];
        src[size_t(q) * nC + c] = s[q];
    }
}

// ---------------------------------------------------------------- FvMatrix::relax (FvMatrix.h:111-131)
__global__ void k_mom_relax(int nC, int nI, int nB, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                            const double* __restrict__ upper, const double* __restrict__ lower,
                            const double* __restrict__ ic, const double* __restrict__ U, double alpha,
                            double* __restrict__ diag, double* __restrict__ src) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double sumOff = 0.0, bD = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = int(e & 0x7fffffffu);
        if (f < nI) {
            sumOff += (e >> 31) ? fabs(lower[f]) : fabs(upper[f]);
        } else {
            const int b = f - nI;
            double m = ic[b];
            const double y = ic[size_t(nB) + b], z = ic[size_t(2) * nB + b];
            if (m < y) m = y;
            if (m < z) m = z;
            bD += m;
        }
    }
    const double Dfull = diag[c] + bD;
    const double aD = fabs(Dfull);
    const double D = aD < sumOff ? sumOff : aD;
    const double dD = D / alpha - Dfull;
    diag[c] += dD;
    for (int q = 0; q < 3; ++q) src[size_t(q) * nC + c] += U[size_t(q) * nC + c] * dD;
}

// M = UEqn - (-grad p): source += (-grad p) V  (FvMatrix.h:89-97); gp: 3 per cell
__global__ void k_mom_gradp(int nC, const double* __restrict__ src, const double* __restrict__ gp,
                            const double* __restrict__ V, double* __restrict__ msrc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    for (int q = 0; q < 3; ++q) msrc[size_t(q) * nC + c] = src[size_t(q) * nC + c] + (-gp[3 * c + q]) * V[c];
}

// A (FvMatrix.h:178-187), rAU = 1/A, H (FvMatrix.h:189-206), HbyA = rAU H
__global__ void k_mom_AH(int nC, int nI, int nB, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                         const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                         const double* __restrict__ diag, const double* __restrict__ upper,
                         const double* __restrict__ lower, const double* __restrict__ ic, const double* __restrict__ bs,
                         const double* __restrict__ src, const double* __restrict__ U, const double* __restrict__ V,
                         double* __restrict__ rAU, double* __restrict__ HbyA) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double a = diag[c];
    double h[3] = {src[c], src[size_t(nC) + c], src[size_t(2) * nC + c]};
    const int k0 = cfOff[c], k1 = cfOff[c + 1];
    // internal faces first (all of them precede the boundary faces in the cell's ascending list)
    for (int k = k0; k < k1; ++k) {
        const uint32_t e = (uint32_t)cf[k];
        const int f = int(e & 0x7fffffffu);
        if (f >= nI) continue;
        if (e >> 31) {
            const double lf = lower[f];
            const int o = own[f];
            for (int q = 0; q < 3; ++q) h[q] -= U[size_t(q) * nC + o] * lf;
        } else {
            const double uf = upper[f];
            const int n = nei[f];
            for (int q = 0; q < 3; ++q) h[q] -= U[size_t(q) * nC + n] * uf;
        }
    }
    for (int k = k0; k < k1; ++k) {
        const int f = int((uint32_t)cf[k] & 0x7fffffffu);
        if (f < nI) continue;
        const int b = f - nI;
        const double icv[3] = {ic[b], ic[size_t(nB) + b], ic[size_t(2) * nB + b]};
        const double av = (icv[0] + icv[1] + icv[2]) / 3.0;
        a += av;
        for (int q = 0; q < 3; ++q) {
            h[q] += bs[size_t(q) * nB + b];
            h[q] -= (icv[q] - av) * U[size_t(q) * nC + c];
        }
    }
    a /= V[c];
    const double r = 1.0 / a;
    rAU[c] = r;
    for (int q = 0; q < 3; ++q) HbyA[size_t(q) * nC + c] = (h[q] / V[c]) * r;
}

// fvc::gradLS (Fvc.h:135-167, 186-205) of an NC-component cell array psi (SoA): boundary faces of the
// patches with fix[p] != 0 constrain by value (d, bVal - psi_P), the others by a zero normal gradient
// (n max(n.d, 0.05|d|), 0); weights 1/|d|^2; the empty direction zeroed in 2D.  Out: SoA rows
// 3 i + j = d psi_j / dx_i (Tensor(i, j) of outer(G d, dpsi)); row i for NC = 1.
template <int NC>
__global__ void k_grad_ls_cells(int nC, int nI, int nF, int nB, const int32_t* __restrict__ cfOff,
                                const int32_t* __restrict__ cf, const int32_t* __restrict__ own,
                                const int32_t* __restrict__ nei, const double* __restrict__ Sf,
                                const double* __restrict__ magSf, const double* __restrict__ d,
                                const double* __restrict__ psi, const double* __restrict__ bVal,
                                const int32_t* __restrict__ bPatch, const int32_t* __restrict__ fix, int twoD,
                                int emptyDir, double* __restrict__ g) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    auto faceVec = [&](int f, double v[3]) -> bool {
        v[0] = d[f];
        v[1] = d[nF + f];
        v[2] = d[2 * size_t(nF) + f];
        if (f < nI || (fix && fix[bPatch[f - nI]] != 0)) return true;
        const double inv = 1.0 / magSf[f];
        const double n[3] = {Sf[f] * inv, Sf[nF + f] * inv, Sf[2 * size_t(nF) + f] * inv};
        const double nd = fmax(n[0] * v[0] + n[1] * v[1] + n[2] * v[2], 0.05 * sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        for (int k = 0; k < 3; ++k) v[k] = n[k] * nd;
        return false;
    };
    double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = int((uint32_t)cf[k] & 0x7fffffffu);
        double v[3];
        faceVec(f, v);
        const double s = 1.0 / (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double o[9] = {v[0] * v[0], v[0] * v[1], v[0] * v[2], v[1] * v[0], v[1] * v[1],
                             v[1] * v[2], v[2] * v[0], v[2] * v[1], v[2] * v[2]};
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
    double acc[3 * NC];
    for (int q = 0; q < 3 * NC; ++q) acc[q] = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = int((uint32_t)cf[k] & 0x7fffffffu);
        double v[3], dp[NC];
        const bool value = faceVec(f, v);
        if (f < nI) {
            for (int j = 0; j < NC; ++j) dp[j] = psi[size_t(j) * nC + nei[f]] - psi[size_t(j) * nC + own[f]];
        } else if (value) {
            for (int j = 0; j < NC; ++j) dp[j] = bVal[size_t(j) * nB + (f - nI)] - psi[size_t(j) * nC + c];
        } else {
            for (int j = 0; j < NC; ++j) dp[j] = 0.0;
        }
        const double wgt = 1.0 / (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double dw[3] = {v[0] * wgt, v[1] * wgt, v[2] * wgt};
        const double Gd[3] = {G[0] * dw[0] + G[1] * dw[1] + G[2] * dw[2], G[3] * dw[0] + G[4] * dw[1] + G[5] * dw[2],
                              G[6] * dw[0] + G[7] * dw[1] + G[8] * dw[2]};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < NC; ++j) acc[i * NC + j] += Gd[i] * dp[j];
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < NC; ++j)
            g[size_t(i * NC + j) * nC + c] = (twoD && i == emptyDir) ? 0.0 : acc[i * NC + j];
}

// (gic u_P + gbc) of component k of a U boundary face that the least-squares gradient constrains by its
// normal gradient (Fvc.h:283-284): zeroGradient 0; symmetry -dc n_k^2 u_k + (-dc (n.u) n_k - gic u_k)
// (VolField.h:183-191); mixed -w dc u_k + w dc v_k (refGrad 0); fixedGradient g_k;
// pressureInletOutletVelocity dc (vic - 1) u_k + dc vbc (BoundaryCondition.h:357-360)
__device__ __forceinline__ double u_ls_gradient(int t, int k, int b, int f, int c, int nB, int nC, int nF,
                                                const double* __restrict__ Sf, const double* __restrict__ magSf,
                                                double dc, const double* __restrict__ U,
                                                const double* __restrict__ uValueB, const double* __restrict__ wIO,
                                                const double* __restrict__ phi, const double* __restrict__ rob) {
    const double uk = U[size_t(k) * nC + c];
    double gic = 0.0, gbc = 0.0;
    if (t == 2 || t == 6) {
        const double A = magSf[f];
        double n[3], u[3];
        for (int j = 0; j < 3; ++j) {
            n[j] = Sf[size_t(j) * nF + f] / A;
            u[j] = U[size_t(j) * nC + c];
        }
        if (t == 2) {
            const double dnu = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
            gic = -dc * (n[k] * n[k]);
            gbc = (-dc * dnu) * n[k] - gic * uk;
        } else {
            double vic, fv;
            if (phi[f] >= 0) {
                vic = 1.0;
                fv = uk;
            } else {
                double ut[3];
                for (int j = 0; j < 3; ++j) ut[j] = uValueB[size_t(j) * nB + b];
                vic = n[k] * n[k];
                const double nu_ = n[0] * u[0] + n[1] * u[1] + n[2] * u[2];
                const double nt = n[0] * ut[0] + n[1] * ut[1] + n[2] * ut[2];
                fv = nu_ * n[k] + (ut[k] - nt * n[k]);
            }
            const double vbc = fv - vic * uk;
            gic = dc * (vic - 1.0);
            gbc = dc * vbc;
        }
    } else if (t == 3 || t == 4 || t == 9) {
        const double w = wIO[b];
        gic = -w * dc;
        gbc = w * dc * uValueB[size_t(k) * nB + b] + (1.0 - w) * 0.0;
    } else if (t == 5) {
        gbc = uValueB[size_t(k) * nB + b];
    } else if (t == 8) {
        const double a = rob[0], rb = rob[1], cv = uValueB[size_t(k) * nB + b];
        gic = dc * (rb * dc / (a + rb * dc) - 1.0);
        gbc = dc * (cv / (a + rb * dc));
    }
    return gic * uk + gbc;
}

// grad U by least squares with U's boundary conditions (fvc::grad(U, leastSquares), Fvc.h:264-289 with
// leastSquaresGrad :135-167 and finishGrad :169-181): value constraint (d, U_b - U_P) on the patches
// whose condition fixes the value (uFix), else the normal-gradient constraint n max(n.d, 0.05|d|) with
// (gic U_P + gbc) max(n.d, 0.05|d|).  Out: SoA rows 3 i + j = dU_j/dx_i.
__global__ void k_grad_ls_u(int nC, int nI, int nF, int nB, const int32_t* __restrict__ cfOff,
                            const int32_t* __restrict__ cf, const int32_t* __restrict__ own,
                            const int32_t* __restrict__ nei, const double* __restrict__ Sf,
                            const double* __restrict__ magSf, const double* __restrict__ d,
                            const double* __restrict__ ndc, const double* __restrict__ U,
                            const double* __restrict__ Ub, const int32_t* __restrict__ bPatch,
                            const int32_t* __restrict__ uType, const int32_t* __restrict__ uFix,
                            const double* __restrict__ uValueB, const double* __restrict__ wIO,
                            const double* __restrict__ phi, const double* __restrict__ uRobin, int twoD, int emptyDir,
                            double* __restrict__ G) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    // constraint vector of face f; nd set for a gradient constraint
    auto faceVec = [&](int f, double v[3], double& nd) -> bool {
        v[0] = d[f];
        v[1] = d[nF + f];
        v[2] = d[2 * size_t(nF) + f];
        if (f < nI || uFix[bPatch[f - nI]]) return true;
        const double inv = 1.0 / magSf[f];
        const double n[3] = {Sf[f] * inv, Sf[nF + f] * inv, Sf[2 * size_t(nF) + f] * inv};
        nd = fmax(n[0] * v[0] + n[1] * v[1] + n[2] * v[2], 0.05 * sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
        for (int k = 0; k < 3; ++k) v[k] = n[k] * nd;
        return false;
    };
    double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = int((uint32_t)cf[k] & 0x7fffffffu);
        double v[3], nd = 0.0;
        faceVec(f, v, nd);
        const double s = 1.0 / (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double o[9] = {v[0] * v[0], v[0] * v[1], v[0] * v[2], v[1] * v[0], v[1] * v[1],
                             v[1] * v[2], v[2] * v[0], v[2] * v[1], v[2] * v[2]};
        for (int q = 0; q < 9; ++q) a[q] += o[q] * s;
    }
    if (twoD) a[4 * emptyDir] += 1.0;
    const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                       a[2] * (a[3] * a[7] - a[4] * a[6]);
    double Gi[9];
    Gi[0] = (a[4] * a[8] - a[5] * a[7]) / det;
    Gi[1] = (a[2] * a[7] - a[1] * a[8]) / det;
    Gi[2] = (a[1] * a[5] - a[2] * a[4]) / det;
    Gi[3] = (a[5] * a[6] - a[3] * a[8]) / det;
    Gi[4] = (a[0] * a[8] - a[2] * a[6]) / det;
    Gi[5] = (a[2] * a[3] - a[0] * a[5]) / det;
    Gi[6] = (a[3] * a[7] - a[4] * a[6]) / det;
    Gi[7] = (a[1] * a[6] - a[0] * a[7]) / det;
    Gi[8] = (a[0] * a[4] - a[1] * a[3]) / det;
    double acc[9];
    for (int q = 0; q < 9; ++q) acc[q] = 0.0;
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = int((uint32_t)cf[k] & 0x7fffffffu);
        double v[3], dp[3], nd = 0.0;
        const bool value = faceVec(f, v, nd);
        if (f < nI) {
            for (int j = 0; j < 3; ++j) dp[j] = U[size_t(j) * nC + nei[f]] - U[size_t(j) * nC + own[f]];
        } else if (value) {
            for (int j = 0; j < 3; ++j) dp[j] = Ub[size_t(j) * nB + (f - nI)] - U[size_t(j) * nC + c];
        } else {
            const int b = f - nI, t = uType[bPatch[b]];
            for (int j = 0; j < 3; ++j)
                dp[j] = u_ls_gradient(t, j, b, f, c, nB, nC, nF, Sf, magSf, ndc[f], U, uValueB, wIO, phi,
                                      uRobin ? uRobin + 2 * bPatch[b] : nullptr) * nd;
        }
        const double wgt = 1.0 / (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        const double dw[3] = {v[0] * wgt, v[1] * wgt, v[2] * wgt};
        const double Gd[3] = {Gi[0] * dw[0] + Gi[1] * dw[1] + Gi[2] * dw[2],
                              Gi[3] * dw[0] + Gi[4] * dw[1] + Gi[5] * dw[2],
                              Gi[6] * dw[0] + Gi[7] * dw[1] + Gi[8] * dw[2]};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) acc[3 * i + j] += Gd[i] * dp[j];
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) G[size_t(3 * i + j) * nC + c] = (twoD && i == emptyDir) ? 0.0 : acc[3 * i + j];
}

__global__ void k_io_patch_reset(int nP, const int32_t* __restrict__ uType, int32_t* __restrict__ uFix) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < nP && (uType[q] == 3 || uType[q] == 9)) uFix[q] = 0;
}

// inletOutlet and advective patches fix U for the least-squares gradient while any face has a positive
// value fraction (MixedBC::fixesValue, BoundaryCondition.h:246-250): inflow, or a transient advective step
__global__ void k_io_patch_fix(int nB, const int32_t* __restrict__ bPatch, const int32_t* __restrict__ uType,
                               const double* __restrict__ wIO, int32_t* __restrict__ uFix) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nB && (uType[bPatch[b]] == 3 || uType[bPatch[b]] == 9) && wIO[b] > 0) uFix[bPatch[b]] = 1;
}

// HbyA boundary values of the skew-corrected Rhie-Chow flux on fixes-flux faces: U_b + rAU_P grad p_P
// (IncompressibleFlow.cpp:262-272); gp: 3 per cell
__global__ void k_hbya_bval(int nB, int nI, const int32_t* __restrict__ own, const int32_t* __restrict__ bPatch,
                            const int32_t* __restrict__ fixesFlux, const double* __restrict__ Ub,
                            const double* __restrict__ rAU, const double* __restrict__ gp, double* __restrict__ hB) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB || !fixesFlux[bPatch[b]]) return;
    const int o = own[nI + b];
    for (int j = 0; j < 3; ++j) hB[size_t(j) * nB + b] = Ub[size_t(j) * nB + b] + rAU[o] * gp[3 * size_t(o) + j];
}

// rAUf = interpolate(rAU) (Fvc.h:24-32) and phiHbyA (IncompressibleFlow.cpp:258-281)
__global__ void k_phi_hbya(int nF, int nI, int nB, int nC, const int32_t* __restrict__ own,
                           const int32_t* __restrict__ nei, const double* __restrict__ w, const double* __restrict__ Sf,
                           const int32_t* __restrict__ bPatch, const int32_t* __restrict__ uFixesFlux,
                           const double* __restrict__ rAU, const double* __restrict__ HbyA,
                           const double* __restrict__ Ub, const double* __restrict__ skew,
                           const double* __restrict__ gR, const double* __restrict__ gH, double* __restrict__ rAUf,
                           double* __restrict__ phiHbyA) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    const double S[3] = {Sf[f], Sf[nF + f], Sf[2 * nF + f]};
    const int o = own[f];
    if (f < nI) {
        const int n = nei[f];
        const double wf = w[f], wn = 1.0 - wf;
        double r = wf * rAU[o] + wn * rAU[n];
        double Hf[3];
        for (int q = 0; q < 3; ++q) Hf[q] = HbyA[size_t(q) * nC + o] * wf + HbyA[size_t(q) * nC + n] * wn;
        if (skew) {
            // skewed mesh: rAUf and HbyA_f with (x_f - x'_f) . grad_f (Fvc.h:73-82; IncompressibleFlow.cpp:252-282)
            const double sv[3] = {skew[f], skew[nF + f], skew[2 * size_t(nF) + f]};
            double gr[3];
            for (int i = 0; i < 3; ++i) gr[i] = wf * gR[size_t(i) * nC + o] + wn * gR[size_t(i) * nC + n];
            r += sv[0] * gr[0] + sv[1] * gr[1] + sv[2] * gr[2];
            double gf[9];
            for (int m = 0; m < 9; ++m) gf[m] = wf * gH[size_t(m) * nC + o] + wn * gH[size_t(m) * nC + n];
            for (int j = 0; j < 3; ++j) Hf[j] += sv[0] * gf[j] + sv[1] * gf[3 + j] + sv[2] * gf[6 + j];
        }
        rAUf[f] = r;
        phiHbyA[f] = Hf[0] * S[0] + Hf[1] * S[1] + Hf[2] * S[2];
    } else {
        const int b = f - nI;
        rAUf[f] = rAU[o];
        if (uFixesFlux[bPatch[b]])  // fixesFlux (BoundaryCondition.h:76, 203, 251)
            phiHbyA[f] = Ub[b] * S[0] + Ub[size_t(nB) + b] * S[1] + Ub[size_t(2) * nB + b] * S[2];
        else
            phiHbyA[f] = HbyA[o] * S[0] + HbyA[size_t(nC) + o] * S[1] + HbyA[size_t(2) * nC + o] * S[2];
    }
}

// totalPressure values (TotalPressureBC::update, VolField.h:217-223): p0 - |U_b|^2 / 2 on inflow faces
// (phi < 0), p0 elsewhere; phi == NULL (no flux yet) gives p0
__global__ void k_total_pressure(int nB, int nI, const int32_t* __restrict__ bPatch, const int32_t* __restrict__ pType,
                                 const double* __restrict__ phi, const double* __restrict__ Ub,
                                 const double* __restrict__ p0, double* __restrict__ pValueB) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB || pType[bPatch[b]] != 7) return;
    if (phi && phi[nI + b] < 0) {
        const double u0 = Ub[b], u1 = Ub[size_t(nB) + b], u2 = Ub[2 * size_t(nB) + b];
        pValueB[b] = p0[b] - 0.5 * (u0 * u0 + u1 * u1 + u2 * u2);
    } else {
        pValueB[b] = p0[b];
    }
}

// constrainPressure (IncompressibleFlow.cpp:17-29): the fixedFluxPressure gradient that makes the
// boundary flux the boundary velocity's, g = (phiHbyA - U_b.S) / (|S| rAUf)
__global__ void k_flux_pressure(int nB, int nI, int nF, const int32_t* __restrict__ bPatch,
                                const int32_t* __restrict__ pType, const double* __restrict__ phiHbyA,
                                const double* __restrict__ Ub, const double* __restrict__ Sf,
                                const double* __restrict__ magSf, const double* __restrict__ rAUf,
                                double* __restrict__ pValueB) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nB || pType[bPatch[b]] != 6) return;
    const int f = nI + b;
    const double ubS = Ub[b] * Sf[f] + Ub[size_t(nB) + b] * Sf[nF + f] + Ub[2 * size_t(nB) + b] * Sf[2 * size_t(nF) + f];
    pValueB[b] = (phiHbyA[f] - ubS) / (magSf[f] * rAUf[f]);
}

// phi = phiHbyA - flux (IncompressibleFlow.cpp:337-340)
__global__ void k_phi_update(int nF, const double* __restrict__ phiHbyA, const double* __restrict__ F,
                             double* __restrict__ phi) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nF) phi[f] = phiHbyA[f] - F[f];
}

// p = pPrev + alphaP (p - pPrev) (IncompressibleFlow.cpp:345-348)
__global__ void k_p_relax(int nC, const double* __restrict__ pPrev, double alpha, double* __restrict__ p) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < nC) p[c] = pPrev[c] + alpha * (p[c] - pPrev[c]);
}

// U = HbyA - rAU grad p, empty direction zeroed (IncompressibleFlow.cpp:355-360)
__global__ void k_u_correct(int nC, const double* __restrict__ HbyA, const double* __restrict__ rAU,
                            const double* __restrict__ gp, int twoD, int emptyDir, double* __restrict__ U) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    for (int q = 0; q < 3; ++q) U[size_t(q) * nC + c] = HbyA[size_t(q) * nC + c] - gp[3 * c + q] * rAU[c];
    if (twoD) U[size_t(emptyDir) * nC + c] = 0.0;
}

// phi = U_f . S_f with boundary faces at the boundary value (Fvc.h:103-109, initialize)
__global__ void k_flux_u(int nF, int nI, int nB, int nC, const int32_t* __restrict__ own,
                         const int32_t* __restrict__ nei, const double* __restrict__ w, const double* __restrict__ Sf,
                         const double* __restrict__ U, const double* __restrict__ Ub, const double* __restrict__ skew,
                         const double* __restrict__ G, double* __restrict__ phi) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    double Uf[3];
    if (f < nI) {
        const int o = own[f], n = nei[f];
        const double wf = w[f], wn = 1.0 - wf;
        for (int q = 0; q < 3; ++q) Uf[q] = U[size_t(q) * nC + o] * wf + U[size_t(q) * nC + n] * wn;
        if (skew) {  // skewed mesh: fvc::flux(U, grad U) (Fvc.h:84-95, IncompressibleFlow.cpp:36)
            const double sv[3] = {skew[f], skew[nF + f], skew[2 * size_t(nF) + f]};
            double gf[9];
            for (int m = 0; m < 9; ++m) gf[m] = wf * G[size_t(m) * nC + o] + wn * G[size_t(m) * nC + n];
            for (int j = 0; j < 3; ++j) Uf[j] += sv[0] * gf[j] + sv[1] * gf[3 + j] + sv[2] * gf[6 + j];
        }
    } else {
        for (int q = 0; q < 3; ++q) Uf[q] = Ub[size_t(q) * nB + (f - nI)];
    }
    phi[f] = Uf[0] * Sf[f] + Uf[1] * Sf[nF + f] + Uf[2] * Sf[2 * nF + f];
}

// max |div phi| (the values are non-negative: the IEEE bit patterns order like the numbers)
__global__ void k_max_abs(int n, const double* __restrict__ v, unsigned long long* __restrict__ out) {
    unsigned long long m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double a = fabs(v[i]);
        const unsigned long long bits = (unsigned long long)__double_as_longlong(a);
        if (bits > m) m = bits;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_down_sync(0xffffffffu, m, o);
        if (t > m) m = t;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// U: SoA <-> AoS (3 per cell)
__global__ void k_soa_from_aos(int n, const double* __restrict__ a, double* __restrict__ s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        for (int q = 0; q < 3; ++q) s[size_t(q) * n + i] = a[3 * size_t(i) + q];
}
__global__ void k_aos_from_soa(int n, const double* __restrict__ s, double* __restrict__ a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        for (int q = 0; q < 3; ++q) a[3 * size_t(i) + q] = s[size_t(q) * n + i];
}

}  // namespace

// ====================================================================== DeviceFlow
DeviceFlow::DeviceFlow(DeviceBatch& batch, DeviceGeom& geom, const vlm_flow_ctrl& ctrl, const int32_t* uType,
                       const double* uValue, const int32_t* pType, const double* pValue, cudaStream_t s)
    : batch_(batch), G_(geom), ctrl_(ctrl), s_(s) {
    nC_ = G_.nCells();
    nI_ = G_.nInternal();
    nF_ = G_.nFaces();
    nB_ = G_.nBoundary();
    const int nP = G_.nPatches();
    VLM_REQUIRE(batch_.plan().nsys == 1, VLM_ERR_UNSUPPORTED, "the device flow step runs on a single-system mesh");
    VLM_REQUIRE(ctrl_.div_scheme >= 0 && ctrl_.div_scheme <= 7, VLM_ERR_BAD_ARG, "unknown divergence scheme");
    if (ctrl_.div_coeff == 0) ctrl_.div_coeff = 1.0;
    VLM_REQUIRE(ctrl_.grad_scheme == 0 || ctrl_.grad_scheme == 1, VLM_ERR_BAD_ARG,
                "grad_scheme must be 0 (Gauss linear) or 1 (leastSquares)");
    VLM_REQUIRE(ctrl_.grad_p_scheme >= 0 && ctrl_.grad_p_scheme <= 2, VLM_ERR_BAD_ARG,
                "grad_p_scheme must be 0 (Gauss linear), 1 (leastSquares) or 2 (GaussSkew)");
    VLM_REQUIRE(ctrl_.grad_p_scheme != 2 || G_.hasSkewVectors(), VLM_ERR_BAD_ARG,
                "the GaussSkew pressure gradient needs the mesh registered with its skew vectors");
    VLM_REQUIRE(ctrl_.ddt_scheme >= 0 && ctrl_.ddt_scheme <= 2, VLM_ERR_BAD_ARG, "unknown ddt scheme");
    VLM_REQUIRE(ctrl_.nu > 0, VLM_ERR_BAD_ARG, "nu must be positive");
    VLM_REQUIRE(ctrl_.n_corr >= 1 && ctrl_.n_outer >= 1 && ctrl_.n_non_orth_corr >= 0, VLM_ERR_BAD_ARG,
                "nOuter, nCorr must be >= 1 and nNonOrthCorr >= 0");
    if (ctrl_.div_scheme == kLinearUpwind || ctrl_.div_scheme == kLUST)
        VLM_REQUIRE(G_.C() && G_.Cf(), VLM_ERR_BAD_ARG,
                    "linearUpwind / LUST need the cell and face centres (vlm_mesh_desc.C, .Cf)");
    uTypeHost_.assign(uType, uType + nP);
    pTypeHost_.assign(pType, pType + nP);
    // the types the assembly sees: fixedFluxPressure is a fixedGradient whose gradient the corrector sets
    pTypeAsm_.assign(pType, pType + nP);
    // and totalPressure a fixedValue whose values the step start sets
    for (int32_t& t : pTypeAsm_)
        if (t == 6) {
            t = 5;
            hasFluxPressure_ = true;
        } else if (t == 7) {
            t = 1;
            hasTotalPressure_ = true;
        }
    // Robin coefficients {a, b} per patch (a phi + b dphi/dn = c); c is the patch value
    uRobinH_.assign(size_t(2) * std::max(nP, 1), 0.0);
    pRobinH_.assign(size_t(2) * std::max(nP, 1), 0.0);
    for (int q = 0; q < nP; ++q) {
        VLM_REQUIRE((uType[q] >= 0 && uType[q] <= 6) || uType[q] == 8 || uType[q] == 9, VLM_ERR_BAD_ARG,
                    "U boundary type must be 0 to 6, 8 or 9");
        if (uType[q] == 3) hasInletOutlet_ = true;
        if (uType[q] == 9) {
            hasAdvective_ = true;
            if (ctrl_.u_advective) {
                const double* a = ctrl_.u_advective + 4 * q;
                VLM_REQUIRE(std::isfinite(a[0]) && a[0] >= 0.0 && std::isfinite(a[1]) && std::isfinite(a[2]) &&
                                std::isfinite(a[3]),
                            VLM_ERR_BAD_ARG, "advective far field: lInf must be finite and not negative");
            }
        }
        VLM_REQUIRE(pType[q] == 0 || pType[q] == 1 || pType[q] == 2 || (pType[q] >= 4 && pType[q] <= 8),
                    VLM_ERR_BAD_ARG, "p boundary type must be 0, 1, 2, 4, 5, 6, 7 or 8");
        for (int side = 0; side < 2; ++side) {
            const bool rob = (side == 0 ? uType[q] : pType[q]) == 8;
            if (!rob) continue;
            const double* src = side == 0 ? ctrl_.u_robin : ctrl_.p_robin;
            VLM_REQUIRE(src != nullptr, VLM_ERR_BAD_ARG, "a Robin boundary needs its {a, b} coefficients (u_robin / p_robin)");
            const double a = src[2 * q], b = src[2 * q + 1];
            VLM_REQUIRE(std::isfinite(a) && std::isfinite(b) && (a != 0.0 || b != 0.0), VLM_ERR_BAD_ARG,
                        "Robin coefficients a and b must be finite and not both zero");
            std::vector<double>& dst = side == 0 ? uRobinH_ : pRobinH_;
            dst[2 * q] = a;
            dst[2 * q + 1] = b;
        }
        VLM_REQUIRE(pType[q] != 4 || uType[q] == 4, VLM_ERR_BAD_ARG,
                    "freestreamPressure needs the freestream velocity condition on the same patch");
    }
    if (hasAdvective_) {
        std::vector<double> adv(size_t(4) * std::max(nP, 1), 0.0);
        for (int q = 0; q < nP; ++q)
            if (uType[q] == 9 && ctrl_.u_advective)
                for (int k = 0; k < 4; ++k) adv[4 * q + k] = ctrl_.u_advective[4 * q + k];
        uAdv_.upload(adv, s_);
    }
    // the stored controls do not keep the caller's Robin and advective arrays
    ctrl_.u_robin = nullptr;
    ctrl_.p_robin = nullptr;
    ctrl_.u_advective = nullptr;
    uRobin_.upload(uRobinH_, s_);
    pRobin_.upload(pRobinH_, s_);
    // pressureNeedsReference (IncompressibleFlow.cpp:109-113): no patch fixes p (Robin fixes it when a != 0)
    needRef_ = true;
    for (int q = 0; q < nP; ++q)
        if ((pType[q] == 1 || pType[q] == 7 || (pType[q] == 8 && pRobinH_[2 * q] != 0.0)) && G_.patchSize()[q] > 0)
            needRef_ = false;
    for (int k = 0; k < 3; ++k)
        if (!G_.twoD() || k != G_.emptyDir()) solved_.push_back(k);  // Mesh.cpp:642-644
    uType_.upload(uTypeHost_, s_);
    pType_.upload(pTypeHost_, s_);
    // fixesFlux per patch (BoundaryCondition.h:76, 203, 251): fixedValue and symmetry
    std::vector<int32_t> fix(size_t(std::max(nP, 1)), 0);
    for (int q = 0; q < nP; ++q) fix[q] = uType[q] == 1 || uType[q] == 2 || (uType[q] == 8 && uRobinH_[2 * q] != 0.0);
    uFixesFlux_.upload(fix, s_);
    // per boundary face: U values of fixedValue faces and inlet values of inletOutlet faces (SoA), p values
    const size_t nBb = size_t(std::max(nB_, 1));
    std::vector<double> uv(3 * nBb, 0.0), pv(nBb, 0.0);
    for (int q = 0; q < nP; ++q)
        for (int i = 0; i < G_.patchSize()[q]; ++i) {
            const size_t b = size_t(G_.patchStart()[q] - nI_ + i);
            for (int k = 0; k < 3; ++k) uv[k * nBb + b] = uValue[3 * q + k];
            pv[b] = pType[q] == 6 ? 0.0 : pValue[q];  // FixedFluxPressureBC starts with a zero gradient
        }
    uValueB_.upload(uv, s_);
    pValueB_.upload(pv, s_);
    if (hasTotalPressure_) pTotal_.upload(pv, s_);  // p0 per face
    wIO_.resize(nBb);
    wIO_.zero(s_);
    if (hasAdvective_) {
        advOld_.resize(3 * nBb);
        advOld_.zero(s_);
        advOldOld_.resize(3 * nBb);
        advOldOld_.zero(s_);
    }
    pFrac_.resize(nBb);
    pFrac_.zero(s_);
    bool freestream = false;
    for (int q = 0; q < nP; ++q) freestream = freestream || uType[q] == 4;
    if (freestream && nB_ > 0) {
        k_freestream_fractions<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, nF_, G_.bPatch(), uType_.get(), pType_.get(),
                                                          uValueB_.get(), G_.Sf(), G_.magSf(), wIO_.get(),
                                                          pFrac_.get()), ++launches_;
        // a freestreamPressure patch fixes p where any of its faces has a positive value fraction
        std::vector<double> pf(nBb);
        VLM_CUDA(cudaMemcpyAsync(pf.data(), pFrac_.get(), sizeof(double) * nBb, cudaMemcpyDeviceToHost, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
        for (int q = 0; q < nP; ++q)
            if (pType[q] == 4)
                for (int i = 0; i < G_.patchSize()[q]; ++i)
                    if (pf[size_t(G_.patchStart()[q] - nI_ + i)] > 0) needRef_ = false;
    }
    if (needRef_)
        VLM_REQUIRE(ctrl_.p_ref_cell >= 0 && ctrl_.p_ref_cell < nC_, VLM_ERR_BAD_ARG, "reference cell out of range");
    {
        // the patches whose conditions fix the value, for the least-squares gradients (bc.fixesValue():
        // fixedValue, totalPressure, and mixed conditions with a positive value fraction somewhere;
        // inletOutlet's flags follow the flux at every gradient)
        std::vector<double> wu(nBb, 0.0), wp(nBb, 0.0);
        if (nB_ > 0) {
            VLM_CUDA(cudaMemcpyAsync(wu.data(), wIO_.get(), sizeof(double) * nBb, cudaMemcpyDeviceToHost, s_));
            VLM_CUDA(cudaMemcpyAsync(wp.data(), pFrac_.get(), sizeof(double) * nBb, cudaMemcpyDeviceToHost, s_));
            VLM_CUDA(cudaStreamSynchronize(s_));
        }
        std::vector<int32_t> uf(size_t(std::max(nP, 1)), 0), pf(size_t(std::max(nP, 1)), 0);
        for (int q = 0; q < nP; ++q) {
            uf[q] = uType[q] == 1 || (uType[q] == 8 && uRobinH_[2 * q] != 0.0);
            pf[q] = pType[q] == 1 || pType[q] == 7 || (pType[q] == 8 && pRobinH_[2 * q] != 0.0);
            for (int i = 0; i < G_.patchSize()[q]; ++i) {
                const size_t b = size_t(G_.patchStart()[q] - nI_ + i);
                if (uType[q] == 4 && wu[b] > 0) uf[q] = 1;
                if (pType[q] == 4 && wp[b] > 0) pf[q] = 1;
            }
        }
        uLsFix_.upload(uf, s_);
        pLsFix_.upload(pf, s_);
        VLM_CUDA(cudaStreamSynchronize(s_));
    }
    const size_t N = size_t(nC_), B = size_t(std::max(nB_, 1)), FI = size_t(std::max(nI_, 1)), F = size_t(nF_);
    for (DBuf<double>* b : {&U_, &U0_, &U00_, &src_, &msrc_, &HbyA_}) b->resize(3 * N);
    for (DBuf<double>* b : {&Ub_, &ic_, &bs_}) b->resize(3 * B);
    for (DBuf<double>* b : {&p_, &diag_, &rAU_, &divPhi_, &pPrev_, &fd_, &fb_, &pdiag_, &psrc_}) b->resize(N);
    for (DBuf<double>* b : {&pB_, &pic_, &pbs_}) b->resize(B);
    for (DBuf<double>* b : {&upper_, &lower_, &loDiv_, &upDiv_, &lapUp_}) b->resize(FI);
    for (DBuf<double>* b : {&cDiv_, &ffc_}) b->resize(3 * FI);
    for (DBuf<double>* b : {&phi_, &rAUf_, &phiHbyA_, &pffc_, &pflux_, &phiOld_, &phiOldOld_}) b->resize(F);
    pupper_.resize(FI);
    gU_.resize(9 * N);
    gP_.resize(3 * N);
    cont_.resize(1);
    if (G_.skewed()) {
        cSkew_.resize(3 * FI);
        gR_.resize(3 * N);
        gH_.resize(9 * N);
        hB_.resize(3 * size_t(std::max(nB_, 1)));
    }
    const int maxSolves = ctrl_.n_outer * (3 + ctrl_.n_corr * (ctrl_.n_non_orth_corr + 1));
    solveState_.resize(size_t(maxSolves));
    solveStatus_.resize(size_t(2) * maxSolves);
    VLM_CUDA(cudaHostAlloc(&pinned_, sizeof(double) + sizeof(SysState) * maxSolves + sizeof(int) * 2 * maxSolves,
                           cudaHostAllocDefault));
    for (DBuf<double>* b : {&U_, &U0_, &U00_, &p_, &phi_, &pffc_, &phiOld_, &phiOldOld_}) b->zero(s_);
    // VLM_FLOW_GRAPH=0: every step enqueued kernel by kernel (the captured steps' default is on)
    const char* fg = std::getenv("VLM_FLOW_GRAPH");
    graphOn_ = !(fg && fg[0] == '0');
}

DeviceFlow::~DeviceFlow() {
    stepGraphs_.clear();
    if (pinned_) cudaFreeHost(pinned_);
}

// Next record slot of this step; the solve writes its SysState and status words there.
// Next record slot(s) of this step: a solve of `group` systems writes one SysState per system into
// consecutive slots and its status words into the first slot's.
int DeviceFlow::solveSlot(bool momentum, bool monitoredP, int group) {
    const int k = nSolves_;
    nSolves_ += group;
    VLM_REQUIRE(size_t(nSolves_) <= solveState_.size(), VLM_ERR_CUDA, "internal: solve records exhausted");
    for (int j = 0; j < group; ++j) {
        if (momentum) uSolves_.push_back(k + j);
        solveGroup_.push_back(j == 0 ? group : 0);
    }
    if (monitoredP) pSolve_ = k;
    if (group > 1)
        VLM_CUDA(cudaMemsetAsync(solveStatus_.get() + 2 * (k + 1), 0, sizeof(int) * 2 * (group - 1), s_));
    (group > 1 ? *uBatch_ : batch_).deferNextSolve(solveState_.get() + k, solveStatus_.get() + 2 * k);
    return k;
}

// The solved velocity components as one batch (one system per component, the same topology): one
// set of launches for all components and their level-scheduled sweeps side by side, each system's
// result the one it would have alone.  Used when every component's sweeps fit one CTA in shared
// memory; larger meshes keep the component-by-component solves (their sweeps span the GPU).
bool DeviceFlow::componentBatch() {
    if (uBatchTried_) return uBatch_ != nullptr;
    uBatchTried_ = true;
    const int nc = int(solved_.size());
    const char* cb = std::getenv("VLM_COMPONENT_BATCH");
    if (nc < 2 || (cb && cb[0] == '0') || nC_ > 25000 || batch_.topology().size() != 1) return false;
    auto b = std::make_unique<DeviceBatch>(std::vector<SysTopo>(size_t(nc), batch_.topology()[0]),
                                           batch_.mergeLevels(), s_);
    if (!b->levelScheduleInSharedMemory(ctrl_.U)) return false;
    const size_t N = size_t(nC_), FI = size_t(std::max(nI_, 1));
    fdU_.resize(nc * N);
    fbU_.resize(nc * N);
    upU_.resize(nc * FI);
    loU_.resize(nc * FI);
    xU_.resize(nc * N);
    uBatch_ = std::move(b);
    return true;
}

void DeviceFlow::boundaryU() {
    if (nB_ > 0)
        k_u_boundary<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, nC_, nF_, G_.own(), G_.bPatch(), uType_.get(),
                                                uValueB_.get(), G_.Sf(), G_.magSf(), G_.ndc(), wIO_.get(),
                                                phi_.get(), uRobin_.get(), U_.get(), Ub_.get()), ++launches_;
}

void DeviceFlow::advectiveAdvance(int ddt, bool fromZero, bool noFlux) {
    adv_ = AdvStep{};
    if (!hasAdvective_ || nB_ == 0) return;
    adv_.on = true;
    if (ddt == 0 || !(dt_ > 0)) return;  // w = 0
    adv_.fromZero = fromZero;
    adv_.noFlux = noFlux;
    if (timeIndex_ != advLastTI_) {
        adv_.shift = true;
        adv_.shiftOldOld = advN_ >= 1;
        advN_ = std::min(advN_ + 1, 2);
        advLastTI_ = timeIndex_;
    }
    // ddtCoeffs (Schemes.h:71-86) with the condition's own old-old level
    const double rDt = 1.0 / dt_;
    if (ddt == 2 && advN_ >= 2 && dt0_ > 0) {
        const double ct = 1.0 + dt_ / (dt_ + dt0_);
        const double ct00 = dt_ * dt_ / (dt0_ * (dt_ + dt0_));
        adv_.c = ct * rDt;
        adv_.c0 = (ct + ct00) * rDt;
        adv_.c00 = ct00 * rDt;
    } else {
        adv_.c = adv_.c0 = rDt;
    }
}

void DeviceFlow::advectiveApply() {
    if (!adv_.on) return;
    if (adv_.c == 0.0) {
        k_adv_steady<<<nblk(nB_), 256, 0, s_>>>(nB_, G_.bPatch(), uType_.get(), wIO_.get()), ++launches_;
        return;
    }
    k_adv_update<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, G_.bPatch(), uType_.get(), adv_.noFlux ? nullptr : phi_.get(),
                                            G_.magSf(), G_.ndc(), Ub_.get(), advOld_.get(), advOldOld_.get(),
                                            uAdv_.get(), adv_.shift ? 1 : 0, adv_.shiftOldOld ? 1 : 0, adv_.fromZero ? 1 : 0,
                                            adv_.c, adv_.c0, adv_.c00, wIO_.get(), uValueB_.get()),
        ++launches_;
}

void DeviceFlow::ioFractions() {
    if (hasInletOutlet_ && nB_ > 0)
        k_io_fraction<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, G_.bPatch(), uType_.get(), phi_.get(), wIO_.get()),
            ++launches_;
}

void DeviceFlow::totalPressure(bool noFlux) {
    if (hasTotalPressure_ && nB_ > 0)
        k_total_pressure<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, G_.bPatch(), pType_.get(), noFlux ? nullptr : phi_.get(),
                                                    Ub_.get(), pTotal_.get(), pValueB_.get()), ++launches_;
}

void DeviceFlow::setBoundaryValues(const double* uFace, const double* pFace) {
    const size_t nBb = size_t(std::max(nB_, 1));
    if (uFace && nB_ > 0) {
        std::vector<double> uv(3 * nBb);
        VLM_CUDA(cudaMemcpyAsync(uv.data(), uValueB_.get(), sizeof(double) * uv.size(), cudaMemcpyDeviceToHost, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
        for (int q = 0; q < G_.nPatches(); ++q) {
            if (uTypeHost_[q] != 1 && uTypeHost_[q] != 3) continue;
            for (int i = 0; i < G_.patchSize()[q]; ++i) {
                const size_t b = size_t(G_.patchStart()[q] - nI_ + i);
                for (int k = 0; k < 3; ++k) uv[k * nBb + b] = uFace[3 * b + k];
            }
        }
        uValueB_.upload(uv, s_);
    }
    if (pFace && nB_ > 0) {
        std::vector<double> pv(nBb);
        VLM_CUDA(cudaMemcpyAsync(pv.data(), pValueB_.get(), sizeof(double) * pv.size(), cudaMemcpyDeviceToHost, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
        for (int q = 0; q < G_.nPatches(); ++q) {
            if (pTypeHost_[q] != 1) continue;
            for (int i = 0; i < G_.patchSize()[q]; ++i) {
                const size_t b = size_t(G_.patchStart()[q] - nI_ + i);
                pv[b] = pFace[b];
            }
        }
        pValueB_.upload(pv, s_);
    }
    boundaryU();
    boundaryP();
    VLM_CUDA(cudaStreamSynchronize(s_));
}

void DeviceFlow::boundaryP() {
    ScalarBC bc;
    bc.type = pTypeAsm_.data();
    bc.value = pValueB_.get();
    bc.frac = pFrac_.get();
    bc.lsFix = pLsFix_.get();
    bc.robin = pRobin_.get();
    G_.correctBoundary(p_.get(), bc, pB_.get(), s_);
}

void DeviceFlow::gradU() {
    if (ctrl_.grad_scheme == 1) {
        if ((hasInletOutlet_ || hasAdvective_) && nB_ > 0) {
            k_io_patch_reset<<<nblk(G_.nPatches()), 256, 0, s_>>>(G_.nPatches(), uType_.get(), uLsFix_.get()),
                ++launches_;
            k_io_patch_fix<<<nblk(nB_), 256, 0, s_>>>(nB_, G_.bPatch(), uType_.get(), wIO_.get(), uLsFix_.get()),
                ++launches_;
        }
        k_grad_ls_u<<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, nF_, nB_, G_.cellFaceOff(), G_.cellFaces(), G_.own(),
                                               G_.nei(), G_.Sf(), G_.magSf(), G_.d(), G_.ndc(), U_.get(), Ub_.get(),
                                               G_.bPatch(), uType_.get(), uLsFix_.get(), uValueB_.get(), wIO_.get(),
                                               phi_.get(), uRobin_.get(), G_.twoD(), G_.emptyDir(), gU_.get()),
            ++launches_;
        return;
    }
    k_grad_tensor<<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, nB_, nF_, G_.cellFaceOff(), G_.cellFaces(), G_.own(), G_.nei(),
                                            G_.w(), G_.Sf(), G_.V(), U_.get(), Ub_.get(), G_.twoD(), G_.emptyDir(),
                                            gU_.get()), ++launches_;
}

void DeviceFlow::setState(const double* U, const double* p) {
    if (U) {
        DBuf<double> tmp;
        tmp.upload(U, size_t(3) * nC_, s_);
        k_soa_from_aos<<<nblk(nC_), 256, 0, s_>>>(nC_, tmp.get(), U_.get()), ++launches_;
        VLM_CUDA(cudaStreamSynchronize(s_));
    }
    if (p) p_.upload(p, size_t(nC_), s_);
    // initialize(): no flux yet, every inletOutlet face evaluates as outflow (the freestream fractions stay)
    if (hasInletOutlet_ && nB_ > 0)
        k_io_fraction<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, G_.bPatch(), uType_.get(), nullptr, wIO_.get()),
            ++launches_;
    // advective faces: a fresh condition (no history) on a fresh field (boundary values 0), updated
    // with the context's initial Euler scheme and no flux
    advN_ = 0;
    advLastTI_ = -1;
    advectiveAdvance(1, true, true);
    advectiveApply();
    totalPressure(true);
    boundaryU();
    boundaryP();
    if (G_.skewed()) gradU();
    k_flux_u<<<nblk(nF_), 256, 0, s_>>>(nF_, nI_, nB_, nC_, G_.own(), G_.nei(), G_.w(), G_.Sf(), U_.get(), Ub_.get(),
                                       G_.skewed() ? G_.skew() : nullptr, gU_.get(), phi_.get()), ++launches_;
    rAU_.zero(s_);
    VLM_CUDA(cudaGetLastError());
    VLM_CUDA(cudaStreamSynchronize(s_));
    initialized_ = true;
}

void DeviceFlow::getState(double* U, double* p, double* phi) {
    if (U) {
        DBuf<double> tmp(size_t(3) * nC_);
        k_aos_from_soa<<<nblk(nC_), 256, 0, s_>>>(nC_, U_.get(), tmp.get()), ++launches_;
        VLM_CUDA(cudaMemcpyAsync(U, tmp.get(), sizeof(double) * 3 * nC_, cudaMemcpyDeviceToHost, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
    }
    if (p) VLM_CUDA(cudaMemcpyAsync(p, p_.get(), sizeof(double) * nC_, cudaMemcpyDeviceToHost, s_));
    if (phi) VLM_CUDA(cudaMemcpyAsync(phi, phi_.get(), sizeof(double) * nF_, cudaMemcpyDeviceToHost, s_));
    VLM_CUDA(cudaStreamSynchronize(s_));
}

// ---------------------------------------------------------------- restart (io/Restart.cpp)
namespace {
constexpr uint64_t kRestartMagic = 0x4346445253543031ull;  // "CFDRST01"

// writeGlobal (Restart.cpp:15-22): magic, count, components, then the doubles
void writeRestartArray(const std::string& file, const std::vector<double>& g, uint64_t n, int nc) {
    std::ofstream os(file, std::ios::binary);
    VLM_REQUIRE(bool(os), VLM_ERR_BAD_ARG, "cannot write " + file);
    const uint64_t h[3] = {kRestartMagic, n, uint64_t(nc)};
    os.write(reinterpret_cast<const char*>(h), sizeof(h));
    os.write(reinterpret_cast<const char*>(g.data()), std::streamsize(g.size() * sizeof(double)));
    VLM_REQUIRE(bool(os), VLM_ERR_BAD_ARG, "cannot write " + file);
}

// readGlobal (Restart.cpp:25-43): false when the file is absent, an error when it does not fit
bool readRestartArray(const std::string& file, uint64_t n, int nc, std::vector<double>& g) {
    std::ifstream is(file, std::ios::binary);
    if (!is) return false;
    uint64_t h[3] = {0, 0, 0};
    is.read(reinterpret_cast<char*>(h), sizeof(h));
    VLM_REQUIRE(h[0] == kRestartMagic && h[1] == n && h[2] == uint64_t(nc), VLM_ERR_BAD_ARG,
                "restart file " + file + " does not match the mesh");
    g.resize(size_t(n) * size_t(nc));
    is.read(reinterpret_cast<char*>(g.data()), std::streamsize(g.size() * sizeof(double)));
    VLM_REQUIRE(bool(is), VLM_ERR_BAD_ARG, "restart file " + file + " is truncated");
    return true;
}
}  // namespace

// restart::write (Restart.cpp:105-132): cell arrays in cell order (vectors as 3 doubles per cell),
// face arrays in face order (one rank: the global orders), and the time / forcing state as text
void DeviceFlow::writeRestart(const std::string& dir) {
    std::filesystem::create_directories(dir);
    const size_t N = size_t(nC_), F = size_t(nF_);
    auto cellVec = [&](const DBuf<double>& soa) {
        DBuf<double> tmp(3 * N);
        k_aos_from_soa<<<nblk(nC_), 256, 0, s_>>>(nC_, soa.get(), tmp.get()), ++launches_;
        std::vector<double> h(3 * N);
        VLM_CUDA(cudaMemcpyAsync(h.data(), tmp.get(), sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
        return h;
    };
    auto plain = [&](const double* d, size_t n) {
        std::vector<double> h(n);
        VLM_CUDA(cudaMemcpyAsync(h.data(), d, sizeof(double) * n, cudaMemcpyDeviceToHost, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
        return h;
    };
    writeRestartArray(dir + "/U.bin", cellVec(U_), N, 3);
    writeRestartArray(dir + "/p.bin", plain(p_.get(), N), N, 1);
    writeRestartArray(dir + "/phi.bin", plain(phi_.get(), F), F, 1);
    if (nOld_ >= 1) {
        writeRestartArray(dir + "/U_0.bin", cellVec(U0_), N, 3);
        writeRestartArray(dir + "/phi_0.bin", plain(phiOld_.get(), F), F, 1);
    }
    if (nOld_ >= 2) {
        writeRestartArray(dir + "/U_00.bin", cellVec(U00_), N, 3);
        writeRestartArray(dir + "/phi_00.bin", plain(phiOldOld_.get(), F), F, 1);
    }
    if (les_) writeRestartArray(dir + "/nut.bin", plain(nut_.get(), N), N, 1);
    double gradP = 0.0;
    if (forcing_ == 2) gradP = plain(forceState_.get(), 1)[0];
    std::ofstream os(dir + "/state.txt");
    VLM_REQUIRE(bool(os), VLM_ERR_BAD_ARG, "cannot write " + dir + "/state.txt");
    os << std::setprecision(17);
    os << "time " << time_ << "\ndt " << dt_ << "\ndt0 " << dt0_ << "\ntimeIndex " << timeIndex_ << "\nnOldTimes "
       << nOld_ << "\ngradP " << gradP << '\n';
    VLM_REQUIRE(bool(os), VLM_ERR_BAD_ARG, "cannot write " + dir + "/state.txt");
}

// restart::read (Restart.cpp:134-190) followed by markRestarted (IncompressibleFlow.cpp:41-47)
bool DeviceFlow::readRestart(const std::string& dir) {
    std::ifstream st(dir + "/state.txt");
    if (!st) return false;
    std::map<std::string, double> kv;
    {
        std::string k;
        double v;
        while (st >> k >> v) kv[k] = v;
    }
    const size_t N = size_t(nC_), F = size_t(nF_);
    std::vector<double> g;
    auto cellVec = [&](const std::string& f, DBuf<double>& soa) {
        if (!readRestartArray(f, N, 3, g)) return;
        DBuf<double> tmp;
        tmp.upload(g, s_);
        k_soa_from_aos<<<nblk(nC_), 256, 0, s_>>>(nC_, tmp.get(), soa.get()), ++launches_;
        VLM_CUDA(cudaStreamSynchronize(s_));
    };
    auto plain = [&](const std::string& f, DBuf<double>& d, size_t n) {
        if (!readRestartArray(f, n, 1, g)) return;
        VLM_CUDA(cudaMemcpyAsync(d.get(), g.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
    };
    cellVec(dir + "/U.bin", U_);
    plain(dir + "/p.bin", p_, N);
    plain(dir + "/phi.bin", phi_, F);
    const int nOld = int(kv["nOldTimes"]);
    if (nOld >= 1) {
        U0_.zero(s_);
        phiOld_.zero(s_);
        cellVec(dir + "/U_0.bin", U0_);
        plain(dir + "/phi_0.bin", phiOld_, F);
    }
    if (nOld >= 2) {
        U00_.zero(s_);
        phiOldOld_.zero(s_);
        cellVec(dir + "/U_00.bin", U00_);
        plain(dir + "/phi_00.bin", phiOldOld_, F);
    }
    nOld_ = nOld;
    if (les_) plain(dir + "/nut.bin", nut_, N);
    time_ = kv["time"];
    dt_ = kv["dt"];
    dt0_ = kv["dt0"];
    timeIndex_ = int(kv["timeIndex"]);
    if (forcing_ == 2) {
        const double gp = kv["gradP"];
        VLM_CUDA(cudaMemcpyAsync(forceState_.get(), &gp, sizeof(double), cudaMemcpyHostToDevice, s_));
        VLM_CUDA(cudaStreamSynchronize(s_));
    }
    ioFractions();  // markRestarted: updateBCs with the restart's flux
    // a fresh advective condition on a fresh field, with the context's initial Euler scheme
    advN_ = 0;
    advLastTI_ = -1;
    advectiveAdvance(1, true, false);
    advectiveApply();
    totalPressure(false);
    boundaryU();
    boundaryP();
    VLM_CUDA(cudaStreamSynchronize(s_));
    initialized_ = true;
    return true;
}

// UEqn = ddt + div(phi, U) - laplacian(nu, U), relaxed by aU (IncompressibleFlow.cpp:176-198)
void DeviceFlow::assembleMomentum(double aU, bool haveGradU) {
    // skewed mesh: linear and LUST add an explicit skew correction from grad U (Fvm.h:83-84)
    const bool skewLin = G_.skewed() && (ctrl_.div_scheme == kLinear || ctrl_.div_scheme == kLUST);
    const bool needG = ctrl_.div_scheme >= kLinearUpwind || G_.nonOrthogonal() || skewLin;
    if (needG && !haveGradU) gradU();
    const double* nuF = les_ ? nuF_.get() : nullptr;
    if (nI_ > 0)
        k_mom_faces<<<nblk(nI_), 256, 0, s_>>>(nI_, nC_, nF_, G_.own(), G_.nei(), G_.w(), G_.magSf(), G_.ndc(), G_.d(),
                                              G_.corr(), G_.C(), G_.Cf(), phi_.get(), ctrl_.nu, nuF, ctrl_.div_scheme,
                                              ctrl_.div_coeff, U_.get(), G_.nonOrthogonal() ? 1 : 0, gU_.get(),
                                              skewLin ? G_.skew() : nullptr, loDiv_.get(), upDiv_.get(),
                                              lapUp_.get(), upper_.get(), lower_.get(), cDiv_.get(),
                                              skewLin ? cSkew_.get() : nullptr, ffc_.get()), ++launches_;
    if (nB_ > 0)
        k_mom_bfaces<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, nC_, nF_, G_.own(), G_.bPatch(), uType_.get(),
                                               uValueB_.get(), wIO_.get(), uRobin_.get(), G_.Sf(), G_.magSf(), G_.ndc(),
                                               phi_.get(), ctrl_.nu,
                                               nuF, U_.get(), ic_.get(), bs_.get()), ++launches_;
    // ddt coefficients (Schemes.h:70-86)
    double kc = 0, kc0 = 0, kc00 = 0;
    const bool transient = !ctrl_.steady;
    if (transient) {
        const double rDt = 1.0 / dt_;
        if (ctrl_.ddt_scheme == 2 && nOld_ >= 2 && dt0_ > 0) {
            const double ct = 1.0 + dt_ / (dt_ + dt0_);
            const double ct00 = dt_ * dt_ / (dt0_ * (dt_ + dt0_));
            kc = ct * rDt;
            kc0 = (ct + ct00) * rDt;
            kc00 = ct00 * rDt;
        } else {
            kc = kc0 = rDt;
        }
    }
    k_mom_cells<<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, G_.cellFaceOff(), G_.cellFaces(), loDiv_.get(), upDiv_.get(),
                                          lapUp_.get(), cDiv_.get(), skewLin && nI_ > 0 ? cSkew_.get() : nullptr,
                                          ffc_.get(), G_.V(), transient ? 1 : 0, kc, kc0,
                                          kc00, U0_.get(), nOld_ >= 2 ? U00_.get() : U0_.get(), diag_.get(),
                                          src_.get()), ++launches_;
    if (les_ || forcing_ != 0) explicitSources();
    if (aU < 1.0)
        k_mom_relax<<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, nB_, G_.cellFaceOff(), G_.cellFaces(), upper_.get(),
                                              lower_.get(), ic_.get(), U_.get(), aU, diag_.get(), src_.get()), ++launches_;
    VLM_CUDA(cudaGetLastError());
}

// Momentum predictor: M = UEqn + grad p, one solve per solved component (FvMatrix.h:144-175)
void DeviceFlow::solveMomentum(vlm_step_info& info, bool first) {
    ScalarBC pbc;
    pbc.type = pTypeAsm_.data();
    pbc.value = pValueB_.get();
    pbc.frac = pFrac_.get();
    pbc.lsFix = pLsFix_.get();
    pbc.robin = pRobin_.get();
    G_.grad(p_.get(), pB_.get(), pbc, ctrl_.grad_p_scheme, gP_.get(), s_);
    k_mom_gradp<<<nblk(nC_), 256, 0, s_>>>(nC_, src_.get(), gP_.get(), G_.V(), msrc_.get()), ++launches_;
    const size_t N = size_t(nC_), B = size_t(std::max(nB_, 1));
    if (componentBatch()) {
        const int nc = int(solved_.size());
        const size_t FI = size_t(std::max(nI_, 1));
        bool contiguous = true;
        for (int i = 0; i < nc; ++i) contiguous = contiguous && solved_[i] == solved_[0] + i;
        for (int i = 0; i < nc; ++i) {
            const int k = solved_[i];
            G_.fold(diag_.get(), msrc_.get() + k * N, ic_.get() + k * B, bs_.get() + k * B, fdU_.get() + i * N,
                    fbU_.get() + i * N, s_);
            if (nI_ > 0) {
                VLM_CUDA(cudaMemcpyAsync(upU_.get() + i * FI, upper_.get(), sizeof(double) * nI_,
                                         cudaMemcpyDeviceToDevice, s_));
                VLM_CUDA(cudaMemcpyAsync(loU_.get() + i * FI, lower_.get(), sizeof(double) * nI_,
                                         cudaMemcpyDeviceToDevice, s_));
            }
            if (!contiguous)
                VLM_CUDA(cudaMemcpyAsync(xU_.get() + i * N, U_.get() + k * N, sizeof(double) * N,
                                         cudaMemcpyDeviceToDevice, s_));
        }
        double* x = contiguous ? U_.get() + solved_[0] * N : xU_.get();
        std::vector<vlm_solver_perf> pf;
        solveSlot(first, false, nc);
        uBatch_->solve(fdU_.get(), upU_.get(), loU_.get(), fbU_.get(), x, ctrl_.U, pf);
        solveLaunches_.push_back(uBatch_->lastDeferred());
        for (int i = 1; i < nc; ++i) solveLaunches_.push_back(DeviceBatch::LaunchCount{});
        if (!contiguous)
            for (int i = 0; i < nc; ++i)
                VLM_CUDA(cudaMemcpyAsync(U_.get() + solved_[i] * N, xU_.get() + i * N, sizeof(double) * N,
                                         cudaMemcpyDeviceToDevice, s_));
    } else {
        for (int k : solved_) {
            G_.fold(diag_.get(), msrc_.get() + k * N, ic_.get() + k * B, bs_.get() + k * B, fd_.get(), fb_.get(),
                    s_);
            std::vector<vlm_solver_perf> pf;
            solveSlot(first, false);
            batch_.solve(fd_.get(), upper_.get(), lower_.get(), fb_.get(), U_.get() + k * N, ctrl_.U, pf);
            solveLaunches_.push_back(batch_.lastDeferred());
        }
    }
    (void)info;
    boundaryU();
}

// One pressure correction (IncompressibleFlow.cpp:244-362)
void DeviceFlow::correctPressure(bool finalCorr, bool first, vlm_step_info& info) {
    k_mom_AH<<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, nB_, G_.cellFaceOff(), G_.cellFaces(), G_.own(), G_.nei(),
                                       diag_.get(), upper_.get(), lower_.get(), ic_.get(), bs_.get(), src_.get(),
                                       U_.get(), G_.V(), rAU_.get(), HbyA_.get()), ++launches_;
    ScalarBC pbc;
    pbc.type = pTypeAsm_.data();
    pbc.value = pValueB_.get();
    pbc.frac = pFrac_.get();
    pbc.lsFix = pLsFix_.get();
    pbc.robin = pRobin_.get();
    const bool skewed = G_.skewed();
    if (skewed) {
        // skewed mesh (IncompressibleFlow.cpp:252-275): grad rAU by least squares with zero-gradient
        // boundaries; grad HbyA by least squares with the fixes-flux faces at U_b + rAU_P grad p_P
        G_.grad(p_.get(), pB_.get(), pbc, ctrl_.grad_p_scheme, gP_.get(), s_);
        if (nB_ > 0)
            k_hbya_bval<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, G_.own(), G_.bPatch(), uFixesFlux_.get(), Ub_.get(),
                                                  rAU_.get(), gP_.get(), hB_.get()), ++launches_;
        k_grad_ls_cells<1><<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, nF_, nB_, G_.cellFaceOff(), G_.cellFaces(), G_.own(),
                                                     G_.nei(), G_.Sf(), G_.magSf(), G_.d(), rAU_.get(), nullptr,
                                                     G_.bPatch(), nullptr, G_.twoD(), G_.emptyDir(), gR_.get()),
            ++launches_;
        k_grad_ls_cells<3><<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, nF_, nB_, G_.cellFaceOff(), G_.cellFaces(), G_.own(),
                                                     G_.nei(), G_.Sf(), G_.magSf(), G_.d(), HbyA_.get(), hB_.get(),
                                                     G_.bPatch(), uFixesFlux_.get(), G_.twoD(), G_.emptyDir(),
                                                     gH_.get()),
            ++launches_;
    }
    k_phi_hbya<<<nblk(nF_), 256, 0, s_>>>(nF_, nI_, nB_, nC_, G_.own(), G_.nei(), G_.w(), G_.Sf(), G_.bPatch(),
                                         uFixesFlux_.get(), rAU_.get(), HbyA_.get(), Ub_.get(),
                                         skewed ? G_.skew() : nullptr, gR_.get(), gH_.get(), rAUf_.get(),
                                         phiHbyA_.get()), ++launches_;
    if (hasFluxPressure_ && nB_ > 0)
        k_flux_pressure<<<nblk(nB_), 256, 0, s_>>>(nB_, nI_, nF_, G_.bPatch(), pType_.get(), phiHbyA_.get(), Ub_.get(),
                                                   G_.Sf(), G_.magSf(), rAUf_.get(), pValueB_.get()), ++launches_;
    G_.div(phiHbyA_.get(), divPhi_.get(), s_);
    if (ctrl_.steady) VLM_CUDA(cudaMemcpyAsync(pPrev_.get(), p_.get(), sizeof(double) * nC_, cudaMemcpyDeviceToDevice, s_));
    const int nNO = ctrl_.n_non_orth_corr;
    for (int no = 0; no <= nNO; ++no) {
        const bool finalNO = no == nNO;
        bool hasFfc = false;
        G_.laplacian(rAUf_.get(), p_.get(), pB_.get(), pbc, true, ctrl_.grad_scheme, pdiag_.get(), pupper_.get(), psrc_.get(),
                     pic_.get(), pbs_.get(), pffc_.get(), &hasFfc, s_);
        G_.addVolumeSource(psrc_.get(), divPhi_.get(), s_);
        if (needRef_) G_.setReference(ctrl_.p_ref_cell, ctrl_.p_ref_value, pdiag_.get(), psrc_.get(), s_);
        G_.fold(pdiag_.get(), psrc_.get(), pic_.get(), pbs_.get(), fd_.get(), fb_.get(), s_);
        std::vector<vlm_solver_perf> pf;
        solveSlot(false, first && no == 0);
        batch_.solve(fd_.get(), pupper_.get(), pupper_.get(), fb_.get(), p_.get(),
                     (finalCorr && finalNO) ? ctrl_.p_final : ctrl_.p, pf);
        solveLaunches_.push_back(batch_.lastDeferred());
        boundaryP();
        if (finalNO) {
            G_.flux(pupper_.get(), p_.get(), pic_.get(), pbs_.get(), hasFfc ? pffc_.get() : nullptr, pflux_.get(), s_);
            k_phi_update<<<nblk(nF_), 256, 0, s_>>>(nF_, phiHbyA_.get(), pflux_.get(), phi_.get()), ++launches_;
        }
    }
    if (ctrl_.steady && ctrl_.alpha_p < 1.0) {
        k_p_relax<<<nblk(nC_), 256, 0, s_>>>(nC_, pPrev_.get(), ctrl_.alpha_p, p_.get()), ++launches_;
        boundaryP();
    }
    G_.grad(p_.get(), pB_.get(), pbc, ctrl_.grad_p_scheme, gP_.get(), s_);
    k_u_correct<<<nblk(nC_), 256, 0, s_>>>(nC_, HbyA_.get(), rAU_.get(), gP_.get(), G_.twoD(), G_.emptyDir(),
                                          U_.get()), ++launches_;
    boundaryU();
    VLM_CUDA(cudaGetLastError());
}

// The device work of one step (everything the host enqueues between the time-state update and the
// read-back of the step's records); records its bookkeeping in nSolves_, uSolves_, pSolve_,
// solveLaunches_.
void DeviceFlow::stepWork(bool copyOld, bool copyOldOld) {
    vlm_step_info info;
    std::memset(&info, 0, sizeof info);
    const bool steady = ctrl_.steady != 0;
    // VolField::storeOld (VolField.h:114-118) and phiOldOld = phiOld, phiOld = phi (IncompressibleFlow.cpp:150-152)
    if (copyOldOld) {
        VLM_CUDA(cudaMemcpyAsync(U00_.get(), U0_.get(), sizeof(double) * 3 * nC_, cudaMemcpyDeviceToDevice, s_));
        VLM_CUDA(cudaMemcpyAsync(phiOldOld_.get(), phiOld_.get(), sizeof(double) * nF_, cudaMemcpyDeviceToDevice, s_));
    }
    if (copyOld) {
        VLM_CUDA(cudaMemcpyAsync(U0_.get(), U_.get(), sizeof(double) * 3 * nC_, cudaMemcpyDeviceToDevice, s_));
        VLM_CUDA(cudaMemcpyAsync(phiOld_.get(), phi_.get(), sizeof(double) * nF_, cudaMemcpyDeviceToDevice, s_));
    }
    ioFractions();
    advectiveApply();
    totalPressure(false);  // p_.updateBCs reads U's boundary values of the previous step
    boundaryU();
    boundaryP();
    nSolves_ = 0;
    uSolves_.clear();
    solveLaunches_.clear();
    solveGroup_.clear();
    pSolve_ = -1;
    for (int outer = 0; outer < ctrl_.n_outer; ++outer) {
        const bool finalOuter = outer == ctrl_.n_outer - 1;
        const double aU = steady ? ctrl_.alpha_u : (finalOuter ? 1.0 : ctrl_.alpha_u);
        // updateGradU + updateTurbulence at the start of every outer pass (IncompressibleFlow.cpp:176-179)
        if (les_) {
            gradU();
            lesCorrect();
        }
        assembleMomentum(aU, les_);
        if (ctrl_.momentum_predictor) solveMomentum(info, outer == 0);
        for (int corr = 0; corr < ctrl_.n_corr; ++corr)
            correctPressure(finalOuter && corr == ctrl_.n_corr - 1, outer == 0 && corr == 0, info);
        if (forcing_ == 2) forcingCorrection(aU);
    }
    // continuity error: max |div phi| (IncompressibleFlow.cpp:367-370)
    G_.div(phi_.get(), divPhi_.get(), s_);
    cont_.zero(s_);
    k_max_abs<<<std::min(nblk(nC_), 1184), 256, 0, s_>>>(nC_, divPhi_.get(), (unsigned long long*)cont_.get()), ++launches_;
}

// One step's device work captured into a graph (the solves' iteration loops embedded as conditional
// nodes); returns null when the capture is not possible, and the step then runs directly.
DeviceFlow::StepGraph* DeviceFlow::stepGraph(bool copyOld, bool copyOldOld) {
    const StepKey key{ctrl_.steady != 0, dt_,         dt0_,     copyOld,   copyOldOld, adv_.shift,
                      adv_.shiftOldOld,  adv_.c, adv_.c0, adv_.c00};
    for (auto& g : stepGraphs_)
        if (g->key == key) return g.get();
    auto g = std::make_unique<StepGraph>();
    g->key = key;
    const int64_t own0 = launches_, geom0 = G_.launches();
    VLM_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeRelaxed));
    batch_.beginEmbedding();
    if (uBatch_) uBatch_->beginEmbedding();
    try {
        stepWork(copyOld, copyOldOld);
    } catch (...) {
        batch_.endEmbedding();
        if (uBatch_) uBatch_->endEmbedding();
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(s_, &junk);
        if (junk) cudaGraphDestroy(junk);
        cudaGetLastError();
        graphOn_ = false;
        return nullptr;
    }
    batch_.endEmbedding();
    if (uBatch_) uBatch_->endEmbedding();
    VLM_CUDA(cudaStreamEndCapture(s_, &g->graph));
    VLM_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
    g->ownLaunches = (launches_ - own0) + (G_.launches() - geom0);
    g->nSolves = nSolves_;
    g->uSolves = uSolves_;
    g->pSolve = pSolve_;
    g->solveLaunches = solveLaunches_;
    g->solveGroup = solveGroup_;
    stepGraphs_.push_back(std::move(g));
    return stepGraphs_.back().get();
}

DeviceFlow::StepGraph::~StepGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
}

vlm_step_info DeviceFlow::step(double dt) {
    if (!initialized_) setState(nullptr, nullptr);
    vlm_step_info info;
    std::memset(&info, 0, sizeof info);
    const bool steady = ctrl_.steady != 0;
    bool copyOld = false, copyOldOld = false;
    if (!steady) {
        VLM_REQUIRE(dt > 0, VLM_ERR_BAD_ARG, "dt must be positive");
        dt0_ = timeIndex_ > 0 ? dt_ : -1.0;
        dt_ = dt;
        time_ += dt;
        ++timeIndex_;
        copyOldOld = nOld_ >= 1;
        copyOld = true;
        nOld_ = std::min(nOld_ + 1, 2);
    } else {
        time_ += 1.0;
        ++timeIndex_;
    }
    advectiveAdvance(steady ? 0 : ctrl_.ddt_scheme, false, false);
    // The first step runs directly (it creates every lazily built resource); later steps replay one
    // captured graph per (steady, dt, old-time-level) configuration: one launch per step.
    StepGraph* sg = nullptr;
    if (graphOn_ && stepsRun_ >= 1 && batch_.embeddable() && (!uBatch_ || uBatch_->embeddable()))
        sg = stepGraph(copyOld, copyOldOld);
    int64_t stepOwn = 0;
    if (sg) {
        VLM_CUDA(cudaGraphLaunch(sg->exec, s_));
        nSolves_ = sg->nSolves;
        uSolves_ = sg->uSolves;
        pSolve_ = sg->pSolve;
        solveLaunches_ = sg->solveLaunches;
        solveGroup_ = sg->solveGroup;
        stepOwn = sg->ownLaunches;
    } else {
        const int64_t own0 = launches_, geom0 = G_.launches();
        stepWork(copyOld, copyOldOld);
        stepOwn = (launches_ - own0) + (G_.launches() - geom0);
    }
    ++stepsRun_;
    // the step's continuity error and solver records, read once into pinned memory (a copy into
    // pageable memory would block in the driver until the stream drains, serialising concurrent flows)
    double* hCont = reinterpret_cast<double*>(pinned_);
    SysState* hSt = reinterpret_cast<SysState*>(hCont + 1);
    int* hStatus = reinterpret_cast<int*>(hSt + solveState_.size());
    VLM_CUDA(cudaMemcpyAsync(hCont, cont_.get(), sizeof(double), cudaMemcpyDeviceToHost, s_));
    if (nSolves_ > 0) {
        VLM_CUDA(cudaMemcpyAsync(hSt, solveState_.get(), sizeof(SysState) * nSolves_, cudaMemcpyDeviceToHost, s_));
        VLM_CUDA(cudaMemcpyAsync(hStatus, solveStatus_.get(), sizeof(int) * 2 * nSolves_, cudaMemcpyDeviceToHost, s_));
    }
    VLM_CUDA(cudaStreamSynchronize(s_));
    VLM_CUDA(cudaGetLastError());
    info.continuityError = *hCont;
    const std::vector<SysState> st(hSt, hSt + nSolves_);
    const std::vector<int> status(hStatus, hStatus + 2 * nSolves_);
    for (int k = 0; k < nSolves_; ++k) {
        if (status[2 * k + 1] != 0) {
            batch_.clearLevelError();
            if (uBatch_) uBatch_->clearLevelError();
            throw Error(VLM_ERR_TIMEOUT, "level-scheduled sweep: a group barrier wait gave up");
        }
        if (status[2 * k] == VLM_ERR_SINGULAR) throw Error(VLM_ERR_SINGULAR, "GAMG: singular coarsest matrix");
        info.iterations += st[k].iterations;
    }
    int64_t launched = stepOwn;
    for (int k = 0; k < nSolves_ && k < int(solveLaunches_.size()); ++k) {
        const auto& c = solveLaunches_[k];
        // a batched solve loops until its last system is done
        int its = st[k].iterations;
        const int g = k < int(solveGroup_.size()) ? solveGroup_[k] : 1;
        for (int j = 1; j < g && k + j < nSolves_; ++j) its = std::max(its, st[k + j].iterations);
        launched += c.eager + c.pre + int64_t(its) * c.body;
    }
    info.launches = int32_t(launched);
    total_ += launched;
    // monitored residuals (IncompressibleFlow.cpp:205-213, 320-327)
    if (!uSolves_.empty()) {
        double r = 0, nf = 0;
        for (int k : uSolves_) {
            r = std::max(r, st[k].residualSum);
            nf = std::max(nf, st[k].normFactor);
        }
        info.UInitialResidual = r / (nf + 1e-30);
    }
    if (pSolve_ >= 0) {
        const SysState& q = st[pSolve_];
        if (pNormSteps_ < 5) {
            pNormRef_ = std::max(pNormRef_, q.normFactor);
            ++pNormSteps_;
        }
        info.pInitialResidual = q.residualSum / (std::max(q.normFactor, pNormRef_) + 1e-30);
    }
    return info;
}

}  // namespace vlm
