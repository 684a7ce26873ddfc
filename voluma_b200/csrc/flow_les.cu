// Turbulence model and momentum forcing of the device flow (flow.h):
//
//   * the LES Smagorinsky model with optional Van Driest damping, as TurbulenceModel::correct
//     (TurbulenceModel.cpp:226-250) runs it for a wall-resolved LES model: wall faces and their
//     friction velocity (updateWallFaces, TurbulenceModel.cpp:199-216; LESModel::correctModel,
//     LESModels.cpp:64-153 without a wall model), the damped filter width
//     min(Delta, kappa/Cdelta y (1 - exp(-y+/A+))) with the nearest wall face of every cell
//     (WallDistance.cpp), nu_t = (Cs Delta)^2 sqrt(2 S:S) (LESModels.cpp:274-287), the nu_t limiter, and
//     the face nu_eff (IncompressibleFlow::nuEffFaces, IncompressibleFlow.cpp:83-95);
//   * the explicit momentum source div(nu_eff dev2(T(grad U))) (IncompressibleFlow.cpp:186-196);
//   * the momentum forcing: a constant body force or the mean-velocity forcing with its per-outer-pass
//     correction (IncompressibleFlow.cpp:115-142, 198-202, 363).
//
// Every cell and face loop keeps the reference's operation order, so with exact sums (reproducible
// mode) the laminar-plus-forcing step and the undamped Smagorinsky step are the reference's bit for
// bit; the Van Driest damping calls exp(), whose last bit may differ between CUDA and the host
// library.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "exactsum.cuh"
#include "flow.h"
#include "walldist.h"

namespace vlm {
namespace {

inline int nblk(int n, int t = 256) { return (n + t - 1) / t; }

constexpr int kForceThreads = 256;
constexpr int kForceWarps = kForceThreads / 32;
constexpr int kForceCtas = 296;

// updateWallFaces + the wall-resolved branch of correctModel: per wall face the tangential velocity
// relative to the wall and u_tau = sqrt(nu |U_t| / y)
__global__ void k_les_wall(int nw, int nI, int nC, int nB, const int32_t* __restrict__ wallFace,
                           const int32_t* __restrict__ wallCell, const double* __restrict__ wn,
                           const double* __restrict__ wy, const double* __restrict__ U,
                           const double* __restrict__ Ub, double nu, double* __restrict__ uTau) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nw) return;
    const int b = wallFace[i] - nI, c = wallCell[i];
    const double n[3] = {wn[i], wn[nw + i], wn[2 * nw + i]};
    double du[3];
    for (int k = 0; k < 3; ++k) du[k] = U[size_t(k) * nC + c] - Ub[size_t(k) * nB + b];
    const double dn = du[0] * n[0] + du[1] * n[1] + du[2] * n[2];
    for (int k = 0; k < 3; ++k) du[k] -= dn * n[k];
    const double magUt = sqrt(du[0] * du[0] + du[1] * du[1] + du[2] * du[2]);
    uTau[i] = sqrt(nu * magUt / wy[i]);
}

// filter width (Van Driest damped), Smagorinsky nu_t, the nu_t limiter, and nu_eff = nu + nu_t
__global__ void k_les_nut(int nC, const double* __restrict__ G, const double* __restrict__ delta0, int vanDriest,
                          const double* __restrict__ yWall, const int32_t* __restrict__ nearest,
                          const double* __restrict__ uTau, double nu, double kOverC, double Aplus, double CsCs,
                          double nutMax, double* __restrict__ nut, double* __restrict__ nuEffC) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double delta = delta0[c];
    if (vanDriest) {
        const double y = yWall[c];
        const double ut = uTau[nearest[c]];
        const double yPlus = y * ut / nu;
        const double dv = kOverC * y * (1 - exp(-yPlus / Aplus));
        delta = dv < delta ? dv : delta;
    }
    // S = symm(G) = 0.5 (G + G^T); magSqr(S) = sum of the squares in component order
    double g[9];
    for (int m = 0; m < 9; ++m) g[m] = G[size_t(m) * nC + c];
    double ss = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            const double s = 0.5 * (g[3 * i + j] + g[3 * j + i]);
            ss += s * s;
        }
    double v = CsCs * delta * delta * sqrt(2 * ss);
    if (!(v <= nutMax)) v = isfinite(v) ? nutMax : 0.0;
    nut[c] = v;
    nuEffC[c] = nu + v;
}

// face nu_eff: linear interpolation inside, the wall value nu + nu_t,w (= nu, no wall model) on wall
// faces, the owner's value on other boundary faces
__global__ void k_les_nueff(int nF, int nI, const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                            const double* __restrict__ w, const double* __restrict__ nuEffC,
                            const int32_t* __restrict__ wallB, double nu, double* __restrict__ nuF) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    if (f < nI)
        nuF[f] = w[f] * nuEffC[own[f]] + (1.0 - w[f]) * nuEffC[nei[f]];
    else
        nuF[f] = wallB[f - nI] ? nu + 0.0 : nuEffC[own[f]];
}

// F_f = nu_eff,f (G_f . S_f - 2/3 tr(G_f) S_f) with G_f the interpolated cell gradient (the owner's on
// boundary faces)
__global__ void k_les_dev2(int nF, int nI, int nC, const int32_t* __restrict__ own, const int32_t* __restrict__ nei,
                           const double* __restrict__ w, const double* __restrict__ Sf, const double* __restrict__ G,
                           const double* __restrict__ nuF, double* __restrict__ F) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    double g[9];
    if (f < nI) {
        const int o = own[f], n = nei[f];
        const double wo = w[f], wn = 1.0 - wo;
        for (int m = 0; m < 9; ++m) g[m] = G[size_t(m) * nC + o] * wo + G[size_t(m) * nC + n] * wn;
    } else {
        const int o = own[f];
        for (int m = 0; m < 9; ++m) g[m] = G[size_t(m) * nC + o];
    }
    const double S[3] = {Sf[f], Sf[nF + f], Sf[2 * nF + f]};
    const double tr = g[0] + g[4] + g[8];
    const double t = (2.0 / 3.0) * tr;
    const double ne = nuF[f];
    for (int i = 0; i < 3; ++i) {
        const double gs = g[3 * i] * S[0] + g[3 * i + 1] * S[1] + g[3 * i + 2] * S[2];
        F[size_t(i) * nF + f] = ne * (gs - t * S[i]);
    }
}

// UEqn -= surfaceIntegrate(F) (source += (sum_f +-F_f * (1/V)) V, faces in ascending order), then
// UEqn -= f (source += f V) for the forcing f (constant force, or Ubar gradP/|Ubar| read from the state)
__global__ void k_les_source(int nC, int nI, const int32_t* __restrict__ cfOff, const int32_t* __restrict__ cf,
                             const double* __restrict__ F, int nF, const double* __restrict__ V, int forcing,
                             double f0, double f1, double f2, const double* __restrict__ state, double magUbar,
                             double* __restrict__ src) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    double s[3] = {src[c], src[nC + c], src[2 * nC + c]};
    const double Vc = V[c];
    if (F != nullptr) {
        double r[3] = {0.0, 0.0, 0.0};
        for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
            const uint32_t e = (uint32_t)cf[k];
            const int f = int(e & 0x7fffffffu);
            for (int j = 0; j < 3; ++j) {
                if (e >> 31)
                    r[j] -= F[size_t(j) * nF + f];
                else
                    r[j] += F[size_t(j) * nF + f];
            }
        }
        (void)nI;
        const double iv = 1.0 / Vc;
        for (int j = 0; j < 3; ++j) s[j] += (r[j] * iv) * Vc;
    }
    if (forcing != 0) {
        double fv[3] = {f0, f1, f2};
        if (forcing == 2) {
            const double q = state[0] / magUbar;
            for (int j = 0; j < 3; ++j) fv[j] = fv[j] * q;
        }
        for (int j = 0; j < 3; ++j) s[j] += fv[j] * Vc;
    }
    src[c] = s[0];
    src[nC + c] = s[1];
    src[2 * nC + c] = s[2];
}

// applyForcingCorrection, reductions and scalar update: sum (dir . U) V and sum rAU V (exact or plain),
// then in the last CTA: dU = |Ubar| - <U>, rAUave, and gradP += relaxation dU / resp with
// resp = 1 / (ddtCoeff + (1 - alphaU) / rAUave).  state = {gradP, dU, rAUave}.
template <bool EXACT>
__global__ void __launch_bounds__(kForceThreads) k_force_sums(int nC, const double* __restrict__ U,
                                                              const double* __restrict__ rAU,
                                                              const double* __restrict__ V, double d0, double d1,
                                                              double d2, double* __restrict__ part,
                                                              long long* __restrict__ bins,
                                                              unsigned long long* __restrict__ counter,
                                                              double totalVolume, double magUbar, double ddtC,
                                                              double alphaU, double relaxation,
                                                              double* __restrict__ state) {
    __shared__ long long sb[2][kForceWarps][kExactBins];
    __shared__ int sf[2][kForceWarps];
    __shared__ double red[2][kForceThreads];
    __shared__ int isLast;
    const int warp = threadIdx.x >> 5;
    if (EXACT) {
        for (int q = threadIdx.x; q < 2 * kForceWarps * kExactBins; q += blockDim.x) (&sb[0][0][0])[q] = 0;
        if (threadIdx.x < 2 * kForceWarps) (&sf[0][0])[threadIdx.x] = 0;
        __syncthreads();
    }
    double a0 = 0.0, a1 = 0.0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nC; c += gridDim.x * blockDim.x) {
        const double t0 = (d0 * U[c] + d1 * U[nC + c] + d2 * U[2 * size_t(nC) + c]) * V[c];
        const double t1 = rAU[c] * V[c];
        if (EXACT) {
            exact_add(sb[0][warp], &sf[0][warp], t0);
            exact_add(sb[1][warp], &sf[1][warp], t1);
        } else {
            a0 += t0;
            a1 += t1;
        }
    }
    if (EXACT) {
        __syncthreads();
        for (int k = threadIdx.x; k < 2 * kExactStride; k += blockDim.x) {
            const int which = k / kExactStride, q = k % kExactStride;
            long long s = 0;
            for (int w = 0; w < kForceWarps; ++w) s = q < kExactBins ? s + sb[which][w][q] : (s | sf[which][w]);
            bins[(size_t(blockIdx.x) * 2 + which) * kExactStride + q] = s;
        }
    } else {
        red[0][threadIdx.x] = a0;
        red[1][threadIdx.x] = a1;
        __syncthreads();
        for (int h = kForceThreads / 2; h > 0; h >>= 1) {
            if (threadIdx.x < h) {
                red[0][threadIdx.x] += red[0][threadIdx.x + h];
                red[1][threadIdx.x] += red[1][threadIdx.x + h];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            part[2 * blockIdx.x] = red[0][0];
            part[2 * blockIdx.x + 1] = red[1][0];
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) isLast = atomicAdd(counter, 1ull) == (unsigned long long)(gridDim.x - 1);
    __syncthreads();
    if (!isLast) return;
    __threadfence();
    __shared__ long long tot[2][kExactStride];
    __shared__ double sums[2];
    if (EXACT) {
        for (int k = threadIdx.x; k < 2 * kExactStride; k += blockDim.x) {
            const int which = k / kExactStride, q = k % kExactStride;
            long long s = 0;
            for (unsigned b = 0; b < gridDim.x; ++b) {
                const long long x = __ldcg(bins + (size_t(b) * 2 + which) * kExactStride + q);
                s = q < kExactBins ? s + x : (s | x);
            }
            tot[which][q] = s;
        }
        __syncthreads();
        if (threadIdx.x < 2) sums[threadIdx.x] = exact_value(tot[threadIdx.x], int(tot[threadIdx.x][kExactBins]));
    } else if (threadIdx.x < 2) {
        double s = 0.0;
        for (unsigned b = 0; b < gridDim.x; ++b) s += __ldcg(part + 2 * b + threadIdx.x);
        sums[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double magUbarAve = sums[0] / totalVolume;
        const double rAUave = sums[1] / totalVolume;
        const double dU = magUbar - magUbarAve;
        const double Aave = 1.0 / rAUave;
        const double resp = 1.0 / (ddtC + (1.0 - alphaU) * Aave);
        state[0] = state[0] + relaxation * dU / resp;
        state[1] = dU;
        state[2] = rAUave;
        *counter = 0;
    }
}

// U += dir (rAU dU / rAUave)
__global__ void k_force_correct(int nC, const double* __restrict__ rAU, double d0, double d1, double d2,
                                const double* __restrict__ state, double* __restrict__ U) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    const double s = rAU[c] * state[1] / state[2];
    U[c] += d0 * s;
    U[nC + c] += d1 * s;
    U[2 * size_t(nC) + c] += d2 * s;
}

template <class T>
std::vector<T> download(const T* d, size_t n) {
    std::vector<T> h(n);
    if (n) VLM_CUDA(cudaMemcpy(h.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
    return h;
}

}  // namespace

void DeviceFlow::setModel(const vlm_flow_model& m) {
    VLM_REQUIRE(!initialized_ || timeIndex_ == 0, VLM_ERR_BAD_ARG, "the flow model is set before the first step");
    VLM_REQUIRE(m.les == 0 || m.les == 1, VLM_ERR_BAD_ARG, "les: 0 laminar or 1 Smagorinsky");
    VLM_REQUIRE(m.forcing >= 0 && m.forcing <= 2, VLM_ERR_BAD_ARG, "forcing: 0 none, 1 constant, 2 mean velocity");
    les_ = m.les == 1;
    forcing_ = m.forcing;
    exactSums_ = ctrl_.p.reproducible != 0 || ctrl_.U.reproducible != 0;
    const double nu = ctrl_.nu;
    const int nP = G_.nPatches();
    if (forcing_ == 1)
        for (int k = 0; k < 3; ++k) force_[k] = m.force[k];
    if (forcing_ == 2) {
        for (int k = 0; k < 3; ++k) Ubar_[k] = m.Ubar[k];
        magUbar_ = std::sqrt(Ubar_[0] * Ubar_[0] + Ubar_[1] * Ubar_[1] + Ubar_[2] * Ubar_[2]);
        VLM_REQUIRE(magUbar_ > 0, VLM_ERR_BAD_ARG, "mean-velocity forcing needs a non-zero Ubar");
        for (int k = 0; k < 3; ++k) dir_[k] = Ubar_[k] / magUbar_;
        relax_ = m.relaxation;
        const double st[3] = {m.grad_p, 0.0, 1.0};
        forceState_.upload(st, 3, s_);
        forcePart_.resize(size_t(2) * kForceCtas);
        forceBins_.resize(size_t(2) * kForceCtas * kExactStride);
        forceCount_.resize(1);
        forceCount_.zero(s_);
        // Mesh::totalVolume (Mesh.cpp:645-647): cells in order
        const std::vector<double> V = download(G_.V(), size_t(nC_));
        double tv = 0;
        for (double v : V) tv += v;
        totalVolume_ = tv;
    }
    if (!les_) {
        VLM_CUDA(cudaStreamSynchronize(s_));
        return;
    }
    VLM_REQUIRE(m.Cs > 0 && m.delta_coeff > 0 && m.nut_max_ratio > 0, VLM_ERR_BAD_ARG, "LES coefficients must be positive");
    VLM_REQUIRE(!G_.twoD() || m.depth > 0, VLM_ERR_BAD_ARG, "a 2D LES needs the mesh depth");
    vanDriest_ = m.van_driest != 0;
    CsCs_ = m.Cs * m.Cs;
    kOverC_ = m.kappa / m.Cdelta;
    Aplus_ = m.Aplus;
    nutMax_ = m.nut_max_ratio * nu;
    const size_t N = size_t(nC_), F = size_t(nF_), B = size_t(std::max(nB_, 1));
    // geometry on the host for the set-up
    const std::vector<double> V = download(G_.V(), N), C = download(G_.C(), 3 * N), Cf = download(G_.Cf(), 3 * F),
                              Sf = download(G_.Sf(), 3 * F), magSf = download(G_.magSf(), F),
                              ndc = download(G_.ndc(), F);
    const std::vector<int32_t> own = download(G_.own(), F);
    // filter width (LESModel ctor, LESModels.cpp:20-33)
    std::vector<double> d0(N);
    for (size_t c = 0; c < N; ++c)
        d0[c] = m.delta_coeff * (G_.twoD() ? std::sqrt(V[c] / m.depth) : std::cbrt(V[c]));
    delta0_.upload(d0, s_);
    // wall faces in patch order (updateWallFaces, TurbulenceModel.cpp:199-216)
    std::vector<int32_t> wf, wc, wb(B, 0);
    std::vector<double> wnx, wny, wnz, wy;
    std::vector<WallDisc> discs;
    for (int q = 0; q < nP; ++q) {
        if (!m.wall_patch || m.wall_patch[q] != 1) continue;
        for (int i = 0; i < G_.patchSize()[q]; ++i) {
            const int f = G_.patchStart()[q] + i, c = own[f];
            const double A = magSf[f];
            const double n[3] = {Sf[f] / A, Sf[F + f] / A, Sf[2 * F + f] / A};
            const double dd[3] = {Cf[f] - C[c], Cf[F + f] - C[N + c], Cf[2 * F + f] - C[2 * N + c]};
            const double y = std::max(dd[0] * n[0] + dd[1] * n[1] + dd[2] * n[2], 1e-3 / ndc[f]);
            wf.push_back(f);
            wc.push_back(c);
            wnx.push_back(n[0]);
            wny.push_back(n[1]);
            wnz.push_back(n[2]);
            wy.push_back(y);
            wb[size_t(f - nI_)] = 1;
            // the disc of WallDistance.cpp (normal into the fluid)
            WallDisc w;
            for (int k = 0; k < 3; ++k) {
                w.c[k] = Cf[size_t(k) * F + f];
                w.n[k] = -1.0 * Sf[size_t(k) * F + f] / A;
            }
            constexpr double kPi = 3.14159265358979323846;
            w.r = G_.twoD() ? 0.5 * A / m.depth : std::sqrt(A / kPi);
            discs.push_back(w);
        }
    }
    nWall_ = int(wf.size());
    wallB_.upload(wb, s_);
    nut_.resize(N);
    nut_.zero(s_);
    nuEffC_.resize(N);
    nuF_.resize(F);
    devF_.resize(3 * F);
    if (nWall_ > 0) {
        wallFace_.upload(wf, s_);
        wallCell_.upload(wc, s_);
        std::vector<double> wn(wnx);
        wn.insert(wn.end(), wny.begin(), wny.end());
        wn.insert(wn.end(), wnz.begin(), wnz.end());
        wallN_.upload(wn, s_);
        wallY_.upload(wy, s_);
        uTau_.resize(size_t(nWall_));
    }
    if (vanDriest_ && nWall_ > 0) {
        // nearest wall face and distance of every cell (WallDistance.cpp compute), on the device
        yWall_.resize(N);
        nearest_.resize(N);
        wallNearestOnDevice(s_, nC_, G_.C(), discs, yWall_.get(), nearest_.get());
    } else {
        vanDriest_ = false;  // no walls: the damping is off (wd->hasWalls false)
    }
    VLM_CUDA(cudaStreamSynchronize(s_));
}

void DeviceFlow::modelState(double* nut, double* gradP) {
    if (nut) {
        if (les_)
            VLM_CUDA(cudaMemcpyAsync(nut, nut_.get(), sizeof(double) * nC_, cudaMemcpyDeviceToHost, s_));
        else
            std::fill(nut, nut + nC_, 0.0);
    }
    if (gradP) {
        *gradP = 0.0;
        if (forcing_ == 2) VLM_CUDA(cudaMemcpyAsync(gradP, forceState_.get(), sizeof(double), cudaMemcpyDeviceToHost, s_));
    }
    VLM_CUDA(cudaStreamSynchronize(s_));
}

void DeviceFlow::lesCorrect() {
    const double nu = ctrl_.nu;
    if (nWall_ > 0)
        k_les_wall<<<nblk(nWall_), 256, 0, s_>>>(nWall_, nI_, nC_, std::max(nB_, 1), wallFace_.get(), wallCell_.get(),
                                                 wallN_.get(), wallY_.get(), U_.get(), Ub_.get(), nu, uTau_.get()),
            ++launches_;
    k_les_nut<<<nblk(nC_), 256, 0, s_>>>(nC_, gU_.get(), delta0_.get(), vanDriest_ ? 1 : 0, yWall_.get(),
                                         nearest_.get(), uTau_.get(), nu, kOverC_, Aplus_, CsCs_, nutMax_, nut_.get(),
                                         nuEffC_.get()), ++launches_;
    k_les_nueff<<<nblk(nF_), 256, 0, s_>>>(nF_, nI_, G_.own(), G_.nei(), G_.w(), nuEffC_.get(), wallB_.get(), nu,
                                           nuF_.get()), ++launches_;
    VLM_CUDA(cudaGetLastError());
}

void DeviceFlow::explicitSources() {
    if (les_)
        k_les_dev2<<<nblk(nF_), 256, 0, s_>>>(nF_, nI_, nC_, G_.own(), G_.nei(), G_.w(), G_.Sf(), gU_.get(), nuF_.get(),
                                              devF_.get()), ++launches_;
    const double* fv = forcing_ == 1 ? force_ : Ubar_;
    k_les_source<<<nblk(nC_), 256, 0, s_>>>(nC_, nI_, G_.cellFaceOff(), G_.cellFaces(), les_ ? devF_.get() : nullptr,
                                            nF_, G_.V(), forcing_, fv[0], fv[1], fv[2],
                                            forcing_ == 2 ? forceState_.get() : nullptr, magUbar_, src_.get()),
        ++launches_;
    VLM_CUDA(cudaGetLastError());
}

void DeviceFlow::forcingCorrection(double aU) {
    // fvm::ddtCoeffs(ddtS, time, nOldTimes >= 2).c (Schemes.h:71-86)
    double ddtC = 0.0;
    if (!ctrl_.steady) {
        const double rDt = 1.0 / dt_;
        if (ctrl_.ddt_scheme == 2 && nOld_ >= 2 && dt0_ > 0)
            ddtC = (1.0 + dt_ / (dt_ + dt0_)) * rDt;
        else if (ctrl_.ddt_scheme != 0)
            ddtC = rDt;
    }
    const int grid = std::max(1, std::min(kForceCtas, nblk(nC_, kForceThreads)));
    if (exactSums_)
        k_force_sums<true><<<grid, kForceThreads, 0, s_>>>(nC_, U_.get(), rAU_.get(), G_.V(), dir_[0], dir_[1], dir_[2],
                                                          forcePart_.get(), forceBins_.get(), forceCount_.get(),
                                                          totalVolume_, magUbar_, ddtC, aU, relax_,
                                                          forceState_.get()), ++launches_;
    else
        k_force_sums<false><<<grid, kForceThreads, 0, s_>>>(nC_, U_.get(), rAU_.get(), G_.V(), dir_[0], dir_[1],
                                                           dir_[2], forcePart_.get(), forceBins_.get(),
                                                           forceCount_.get(), totalVolume_, magUbar_, ddtC, aU, relax_,
                                                           forceState_.get()), ++launches_;
    k_force_correct<<<nblk(nC_), 256, 0, s_>>>(nC_, rAU_.get(), dir_[0], dir_[1], dir_[2], forceState_.get(),
                                               U_.get()), ++launches_;
    boundaryU();
    VLM_CUDA(cudaGetLastError());
}

}  // namespace vlm
