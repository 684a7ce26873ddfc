// Device-side mesh setup for boxes: generateBox (src/fvm/mesh/RawMesh.cpp:391-502) and the serial
// Mesh::build geometry (src/fvm/mesh/Mesh.cpp:21-48 faceGeometry, :135-153 cell geometry, :239-320
// compute faces with merged cyclic pairs, :600-648 finishLocal) as kernels: one thread per raw face,
// per cell and per compute face.  Every sum runs in the reference's order and the build has no
// contraction (-fmad=false), so the arrays equal the reference's bit for bit.
//
// Raw mesh numbering (as generateBox emits it): points P(i,j,k) = i + (nx+1)(j + (ny+1)k); cells
// C(i,j,k) = i + nx(j + ny k); internal faces cell by cell, +x, +y, +z where the neighbour exists;
// then the six side patches xMin xMax yMin yMax zMin zMax.  Compute mesh: the raw internal faces,
// then the cyclic pairs merged into internal faces (owner on the min side), then the wall patches
// in side order; the empty sides of a 2D box are dropped.
#include "meshgen.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

namespace vlm {

namespace {

constexpr double kVSmall = 1.0e-300;

inline int nblk(int64_t n, int t = 256) { return int((n + t - 1) / t); }

struct Box {
    int nx, ny, nz;
    int nIraw;         // raw internal faces
    int start[7];      // raw face index of each side patch's first face; start[6] = raw face count
};

__device__ __forceinline__ int pointId(const Box& b, int i, int j, int k) { return i + (b.nx + 1) * (j + (b.ny + 1) * k); }
__device__ __forceinline__ int cellId(const Box& b, int i, int j, int k) { return i + b.nx * (j + b.ny * k); }

// number of raw internal faces emitted before cell (i, j, k): x faces of the cells before it with
// i < nx-1, y faces of those with j < ny-1, z faces of those with k < nz-1
__device__ __forceinline__ int facesBefore(const Box& b, int i, int j, int k) {
    const int nx = b.nx, ny = b.ny, nz = b.nz;
    const int fx = (j + ny * k) * (nx - 1) + (i < nx - 1 ? i : nx - 1);
    const int fy = k * nx * (ny - 1) + (j < ny - 1 ? j * nx + i : (ny - 1) * nx);
    const int c = cellId(b, i, j, k);
    const int fz = k < nz - 1 ? c : (nz - 1) * nx * ny;
    return fx + fy + fz;
}

// raw internal face of cell (i, j, k) towards +dir (the neighbour exists)
__device__ __forceinline__ int internalFace(const Box& b, int i, int j, int k, int dir) {
    return facesBefore(b, i, j, k) + (dir > 0 && i < b.nx - 1) + (dir > 1 && j < b.ny - 1);
}

__device__ __forceinline__ void ld(const double* p, int id, double v[3]) {
    v[0] = p[3 * size_t(id)];
    v[1] = p[3 * size_t(id) + 1];
    v[2] = p[3 * size_t(id) + 2];
}

// faceGeometry (Mesh.cpp:21-48) of a quad: triangles about the vertex average
__device__ void quadGeometry(const double* pts, const int fp[4], double Sf[3], double Cf[3]) {
    double q[4][3];
    for (int k = 0; k < 4; ++k) ld(pts, fp[k], q[k]);
    double pavg[3];
    for (int c = 0; c < 3; ++c) pavg[c] = (((q[0][c] + q[1][c]) + q[2][c]) + q[3][c]) / 4.0;
    double sumN[3] = {0.0, 0.0, 0.0}, sumA = 0.0, sumAc[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 4; ++k) {
        const double* p0 = q[k];
        const double* p1 = q[(k + 1) % 4];
        double e[3], r[3], cc[3];
        for (int c = 0; c < 3; ++c) {
            cc[c] = (p0[c] + p1[c]) + pavg[c];
            e[c] = p1[c] - p0[c];
            r[c] = pavg[c] - p0[c];
        }
        const double nk[3] = {e[1] * r[2] - e[2] * r[1], e[2] * r[0] - e[0] * r[2], e[0] * r[1] - e[1] * r[0]};
        const double a = sqrt(nk[0] * nk[0] + nk[1] * nk[1] + nk[2] * nk[2]);
        for (int c = 0; c < 3; ++c) {
            sumN[c] = sumN[c] + nk[c];
            sumAc[c] = sumAc[c] + a * cc[c];
        }
        sumA = sumA + a;
    }
    for (int c = 0; c < 3; ++c) {
        Cf[c] = sumA < kVSmall ? pavg[c] : sumAc[c] / (3.0 * sumA);
        Sf[c] = 0.5 * sumN[c];
    }
}

// raw faces: geometry, owner (and neighbour of the internal ones); one thread per raw face
__global__ void k_box_raw_faces(Box b, const double* __restrict__ pts, int32_t* __restrict__ rOwn,
                                int32_t* __restrict__ rNei, double* __restrict__ rSf, double* __restrict__ rCf) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.start[6]) return;
    int fp[4], own, nei = -1;
    if (f < b.nIraw) {
        // the cell that emits f: the last cell whose first face index is <= f (binary search)
        int lo = 0, hi = b.nx * b.ny * b.nz - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            const int mi = mid % b.nx, mj = (mid / b.nx) % b.ny, mk = mid / (b.nx * b.ny);
            if (facesBefore(b, mi, mj, mk) <= f) lo = mid;
            else hi = mid - 1;
        }
        const int i = lo % b.nx, j = (lo / b.nx) % b.ny, k = lo / (b.nx * b.ny);
        int r = f - facesBefore(b, i, j, k);
        int dir = -1;
        const bool has[3] = {i + 1 < b.nx, j + 1 < b.ny, k + 1 < b.nz};
        for (int q = 0; q < 3 && dir < 0; ++q)
            if (has[q]) {
                if (r == 0) dir = q;
                --r;
            }
        own = cellId(b, i, j, k);
        if (dir == 0) {
            const int v[4] = {pointId(b, i + 1, j, k), pointId(b, i + 1, j + 1, k), pointId(b, i + 1, j + 1, k + 1),
                              pointId(b, i + 1, j, k + 1)};
            for (int q = 0; q < 4; ++q) fp[q] = v[q];
            nei = cellId(b, i + 1, j, k);
        } else if (dir == 1) {
            const int v[4] = {pointId(b, i, j + 1, k), pointId(b, i, j + 1, k + 1), pointId(b, i + 1, j + 1, k + 1),
                              pointId(b, i + 1, j + 1, k)};
            for (int q = 0; q < 4; ++q) fp[q] = v[q];
            nei = cellId(b, i, j + 1, k);
        } else {
            const int v[4] = {pointId(b, i, j, k + 1), pointId(b, i + 1, j, k + 1), pointId(b, i + 1, j + 1, k + 1),
                              pointId(b, i, j + 1, k + 1)};
            for (int q = 0; q < 4; ++q) fp[q] = v[q];
            nei = cellId(b, i, j, k + 1);
        }
    } else {
        int s = 0;
        while (f >= b.start[s + 1]) ++s;
        const int q = f - b.start[s];
        if (s < 2) {  // x sides: j fastest, then k
            const int j = q % b.ny, k = q / b.ny, i = s == 0 ? 0 : b.nx;
            if (s == 0) {
                const int v[4] = {pointId(b, i, j, k), pointId(b, i, j, k + 1), pointId(b, i, j + 1, k + 1), pointId(b, i, j + 1, k)};
                for (int t = 0; t < 4; ++t) fp[t] = v[t];
            } else {
                const int v[4] = {pointId(b, i, j, k), pointId(b, i, j + 1, k), pointId(b, i, j + 1, k + 1), pointId(b, i, j, k + 1)};
                for (int t = 0; t < 4; ++t) fp[t] = v[t];
            }
            own = cellId(b, s == 0 ? 0 : b.nx - 1, j, k);
        } else if (s < 4) {  // y sides: i fastest, then k
            const int i = q % b.nx, k = q / b.nx, j = s == 2 ? 0 : b.ny;
            if (s == 2) {
                const int v[4] = {pointId(b, i, j, k), pointId(b, i + 1, j, k), pointId(b, i + 1, j, k + 1), pointId(b, i, j, k + 1)};
                for (int t = 0; t < 4; ++t) fp[t] = v[t];
            } else {
                const int v[4] = {pointId(b, i, j, k), pointId(b, i, j, k + 1), pointId(b, i + 1, j, k + 1), pointId(b, i + 1, j, k)};
                for (int t = 0; t < 4; ++t) fp[t] = v[t];
            }
            own = cellId(b, i, s == 2 ? 0 : b.ny - 1, k);
        } else {  // z sides: i fastest, then j
            const int i = q % b.nx, j = q / b.nx, k = s == 4 ? 0 : b.nz;
            if (s == 4) {
                const int v[4] = {pointId(b, i, j, k), pointId(b, i, j + 1, k), pointId(b, i + 1, j + 1, k), pointId(b, i + 1, j, k)};
                for (int t = 0; t < 4; ++t) fp[t] = v[t];
            } else {
                const int v[4] = {pointId(b, i, j, k), pointId(b, i + 1, j, k), pointId(b, i + 1, j + 1, k), pointId(b, i, j + 1, k)};
                for (int t = 0; t < 4; ++t) fp[t] = v[t];
            }
            own = cellId(b, i, j, s == 4 ? 0 : b.nz - 1);
        }
    }
    double Sf[3], Cf[3];
    quadGeometry(pts, fp, Sf, Cf);
    rOwn[f] = own;
    if (f < b.nIraw) rNei[f] = nei;
    for (int c = 0; c < 3; ++c) {
        rSf[3 * size_t(f) + c] = Sf[c];
        rCf[3 * size_t(f) + c] = Cf[c];
    }
}

// cell centres and volumes (Mesh.cpp:135-153): pyramids about the face-centre average, the cell's
// faces in ascending raw face order; one thread per cell
__global__ void k_box_cells(Box b, const int32_t* __restrict__ rOwn, const double* __restrict__ rSf,
                            const double* __restrict__ rCf, double* __restrict__ C, double* __restrict__ V) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= b.nx * b.ny * b.nz) return;
    const int i = c % b.nx, j = (c / b.nx) % b.ny, k = c / (b.nx * b.ny);
    int f[6];
    f[0] = i > 0 ? internalFace(b, i - 1, j, k, 0) : b.start[0] + (j + b.ny * k);
    f[1] = i < b.nx - 1 ? internalFace(b, i, j, k, 0) : b.start[1] + (j + b.ny * k);
    f[2] = j > 0 ? internalFace(b, i, j - 1, k, 1) : b.start[2] + (i + b.nx * k);
    f[3] = j < b.ny - 1 ? internalFace(b, i, j, k, 1) : b.start[3] + (i + b.nx * k);
    f[4] = k > 0 ? internalFace(b, i, j, k - 1, 2) : b.start[4] + (i + b.nx * j);
    f[5] = k < b.nz - 1 ? internalFace(b, i, j, k, 2) : b.start[5] + (i + b.nx * j);
    for (int a = 1; a < 6; ++a)  // ascending raw face order
        for (int q = a; q > 0 && f[q - 1] > f[q]; --q) {
            const int t = f[q];
            f[q] = f[q - 1];
            f[q - 1] = t;
        }
    double cEst[3] = {0.0, 0.0, 0.0};
    for (int q = 0; q < 6; ++q)
        for (int d = 0; d < 3; ++d) cEst[d] = cEst[d] + rCf[3 * size_t(f[q]) + d];
    for (int d = 0; d < 3; ++d) cEst[d] = cEst[d] / 6.0;
    double cSum[3] = {0.0, 0.0, 0.0}, vSum = 0.0;
    for (int q = 0; q < 6; ++q) {
        const int g = f[q];
        const bool own = rOwn[g] == c;
        double S[3], Cf[3];
        ld(rSf, g, S);
        ld(rCf, g, Cf);
        if (!own)
            for (int d = 0; d < 3; ++d) S[d] = -S[d];
        const double pv = fmax(S[0] * (Cf[0] - cEst[0]) + S[1] * (Cf[1] - cEst[1]) + S[2] * (Cf[2] - cEst[2]), kVSmall);
        for (int d = 0; d < 3; ++d) cSum[d] = cSum[d] + pv * (0.75 * Cf[d] + 0.25 * cEst[d]);
        vSum = vSum + pv;
    }
    for (int d = 0; d < 3; ++d) C[3 * size_t(c) + d] = cSum[d] / vSum;
    V[c] = vSum / 3.0;
}

// compute faces (Mesh.cpp:239-320) and finishLocal (Mesh.cpp:600-626); one thread per compute face.
// seg: [0] raw internal count, then per block (cyclic pair or wall patch) its first compute face,
// first raw face of side a, of side b (cyclic only; -1 for a wall patch)
struct FaceBlocks {
    int n;             // blocks after the raw internal faces
    int first[8];      // first compute face of each block; first[n] = compute face count
    int sideA[7], sideB[7];
};

__global__ void k_box_faces(Box b, FaceBlocks fb, const int32_t* __restrict__ rOwn, const int32_t* __restrict__ rNei,
                            const double* __restrict__ rSf, const double* __restrict__ rCf, const double* __restrict__ C,
                            int nI, int32_t* __restrict__ own, int32_t* __restrict__ nei, double* __restrict__ Sf,
                            double* __restrict__ Cf, double* __restrict__ d, double* __restrict__ magSf,
                            double* __restrict__ w, double* __restrict__ ndc, double* __restrict__ corr,
                            double* __restrict__ skew) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= fb.first[fb.n]) return;
    int o, n = -1, rf;
    double dd[3], CP[3], S[3], F[3];
    if (g < b.nIraw) {
        rf = g;
        o = rOwn[rf];
        n = rNei[rf];
        ld(rSf, rf, S);
        ld(rCf, rf, F);
        double CN[3];
        ld(C, o, CP);
        ld(C, n, CN);
        for (int q = 0; q < 3; ++q) dd[q] = CN[q] - CP[q];
    } else {
        int blk = 0;
        while (g >= fb.first[blk + 1]) ++blk;
        const int loc = g - fb.first[blk];
        rf = b.start[fb.sideA[blk]] + loc;
        o = rOwn[rf];
        ld(rSf, rf, S);
        ld(rCf, rf, F);
        ld(C, o, CP);
        if (fb.sideB[blk] >= 0) {  // cyclic pair: neighbour across the period, d with the shift
            const int rb = b.start[fb.sideB[blk]] + loc;
            n = rOwn[rb];
            double CN[3], Fb[3];
            ld(C, n, CN);
            ld(rCf, rb, Fb);
            for (int q = 0; q < 3; ++q) dd[q] = (CN[q] + (F[q] - Fb[q])) - CP[q];
        } else {
            for (int q = 0; q < 3; ++q) dd[q] = F[q] - CP[q];
        }
    }
    own[g] = o;
    if (g < nI) nei[g] = n;
    for (int q = 0; q < 3; ++q) {
        Sf[3 * size_t(g) + q] = S[q];
        Cf[3 * size_t(g) + q] = F[q];
        d[3 * size_t(g) + q] = dd[q];
    }
    const double mS = sqrt(S[0] * S[0] + S[1] * S[1] + S[2] * S[2]);
    magSf[g] = mS;
    const double nr[3] = {S[0] / mS, S[1] / mS, S[2] / mS};
    double wf = 1.0, sk[3] = {0.0, 0.0, 0.0};
    if (g < nI) {
        const double sOwn = fabs(S[0] * (F[0] - CP[0]) + S[1] * (F[1] - CP[1]) + S[2] * (F[2] - CP[2]));
        double e[3];
        for (int q = 0; q < 3; ++q) e[q] = (CP[q] + dd[q]) - F[q];
        const double sNei = fabs(S[0] * e[0] + S[1] * e[1] + S[2] * e[2]);
        wf = sNei / (sOwn + sNei);
        for (int q = 0; q < 3; ++q) sk[q] = F[q] - (CP[q] + dd[q] * (1.0 - wf));
    }
    w[g] = wf;
    const double magd = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
    const double nd = fmax(nr[0] * dd[0] + nr[1] * dd[1] + nr[2] * dd[2], 0.05 * magd);
    const double ic = 1.0 / nd;
    ndc[g] = ic;
    for (int q = 0; q < 3; ++q) {
        corr[3 * size_t(g) + q] = nr[q] - dd[q] * ic;
        skew[3 * size_t(g) + q] = sk[q];
    }
}

}  // namespace

BoxMesh buildBoxMesh(const vlm_box_spec& spec, cudaStream_t s) {
    const int nx = spec.n[0], ny = spec.n[1], nz = spec.n[2];
    VLM_REQUIRE(nx >= 1 && ny >= 1 && nz >= 1, VLM_ERR_BAD_ARG, "bad box resolution");
    VLM_REQUIRE(!spec.two_d || nz == 1, VLM_ERR_BAD_ARG, "a 2D box needs n[2] == 1");
    for (int d = 0; d < 3; ++d)
        VLM_REQUIRE(!spec.periodic[d] || spec.n[d] >= 2 || (d == 2 && spec.two_d), VLM_ERR_BAD_ARG,
                    "a periodic direction needs at least 2 cells");
    const int64_t nC64 = int64_t(nx) * ny * nz;
    const int64_t nP64 = int64_t(nx + 1) * (ny + 1) * (nz + 1);
    const int64_t nIraw64 = int64_t(nx - 1) * ny * nz + int64_t(nx) * (ny - 1) * nz + int64_t(nx) * ny * (nz - 1);
    const int64_t sides64 = 2 * (int64_t(ny) * nz + int64_t(nx) * nz + int64_t(nx) * ny);
    VLM_REQUIRE(nIraw64 + sides64 < (int64_t(1) << 31) - 1 && nP64 < (int64_t(1) << 31) - 1, VLM_ERR_BAD_ARG,
                "box exceeds 2^31 faces or points");
    Box b;
    b.nx = nx;
    b.ny = ny;
    b.nz = nz;
    b.nIraw = int(nIraw64);
    const int sideSize[6] = {ny * nz, ny * nz, nx * nz, nx * nz, nx * ny, nx * ny};
    b.start[0] = b.nIraw;
    for (int q = 0; q < 6; ++q) b.start[q + 1] = b.start[q] + sideSize[q];
    const int nFraw = b.start[6];
    const int nC = int(nC64);

    BoxMesh M;
    M.nCells = nC;
    // points: the caller's, or the graded box (tanhStretch, RawMesh.cpp:387-389, on the host where the
    // reference evaluates it)
    std::vector<double> pts(size_t(3) * size_t(nP64));
    if (spec.points) {
        std::copy(spec.points, spec.points + 3 * nP64, pts.begin());
    } else {
        std::vector<double> ax[3];
        for (int d = 0; d < 3; ++d) {
            const int nd = spec.n[d];
            ax[d].resize(size_t(nd) + 1);
            const double beta = spec.beta[d];
            const double tb = beta > 0 ? std::tanh(beta) : 1.0;
            for (int i = 0; i <= nd; ++i) {
                double t = double(i) / double(nd);
                if (beta > 0) t = 0.5 * (1.0 + std::tanh(beta * (2.0 * t - 1.0)) / tb);
                ax[d][i] = spec.lo[d] + (spec.hi[d] - spec.lo[d]) * t;
            }
        }
        size_t p = 0;
        for (int k = 0; k <= nz; ++k)
            for (int j = 0; j <= ny; ++j)
                for (int i = 0; i <= nx; ++i) {
                    pts[p++] = ax[0][i];
                    pts[p++] = ax[1][j];
                    pts[p++] = ax[2][k];
                }
    }
    DBuf<double> dPts, rSf, rCf, dC, dV;
    DBuf<int32_t> rOwn, rNei;
    dPts.upload(pts, s);
    rOwn.resize(size_t(nFraw));
    rNei.resize(size_t(std::max(b.nIraw, 1)));
    rSf.resize(size_t(3) * nFraw);
    rCf.resize(size_t(3) * nFraw);
    dC.resize(size_t(3) * nC);
    dV.resize(size_t(nC));
    k_box_raw_faces<<<nblk(nFraw), 256, 0, s>>>(b, dPts.get(), rOwn.get(), rNei.get(), rSf.get(), rCf.get());
    k_box_cells<<<nblk(nC), 256, 0, s>>>(b, rOwn.get(), rSf.get(), rCf.get(), dC.get(), dV.get());
    VLM_CUDA(cudaGetLastError());

    // compute-face blocks: cyclic pairs (x, y, z), then the wall patches in side order
    const bool cyc[3] = {spec.periodic[0] != 0, spec.periodic[1] != 0, spec.periodic[2] != 0 && !spec.two_d};
    FaceBlocks fb{};
    int nextFace = b.nIraw;
    for (int d = 0; d < 3; ++d)
        if (cyc[d]) {
            fb.first[fb.n] = nextFace;
            fb.sideA[fb.n] = 2 * d;
            fb.sideB[fb.n] = 2 * d + 1;
            nextFace += sideSize[2 * d];
            ++fb.n;
        }
    const int nI = nextFace;
    for (int q = 0; q < 6; ++q) {
        const int d = q / 2;
        if (cyc[d] || (d == 2 && spec.two_d)) continue;
        fb.first[fb.n] = nextFace;
        fb.sideA[fb.n] = q;
        fb.sideB[fb.n] = -1;
        M.patchSide.push_back(q);
        M.patchStart.push_back(nextFace);
        M.patchSize.push_back(sideSize[q]);
        nextFace += sideSize[q];
        ++fb.n;
    }
    fb.first[fb.n] = nextFace;
    const int nF = nextFace;
    M.nInternal = nI;
    M.nFaces = nF;
    DBuf<int32_t> own, nei;
    DBuf<double> Sf, Cf, d, magSf, w, ndc, corr, skew;
    own.resize(size_t(nF));
    nei.resize(size_t(std::max(nI, 1)));
    for (DBuf<double>* v : {&Sf, &Cf, &d, &corr, &skew}) v->resize(size_t(3) * nF);
    for (DBuf<double>* v : {&magSf, &w, &ndc}) v->resize(size_t(nF));
    k_box_faces<<<nblk(nF), 256, 0, s>>>(b, fb, rOwn.get(), rNei.get(), rSf.get(), rCf.get(), dC.get(), nI, own.get(),
                                         nei.get(), Sf.get(), Cf.get(), d.get(), magSf.get(), w.get(), ndc.get(),
                                         corr.get(), skew.get());
    VLM_CUDA(cudaGetLastError());

    auto back = [&](auto& dst, auto& src, size_t n) {
        dst.resize(n);
        if (n) VLM_CUDA(cudaMemcpyAsync(dst.data(), src.get(), sizeof(dst[0]) * n, cudaMemcpyDeviceToHost, s));
    };
    back(M.owner, own, size_t(nF));
    back(M.neighbour, nei, size_t(nI));
    back(M.V, dV, size_t(nC));
    back(M.C, dC, size_t(3) * nC);
    back(M.Sf, Sf, size_t(3) * nF);
    back(M.Cf, Cf, size_t(3) * nF);
    back(M.d, d, size_t(3) * nF);
    back(M.magSf, magSf, size_t(nF));
    back(M.w, w, size_t(nF));
    back(M.ndc, ndc, size_t(nF));
    back(M.corrVecs, corr, size_t(3) * nF);
    back(M.skewVecs, skew, size_t(3) * nF);
    // a 2D box's empty direction: the largest summed |S| over the dropped faces (Mesh.cpp, strict >)
    std::vector<double> eSf;
    if (spec.two_d) {
        eSf.resize(size_t(3) * 2 * sideSize[4]);
        VLM_CUDA(cudaMemcpyAsync(eSf.data(), rSf.get() + size_t(3) * b.start[4], sizeof(double) * eSf.size(),
                                 cudaMemcpyDeviceToHost, s));
    }
    VLM_CUDA(cudaStreamSynchronize(s));
    M.twoD = spec.two_d ? 1 : 0;
    M.emptyDir = -1;
    if (spec.two_d) {
        double en[3] = {0.0, 0.0, 0.0};
        for (size_t f = 0; f < eSf.size() / 3; ++f)
            for (int q = 0; q < 3; ++q) en[q] += std::fabs(eSf[3 * f + q]);
        M.emptyDir = 0;
        for (int a = 1; a < 3; ++a)
            if (en[a] > en[M.emptyDir]) M.emptyDir = a;
    }
    return M;
}

}  // namespace vlm
