// Nearest wall face of every cell on the device (walldist.h).
//
// Search structure: the wall-face centres sorted along a Morton (Z-order) curve of their bounding
// box, and above them a 32-ary hierarchy of axis-aligned bounding boxes: a node of level 1 bounds
// 32 consecutive centres, a node of level l+1 bounds 32 consecutive nodes of level l, up to one
// root.  One thread per cell walks the hierarchy depth first with an explicit stack, pushing the
// children of a node nearest last (so they are searched first), and skips every node whose box is
// farther than the 8th-best centre found so far.  The 8 best are kept in the order (squared
// distance, wall-face index).  A box's squared distance is computed per axis with the same
// subtraction as a centre's, so in floating point it never exceeds the distance of a centre it
// bounds and the pruning is exact.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "common.h"
#include "walldist.h"

namespace vlm {

namespace {

constexpr int kFan = 32;        // children per node
constexpr int kMaxLevels = 6;   // up to 32^6 wall faces
constexpr int kK = 8;           // nearest centres kept (WallDistance.cpp K)
constexpr double kGreatDist = 1.0e15;  // core/Types.h GREAT, the initial best distance

struct DiscsDev {
    const double *cx, *cy, *cz, *nx, *ny, *nz, *r;
    const int32_t* id;  // wall-face index of the sorted centre
    int n;
};

struct TreeDev {
    const double* box;           // 6 doubles per node (lo xyz, hi xyz), level 1 first
    int off[kMaxLevels + 1];     // first node of level l (l >= 1)
    int count[kMaxLevels + 1];   // nodes of level l; count[0] = centres
    int top;                     // root level
};

__device__ __forceinline__ double axis_gap(double x, double lo, double hi) {
    return x < lo ? lo - x : (x > hi ? x - hi : 0.0);
}

__device__ __forceinline__ double box_d2(const TreeDev& T, int lev, int idx, double x, double y, double z) {
    const double* b = T.box + 6 * size_t(T.off[lev] + idx);
    const double gx = axis_gap(x, b[0], b[3]), gy = axis_gap(y, b[1], b[4]), gz = axis_gap(z, b[2], b[5]);
    return gx * gx + gy * gy + gz * gz;
}

// faceDistance of WallDistance.cpp: distance to the disc (centre c, normal n, radius r)
__device__ __forceinline__ double disc_distance(const DiscsDev& D, int k, double x, double y, double z) {
    const double d0 = x - D.cx[k], d1 = y - D.cy[k], d2 = z - D.cz[k];
    const double n0 = D.nx[k], n1 = D.ny[k], n2 = D.nz[k];
    const double dn = d0 * n0 + d1 * n1 + d2 * n2;
    const double t0 = d0 - dn * n0, t1 = d1 - dn * n1, t2 = d2 - dn * n2;
    const double lat = sqrt(t0 * t0 + t1 * t1 + t2 * t2);
    const double out = fmax(lat - D.r[k], 0.0);
    return sqrt(dn * dn + out * out);
}

__global__ void k_wall_nearest(int nC, const double* __restrict__ C, DiscsDev D, TreeDev T, double* __restrict__ yOut,
                               int32_t* __restrict__ nearestOut) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    const double x = C[c], y = C[nC + c], z = C[2 * size_t(nC) + c];
    double bd[kK];
    int bs[kK], bi[kK];  // sorted position and wall-face index of the best centres
    int nb = 0;
    // (d, i) enters when fewer than K are kept or it precedes the K-th in (distance, index) order
    auto insert = [&](double d, int s, int i) {
        if (nb == kK && !(d < bd[kK - 1] || (d == bd[kK - 1] && i < bi[kK - 1]))) return;
        int k = nb < kK ? nb++ : kK - 1;
        while (k > 0 && (bd[k - 1] > d || (bd[k - 1] == d && bi[k - 1] > i))) {
            bd[k] = bd[k - 1];
            bs[k] = bs[k - 1];
            bi[k] = bi[k - 1];
            --k;
        }
        bd[k] = d;
        bs[k] = s;
        bi[k] = i;
    };
    int stack[kFan * kMaxLevels];
    int sp = 0;
    stack[sp++] = T.top << 27;
    while (sp > 0) {
        const int e = stack[--sp];
        const int lev = e >> 27, idx = e & ((1 << 27) - 1);
        if (nb == kK && box_d2(T, lev, idx, x, y, z) > bd[kK - 1]) continue;
        const int b0 = idx * kFan, b1 = min(b0 + kFan, T.count[lev - 1]);
        if (lev == 1) {
            for (int k = b0; k < b1; ++k) {
                const double dx = x - D.cx[k], dy = y - D.cy[k], dz = z - D.cz[k];
                insert(dx * dx + dy * dy + dz * dz, k, D.id[k]);
            }
            continue;
        }
        // children that may still hold a better centre, ordered by box distance (farthest first)
        double cd[kFan];
        int ci[kFan];
        int m = 0;
        for (int k = b0; k < b1; ++k) {
            const double d = box_d2(T, lev - 1, k, x, y, z);
            if (nb == kK && d > bd[kK - 1]) continue;
            int q = m++;
            while (q > 0 && cd[q - 1] < d) {
                cd[q] = cd[q - 1];
                ci[q] = ci[q - 1];
                --q;
            }
            cd[q] = d;
            ci[q] = k;
        }
        for (int q = 0; q < m; ++q) stack[sp++] = ((lev - 1) << 27) | ci[q];
    }
    double best = kGreatDist;
    int win = 0;
    for (int k = 0; k < nb; ++k) {
        const double d = disc_distance(D, bs[k], x, y, z);
        if (d < best || (d == best && bi[k] < win)) {
            best = d;
            win = bi[k];
        }
    }
    yOut[c] = best;
    nearestOut[c] = win;
}

// 10 bits of v spread to every third bit
uint32_t spread3(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

}  // namespace

void wallNearestOnDevice(cudaStream_t s, int nC, const double* cellC, const std::vector<WallDisc>& discs, double* y,
                         int32_t* nearest) {
    const int nW = int(discs.size());
    if (nW == 0 || nC == 0) return;
    // Morton order of the centres inside their bounding box
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (const WallDisc& w : discs)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], w.c[a]);
            hi[a] = std::max(hi[a], w.c[a]);
        }
    std::vector<uint32_t> code(size_t(nW), 0);
    for (int k = 0; k < nW; ++k) {
        uint32_t q[3];
        for (int a = 0; a < 3; ++a) {
            const double span = hi[a] - lo[a];
            const double t = span > 0 ? (discs[k].c[a] - lo[a]) / span : 0.0;
            q[a] = uint32_t(std::min(1023.0, std::max(0.0, std::floor(t * 1024.0))));
        }
        code[k] = spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2;
    }
    std::vector<int32_t> order(static_cast<size_t>(nW));
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return code[a] != code[b] ? code[a] < code[b] : a < b; });
    // sorted centres (structure of arrays) and the box levels above them
    std::vector<double> soa(size_t(7) * nW);
    for (int k = 0; k < nW; ++k) {
        const WallDisc& w = discs[order[k]];
        for (int a = 0; a < 3; ++a) {
            soa[size_t(a) * nW + k] = w.c[a];
            soa[size_t(3 + a) * nW + k] = w.n[a];
        }
        soa[size_t(6) * nW + k] = w.r;
    }
    TreeDev T = {};
    std::vector<double> box;
    T.count[0] = nW;
    int lev = 0;
    do {
        if (lev + 1 > kMaxLevels) throw Error(VLM_ERR_UNSUPPORTED, "too many wall faces for the wall-distance search");
        const int nChild = T.count[lev], nNode = (nChild + kFan - 1) / kFan;
        T.off[lev + 1] = int(box.size() / 6);
        T.count[lev + 1] = nNode;
        const size_t childOff = lev == 0 ? 0 : size_t(T.off[lev]);
        for (int t = 0; t < nNode; ++t) {
            double b[6] = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
            for (int k = t * kFan; k < std::min(nChild, (t + 1) * kFan); ++k)
                for (int a = 0; a < 3; ++a) {
                    const double vlo = lev == 0 ? soa[size_t(a) * nW + k] : box[6 * (childOff + k) + a];
                    const double vhi = lev == 0 ? soa[size_t(a) * nW + k] : box[6 * (childOff + k) + 3 + a];
                    b[a] = std::min(b[a], vlo);
                    b[3 + a] = std::max(b[3 + a], vhi);
                }
            box.insert(box.end(), b, b + 6);
        }
        ++lev;
    } while (T.count[lev] > 1);
    T.top = lev;
    DBuf<double> dSoa, dBox;
    DBuf<int32_t> dId;
    dSoa.upload(soa, s);
    dBox.upload(box, s);
    dId.upload(order, s);
    DiscsDev D;
    const double* p = dSoa.get();
    D.cx = p;
    D.cy = p + nW;
    D.cz = p + 2 * size_t(nW);
    D.nx = p + 3 * size_t(nW);
    D.ny = p + 4 * size_t(nW);
    D.nz = p + 5 * size_t(nW);
    D.r = p + 6 * size_t(nW);
    D.id = dId.get();
    D.n = nW;
    T.box = dBox.get();
    k_wall_nearest<<<(nC + 127) / 128, 128, 0, s>>>(nC, cellC, D, T, y, nearest);
    VLM_CUDA(cudaGetLastError());
    VLM_CUDA(cudaStreamSynchronize(s));  // the search arrays are freed on return
}

}  // namespace vlm
