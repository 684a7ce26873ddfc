// Device-side GAMG agglomeration (aggl.h): parallel handshake matching, aggregate numbering and
// coarse faces by a stable radix sort of (lower, upper) aggregate pairs.
#include "aggl.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.h"

namespace vlm {

namespace {

constexpr int kAggThreads = 256;
inline int nblocks(int64_t n) { return int((n + kAggThreads - 1) / kAggThreads); }

// SplitMix64 finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014): orders equal couplings by a hash of their two cells, the same seen from either end.
__device__ __forceinline__ uint64_t pairHash(int a, int b) {
    const uint32_t lo = uint32_t(a < b ? a : b), hi = uint32_t(a < b ? b : a);
    uint64_t z = (uint64_t(lo) << 32 | hi) + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ bool heavier(double w, uint64_t h, double bw, uint64_t bh) {
    return w > bw || (w == bw && h > bh);
}

__global__ void k_agg_degree(int nf, const int* __restrict__ l, const int* __restrict__ u, int* __restrict__ deg) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    atomicAdd(deg + l[f], 1);
    atomicAdd(deg + u[f], 1);
}

// Row adjacency in any order: the matching only compares couplings, never their position.
__global__ void k_agg_fill(int nf, const int* __restrict__ l, const int* __restrict__ u, const double* __restrict__ w,
                           int* __restrict__ cursor, int* __restrict__ adjCell, double* __restrict__ adjW) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    int k = atomicAdd(cursor + l[f], 1);
    adjCell[k] = u[f];
    adjW[k] = w[f];
    k = atomicAdd(cursor + u[f], 1);
    adjCell[k] = l[f];
    adjW[k] = w[f];
}

// Every unpaired cell names its heaviest unpaired neighbour (-1: none).
__global__ void k_agg_prefer(int n, const int* __restrict__ off, const int* __restrict__ adjCell,
                             const double* __restrict__ adjW, const int* __restrict__ match, int* __restrict__ pref) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int best = -1;
    if (match[i] < 0) {
        double bw = 0.0;
        uint64_t bh = 0;
        for (int k = off[i]; k < off[i + 1]; ++k) {
            const int j = adjCell[k];
            if (match[j] >= 0) continue;
            const double w = adjW[k];
            const uint64_t h = pairHash(i, j);
            if (best < 0 || heavier(w, h, bw, bh)) {
                best = j;
                bw = w;
                bh = h;
            }
        }
    }
    pref[i] = best;
}

// Mutual choices pair up.
__global__ void k_agg_handshake(int n, const int* __restrict__ pref, int* __restrict__ match, int* __restrict__ paired) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || match[i] >= 0) return;
    const int j = pref[i];
    if (j >= 0 && pref[j] == i) {
        match[i] = j;
        atomicAdd(paired, 1);
    }
}

// Aggregate leaders: the lower cell of a pair, and a cell without neighbours.
__global__ void k_agg_leaders(int n, const int* __restrict__ off, const int* __restrict__ match, int* __restrict__ lead) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = match[i];
    lead[i] = m >= 0 ? (i < m ? 1 : 0) : (off[i + 1] == off[i] ? 1 : 0);
}

// Aggregate of every cell; a cell left unpaired (every neighbour paired) joins its heaviest neighbour's.
__global__ void k_agg_assign(int n, const int* __restrict__ off, const int* __restrict__ adjCell,
                             const double* __restrict__ adjW, const int* __restrict__ match,
                             const int* __restrict__ lead, const int* __restrict__ id, int* __restrict__ agg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int m = match[i];
    if (m >= 0) {
        agg[i] = id[i < m ? i : m];
        return;
    }
    if (lead[i]) {
        agg[i] = id[i];
        return;
    }
    int best = -1;
    double bw = 0.0;
    uint64_t bh = 0;
    for (int k = off[i]; k < off[i + 1]; ++k) {
        const int j = adjCell[k];
        const uint64_t h = pairHash(i, j);
        if (best < 0 || heavier(adjW[k], h, bw, bh)) {
            best = j;
            bw = adjW[k];
            bh = h;
        }
    }
    const int mb = match[best];
    agg[i] = id[best < mb ? best : mb];
}

// Sort keys of the fine faces: (lower, upper) aggregate pair; faces inside an aggregate sort last.
__global__ void k_agg_face_keys(int nf, const int* __restrict__ l, const int* __restrict__ u,
                                const int* __restrict__ agg, uint64_t* __restrict__ key, int* __restrict__ face) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int a = agg[l[f]], b = agg[u[f]];
    key[f] = a == b ? ~uint64_t(0) : (uint64_t(uint32_t(a < b ? a : b)) << 32 | uint32_t(a < b ? b : a));
    face[f] = f;
}

__global__ void k_agg_heads(int nf, const uint64_t* __restrict__ key, int* __restrict__ head) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    head[k] = key[k] != ~uint64_t(0) && (k == 0 || key[k] != key[k - 1]) ? 1 : 0;
}

// Coarse faces: numbered in (lower, upper) order; weights summed over their fine faces in face
// order (the stable sort keeps it); fine face -> coarse face and orientation.
__global__ void k_agg_coarse_faces(int nf, const uint64_t* __restrict__ key, const int* __restrict__ face,
                                   const int* __restrict__ head, const int* __restrict__ cid,
                                   const int* __restrict__ l, const int* __restrict__ agg,
                                   const double* __restrict__ w, int* __restrict__ cl, int* __restrict__ cu,
                                   double* __restrict__ cw, int* __restrict__ faceMap, int8_t* __restrict__ flip) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nf) return;
    const int f = face[k];
    const uint64_t kk = key[k];
    if (kk == ~uint64_t(0)) {
        faceMap[f] = -1;
        flip[f] = 0;
        return;
    }
    const int c = cid[k] + head[k] - 1;  // cid counts the heads before k: a segment's number is its head's
    const int lo = int(kk >> 32), hi = int(kk & 0xffffffffu);
    faceMap[f] = c;
    flip[f] = int8_t(agg[l[f]] != lo);
    if (!head[k]) return;
    cl[c] = lo;
    cu[c] = hi;
    double s = 0.0;
    for (int q = k; q < nf && key[q] == kk; ++q) s += w[face[q]];
    cw[c] = s;
}

template <class T>
std::vector<T> download(const DBuf<T>& d, size_t n, cudaStream_t s) {
    std::vector<T> h(n);
    if (n) VLM_CUDA(cudaMemcpyAsync(h.data(), d.get(), n * sizeof(T), cudaMemcpyDeviceToHost, s));
    VLM_CUDA(cudaStreamSynchronize(s));
    return h;
}

template <class T>
void exclusiveScan(const T* in, T* out, int n, cudaStream_t s) {
    size_t bytes = 0;
    VLM_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n, s));
    DBuf<unsigned char> tmp(std::max<size_t>(bytes, 1));
    VLM_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, in, out, n, s));
    VLM_CUDA(cudaStreamSynchronize(s));  // tmp is released on return
}

// One level on the device: n cells, faces (l < u) with weights.
struct DevLevelFaces {
    int n = 0, nf = 0;
    DBuf<int> l, u;
    DBuf<double> w;
};

// One pairwise pass: the level's aggregates, face map and flips (host), and the coarse level.
struct PassResult {
    std::vector<int> agg, faceMap;
    std::vector<char> flip;
    DevLevelFaces coarse;
};

PassResult devicePass(cudaStream_t s, const DevLevelFaces& F) {
    const int n = F.n, nf = F.nf;
    PassResult R;
    // adjacency
    DBuf<int> off(size_t(n) + 1), deg(size_t(n) + 1), cursor(size_t(n) + 1);
    deg.zero(s);
    if (nf) k_agg_degree<<<nblocks(nf), kAggThreads, 0, s>>>(nf, F.l.get(), F.u.get(), deg.get());
    exclusiveScan(deg.get(), off.get(), n + 1, s);
    VLM_CUDA(cudaMemcpyAsync(cursor.get(), off.get(), sizeof(int) * (size_t(n) + 1), cudaMemcpyDeviceToDevice, s));
    const size_t nnz = size_t(2) * nf;
    DBuf<int> adjCell(std::max<size_t>(nnz, 1));
    DBuf<double> adjW(std::max<size_t>(nnz, 1));
    if (nf)
        k_agg_fill<<<nblocks(nf), kAggThreads, 0, s>>>(nf, F.l.get(), F.u.get(), F.w.get(), cursor.get(),
                                                       adjCell.get(), adjW.get());
    // handshake rounds until no pair forms (then no unpaired cell has an unpaired neighbour: the
    // heaviest coupling among unpaired cells is always mutual)
    DBuf<int> match(size_t(std::max(n, 1))), pref(size_t(std::max(n, 1))), paired(1);
    VLM_CUDA(cudaMemsetAsync(match.get(), 0xff, sizeof(int) * size_t(n), s));
    for (int round = 0;; ++round) {
        if (round > 10000) throw Error(VLM_ERR_CUDA, "internal: device agglomeration did not converge");
        paired.zero(s);
        k_agg_prefer<<<nblocks(n), kAggThreads, 0, s>>>(n, off.get(), adjCell.get(), adjW.get(), match.get(),
                                                        pref.get());
        k_agg_handshake<<<nblocks(n), kAggThreads, 0, s>>>(n, pref.get(), match.get(), paired.get());
        int h = 0;
        VLM_CUDA(cudaMemcpyAsync(&h, paired.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
        if (h == 0) break;
    }
    // aggregates
    DBuf<int> lead(size_t(n) + 1), id(size_t(n) + 1), agg(size_t(std::max(n, 1)));
    lead.zero(s);
    k_agg_leaders<<<nblocks(n), kAggThreads, 0, s>>>(n, off.get(), match.get(), lead.get());
    exclusiveScan(lead.get(), id.get(), n + 1, s);
    int nAgg = 0;
    VLM_CUDA(cudaMemcpyAsync(&nAgg, id.get() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    k_agg_assign<<<nblocks(n), kAggThreads, 0, s>>>(n, off.get(), adjCell.get(), adjW.get(), match.get(),
                                                    lead.get(), id.get(), agg.get());
    // coarse faces
    DBuf<uint64_t> key(std::max<size_t>(size_t(nf), 1)), keyS(std::max<size_t>(size_t(nf), 1));
    DBuf<int> face(std::max<size_t>(size_t(nf), 1)), faceS(std::max<size_t>(size_t(nf), 1));
    DBuf<int> head(size_t(nf) + 1), cid(size_t(nf) + 1);
    DBuf<int> faceMap(std::max<size_t>(size_t(nf), 1));
    DBuf<int8_t> flip(std::max<size_t>(size_t(nf), 1));
    int nc = 0;
    head.zero(s);
    if (nf) {
        k_agg_face_keys<<<nblocks(nf), kAggThreads, 0, s>>>(nf, F.l.get(), F.u.get(), agg.get(), key.get(), face.get());
        size_t bytes = 0;
        VLM_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, key.get(), keyS.get(), face.get(), faceS.get(), nf,
                                                 0, 64, s));
        DBuf<unsigned char> tmp(std::max<size_t>(bytes, 1));
        VLM_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), bytes, key.get(), keyS.get(), face.get(), faceS.get(),
                                                 nf, 0, 64, s));
        k_agg_heads<<<nblocks(nf), kAggThreads, 0, s>>>(nf, keyS.get(), head.get());
        exclusiveScan(head.get(), cid.get(), nf + 1, s);
        VLM_CUDA(cudaMemcpyAsync(&nc, cid.get() + nf, sizeof(int), cudaMemcpyDeviceToHost, s));
        VLM_CUDA(cudaStreamSynchronize(s));
    }
    DevLevelFaces& C = R.coarse;
    VLM_CUDA(cudaStreamSynchronize(s));
    C.n = nAgg;
    C.nf = nc;
    C.l.resize(size_t(std::max(nc, 1)));
    C.u.resize(size_t(std::max(nc, 1)));
    C.w.resize(size_t(std::max(nc, 1)));
    if (nf) {
        k_agg_coarse_faces<<<nblocks(nf), kAggThreads, 0, s>>>(nf, keyS.get(), faceS.get(), head.get(), cid.get(),
                                                               F.l.get(), agg.get(), F.w.get(), C.l.get(), C.u.get(),
                                                               C.w.get(), faceMap.get(), flip.get());
        VLM_CUDA(cudaGetLastError());
    }
    R.agg = download(agg, size_t(n), s);
    R.faceMap = download(faceMap, size_t(nf), s);
    const std::vector<int8_t> fl = download(flip, size_t(nf), s);
    R.flip.assign(fl.begin(), fl.end());
    return R;
}

}  // namespace

Hierarchy buildHierarchyDevice(cudaStream_t s, int nCells, int nInternal, const int32_t* own, const int32_t* nei,
                               const double* magSf, const double* ndc, int mergeLevels, int nCoarsest) {
    if (mergeLevels < 1) mergeLevels = 1;
    Hierarchy H;
    HLevel L0;
    L0.n = nCells;
    L0.l.reserve(size_t(nInternal));
    L0.u.reserve(size_t(nInternal));
    L0.weight.reserve(size_t(nInternal));
    H.ownerIsL.reserve(size_t(nInternal));
    for (int f = 0; f < nInternal; ++f) {
        const int o = own[f], n = nei[f];
        if (o < 0 || n < 0 || o >= nCells || n >= nCells || o == n)
            throw std::invalid_argument("mesh face " + std::to_string(f) + " has an invalid or self-coupled cell pair");
        L0.l.push_back(o < n ? o : n);
        L0.u.push_back(o < n ? n : o);
        L0.weight.push_back(magSf[f] * ndc[f]);
        H.ownerIsL.push_back(char(o < n));
    }
    DevLevelFaces cur;
    cur.n = nCells;
    cur.nf = nInternal;
    cur.l.upload(L0.l, s);
    cur.u.upload(L0.u, s);
    cur.w.upload(L0.weight, s);
    makeAdjacency(L0);
    H.levels.push_back(std::move(L0));
    while (H.levels.size() < 40) {
        HLevel& F = H.levels.back();
        const int nF = F.n;
        if (nF <= nCoarsest) break;
        PassResult P = devicePass(s, cur);
        F.agg = std::move(P.agg);
        F.faceMap = std::move(P.faceMap);
        F.faceFlip = std::move(P.flip);
        DevLevelFaces C = std::move(P.coarse);
        for (int pass = 1; pass < mergeLevels && C.n > nCoarsest; ++pass) {
            PassResult Q = devicePass(s, C);
            for (auto& a : F.agg) a = Q.agg[size_t(a)];
            for (size_t f = 0; f < F.faceMap.size(); ++f) {
                const int cf = F.faceMap[f];
                if (cf < 0) continue;
                F.faceMap[f] = Q.faceMap[size_t(cf)];
                F.faceFlip[f] = char(F.faceFlip[f] != Q.flip[size_t(cf)]);
            }
            C = std::move(Q.coarse);
        }
        if (C.n >= nF) {  // no further coarsening possible
            F.agg.clear();
            break;
        }
        HLevel L;
        L.n = C.n;
        L.l.resize(size_t(C.nf));
        L.u.resize(size_t(C.nf));
        L.weight.resize(size_t(C.nf));
        if (C.nf) {
            VLM_CUDA(cudaMemcpyAsync(L.l.data(), C.l.get(), sizeof(int) * size_t(C.nf), cudaMemcpyDeviceToHost, s));
            VLM_CUDA(cudaMemcpyAsync(L.u.data(), C.u.get(), sizeof(int) * size_t(C.nf), cudaMemcpyDeviceToHost, s));
            VLM_CUDA(cudaMemcpyAsync(L.weight.data(), C.w.get(), sizeof(double) * size_t(C.nf),
                                     cudaMemcpyDeviceToHost, s));
            VLM_CUDA(cudaStreamSynchronize(s));
        }
        makeAdjacency(L);
        H.levels.push_back(std::move(L));
        cur = std::move(C);
    }
    // the coarsest level never carries transfer maps
    H.levels.back().agg.clear();
    H.levels.back().faceMap.clear();
    H.levels.back().faceFlip.clear();
    return H;
}

}  // namespace vlm
