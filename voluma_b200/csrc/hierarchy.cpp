// Host-side GAMG topology (once per mesh, cached on the vlm_mesh like the reference caches
// it on the Mesh, src/fvm/linalg/GAMG.cpp:204).
//
// The agglomeration must reproduce the reference hierarchy exactly (same aggregates, same
// coarse-face numbering, same weights summed in the same order), because the coarse
// operators and therefore the iteration counts depend on it.  The steps follow
// GAMG.cpp:15-94 (adjacency, greedy heaviest-edge pairing, orphan merge, first-occurrence
// coarse-face numbering) and GAMG.cpp:206-252 (level loop with mergeLevels passes).
#include "hierarchy.h"

#include <algorithm>
#include <stdexcept>

namespace vlm {

// Row adjacency in face order: each face f adds (l -> u) then (u -> l)  (GAMG.cpp:15-37).
void makeAdjacency(HLevel& L) {
    const size_t nf = L.l.size();
    L.off.assign(size_t(L.n) + 1, 0);
    for (size_t f = 0; f < nf; ++f) {
        L.off[L.l[f] + 1]++;
        L.off[L.u[f] + 1]++;
    }
    for (int i = 0; i < L.n; ++i) L.off[i + 1] += L.off[i];
    const size_t nnz = size_t(L.off[L.n]);
    L.adjCell.resize(nnz);
    L.adjFace.resize(nnz);
    L.adjIsL.resize(nnz);
    std::vector<int> pos(L.off.begin(), L.off.end() - 1);
    for (size_t f = 0; f < nf; ++f) {
        int k = pos[L.l[f]]++;
        L.adjCell[k] = L.u[f];
        L.adjFace[k] = int(f);
        L.adjIsL[k] = 1;
        k = pos[L.u[f]]++;
        L.adjCell[k] = L.l[f];
        L.adjFace[k] = int(f);
        L.adjIsL[k] = 0;
    }
}

namespace {

// One pairwise pass; fills L.agg/faceMap/faceFlip and returns the coarse level's faces and
// weights (no adjacency yet)  (GAMG.cpp:40-94).
HLevel pairPass(HLevel& L) {
    L.agg.assign(size_t(L.n), -1);
    int nAgg = 0;
    for (int i = 0; i < L.n; ++i) {
        if (L.agg[i] >= 0) continue;
        int partner = -1;
        double heaviest = -1.0;
        for (int k = L.off[i]; k < L.off[i + 1]; ++k) {
            const int j = L.adjCell[k];
            const double wgt = L.weight[L.adjFace[k]];
            if (j != i && L.agg[j] < 0 && wgt > heaviest) {
                heaviest = wgt;
                partner = j;
            }
        }
        if (partner >= 0) {
            L.agg[i] = nAgg;
            L.agg[partner] = nAgg;
            ++nAgg;
            continue;
        }
        // every neighbour is taken: join the aggregate of the most strongly coupled one
        for (int k = L.off[i]; k < L.off[i + 1]; ++k) {
            const double wgt = L.weight[L.adjFace[k]];
            if (wgt > heaviest) {
                heaviest = wgt;
                partner = L.adjCell[k];
            }
        }
        L.agg[i] = partner >= 0 ? L.agg[partner] : nAgg++;
    }
    HLevel C;
    C.n = nAgg;
    const int nf = int(L.l.size());
    L.faceMap.assign(size_t(nf), -1);
    L.faceFlip.assign(size_t(nf), 0);
    // Coarse faces are numbered by the first fine face (in face order) that joins their aggregate
    // pair.  That first face (the pair's leader) is found without hashing: the fine faces are
    // bucketed by their lower aggregate (a stable counting sort, so each bucket is in face order)
    // and each bucket is scanned with a per-aggregate marker of the last bucket that saw it.
    std::vector<int> fa(static_cast<size_t>(nf)), fb(static_cast<size_t>(nf));  // each face's two aggregates
    std::vector<int> start(size_t(nAgg) + 1, 0);
    for (int f = 0; f < nf; ++f) {
        const int a = L.agg[L.l[f]], b = L.agg[L.u[f]];
        fa[f] = a;
        fb[f] = b;
        if (a != b) start[size_t(a < b ? a : b) + 1]++;
    }
    for (int c = 0; c < nAgg; ++c) start[c + 1] += start[c];
    std::vector<int> bucketFace(static_cast<size_t>(start[nAgg])), bucketHi(static_cast<size_t>(start[nAgg]));
    {
        std::vector<int> pos(start.begin(), start.end() - 1);
        for (int f = 0; f < nf; ++f) {
            const int a = fa[f], b = fb[f];
            if (a == b) continue;
            const int k = pos[a < b ? a : b]++;
            bucketFace[k] = f;
            bucketHi[k] = a < b ? b : a;
        }
    }
    std::vector<int> leader(size_t(nf), -1), markLo(size_t(nAgg), -1), markFace(size_t(nAgg), -1);
    size_t nCoarseFaces = 0;
    for (int lo = 0; lo < nAgg; ++lo)
        for (int k = start[lo]; k < start[lo + 1]; ++k) {
            const int f = bucketFace[k], hi = bucketHi[k];
            if (markLo[hi] != lo) {
                markLo[hi] = lo;
                markFace[hi] = f;
                ++nCoarseFaces;
            }
            leader[f] = markFace[hi];
        }
    C.l.reserve(nCoarseFaces);
    C.u.reserve(nCoarseFaces);
    C.weight.reserve(nCoarseFaces);
    for (int f = 0; f < nf; ++f) {
        const int a = fa[f], b = fb[f];
        if (a == b) continue;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        int cf;
        if (leader[f] == f) {
            cf = int(C.l.size());
            C.l.push_back(lo);
            C.u.push_back(hi);
            C.weight.push_back(0.0);
        } else {
            cf = L.faceMap[leader[f]];  // the leader precedes f and is numbered already
        }
        L.faceMap[f] = cf;
        L.faceFlip[f] = char(a != lo);
        C.weight[cf] += L.weight[f];
    }
    return C;
}

}  // namespace

Hierarchy buildHierarchy(int nCells, int nInternal, const int32_t* own, const int32_t* nei, const double* magSf,
                         const double* ndc, int mergeLevels, int nCoarsest) {
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
    makeAdjacency(L0);
    H.levels.push_back(std::move(L0));
    while (H.levels.size() < 40) {
        HLevel& F = H.levels.back();
        const int nF = F.n;
        if (nF <= nCoarsest) break;
        HLevel C = pairPass(F);
        for (int pass = 1; pass < mergeLevels && C.n > nCoarsest; ++pass) {
            makeAdjacency(C);
            HLevel C2 = pairPass(C);
            for (auto& a : F.agg) a = C.agg[a];
            for (size_t f = 0; f < F.faceMap.size(); ++f) {
                const int cf = F.faceMap[f];
                if (cf < 0) continue;
                F.faceMap[f] = C.faceMap[cf];
                F.faceFlip[f] = char(F.faceFlip[f] != C.faceFlip[cf]);
            }
            C = std::move(C2);
        }
        if (C.n >= nF) {  // no further coarsening possible
            F.agg.clear();
            break;
        }
        makeAdjacency(C);
        H.levels.push_back(std::move(C));
    }
    // The coarsest level never carries transfer maps.
    H.levels.back().agg.clear();
    H.levels.back().faceMap.clear();
    H.levels.back().faceFlip.clear();
    return H;
}

std::vector<int> greedyColour(const HLevel& L, int* nColours) {
    std::vector<int> colour(size_t(L.n), -1);
    std::vector<int> mark;  // mark[c] == i  <=>  colour c is used by a neighbour of i
    int nc = 0;
    for (int i = 0; i < L.n; ++i) {
        for (int k = L.off[i]; k < L.off[i + 1]; ++k) {
            const int c = colour[L.adjCell[k]];
            if (c >= 0) {
                if (size_t(c) >= mark.size()) mark.resize(size_t(c) + 1, -1);
                mark[c] = i;
            }
        }
        int c = 0;
        while (size_t(c) < mark.size() && mark[c] == i) ++c;
        colour[i] = c;
        nc = std::max(nc, c + 1);
    }
    *nColours = nc;
    return colour;
}

}  // namespace vlm
