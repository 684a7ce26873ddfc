// Host-side GAMG topology: pairwise agglomeration hierarchy and per-level colouring.
#pragma once

#include <cstdint>
#include <vector>

namespace vlm {

// One level of the agglomeration hierarchy, natural (hierarchy) numbering.
// Same content as the reference's GamgLevel (src/fvm/linalg/GAMG.h:18-27).
struct HLevel {
    int n = 0;
    std::vector<int> l, u;            // faces with l < u
    std::vector<double> weight;       // geometric agglomeration weight per face
    std::vector<int> off, adjCell, adjFace;  // row adjacency CSR in face order
    std::vector<char> adjIsL;         // row is the l end of the face (A(i,j) = upper)
    std::vector<int> agg;             // cell -> next-level cell (empty on the coarsest level)
    std::vector<int> faceMap;         // face -> next-level face, -1 inside an aggregate
    std::vector<char> faceFlip;       // next-level face orientation reversed
};

struct Hierarchy {
    std::vector<HLevel> levels;
    std::vector<char> ownerIsL;       // level-0 face k (= mesh face k): owner is the l end
};

// buildHierarchy (src/fvm/linalg/GAMG.cpp:206-261), serial form: level 0 = all internal
// faces (self-coupled faces are rejected by the caller), weight = magSf*ndc, coarsen while
// n > nCoarsest with mergeLevels pairwise passes per level.
Hierarchy buildHierarchy(int nCells, int nInternal, const int32_t* own, const int32_t* nei, const double* magSf,
                         const double* ndc, int mergeLevels, int nCoarsest = 64);

// Row adjacency (off/adjCell/adjFace/adjIsL) of a level from its faces, in face order.
void makeAdjacency(HLevel& L);

// Greedy colouring in natural order (smallest colour unused by already coloured neighbours).
std::vector<int> greedyColour(const HLevel& L, int* nColours);

}  // namespace vlm
