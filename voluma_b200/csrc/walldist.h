// Nearest wall face of every cell, as WallDistance.cpp (src/fvm/mesh/WallDistance.cpp) defines it:
// among the K = 8 wall faces whose centres lie nearest the cell centre, the one at the smallest
// distance when each face is taken as a disc of its area (ties to the lower wall-face index).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace vlm {

// One wall face as a disc: centre, unit normal into the fluid, radius.
struct WallDisc {
    double c[3], n[3], r;
};

// The 8 nearest centres are taken in the order (squared distance, wall-face index), so where the
// 8th and 9th nearest centres are equally far the lower index is kept.
// cellC: device array of cell centres (x of every cell, then y, then z).  Writes y[c] (the disc
// distance) and nearest[c] (the wall-face index) for the nC cells, on stream s.
void wallNearestOnDevice(cudaStream_t s, int nC, const double* cellC, const std::vector<WallDisc>& discs,
                         double* y, int32_t* nearest);

}  // namespace vlm
