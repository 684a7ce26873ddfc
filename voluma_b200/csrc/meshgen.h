// Device-side box mesh setup: generateBox + Mesh::build geometry as kernels (meshgen.cu).
#pragma once

#include <cstdint>
#include <vector>

#include "common.h"

namespace vlm {

// The compute mesh of a box in host memory (the vlm_mesh_desc arrays, vectors AoS), built on the device.
struct BoxMesh {
    int nCells = 0, nInternal = 0, nFaces = 0, twoD = 0, emptyDir = -1;
    std::vector<int32_t> owner, neighbour, patchStart, patchSize, patchSide;
    std::vector<double> V, C, Sf, Cf, d, magSf, w, ndc, corrVecs, skewVecs;
};

BoxMesh buildBoxMesh(const vlm_box_spec& spec, cudaStream_t stream);

}  // namespace vlm
