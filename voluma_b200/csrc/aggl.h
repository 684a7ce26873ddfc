// Device-side GAMG agglomeration for meshes registered with VLM_MESH_DEVICE_AGGLOMERATION.
//
// The reference builds its pairwise aggregates by a sequential greedy pass in cell order
// (GAMG.cpp:40-94): each unpaired cell takes its most strongly coupled unpaired neighbour.  The
// device form is a parallel handshake matching of the same couplings: in rounds, every unpaired
// cell names its heaviest unpaired neighbour (weight magSf*ndc as in GAMG.cpp:215; equal weights
// are ordered by a hash of the two cells, identical from both ends) and mutual choices pair up,
// until no unpaired cell has an unpaired neighbour; a cell left alone joins the aggregate of its
// heaviest neighbour, as in the reference.  Aggregates are numbered by their first cell, coarse faces
// by their (lower, upper) aggregate pair, coarse weights are the fine weights summed in face order.
// The level structure (mergeLevels passes per level, coarsening while n > nCoarsest) is
// buildHierarchy's, so everything downstream (plan, Galerkin, V-cycle) is unchanged; the aggregates
// differ from the sequential pass, so iteration counts are compared with the same algorithm's
// CPU restatement, not with the reference's.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "hierarchy.h"

namespace vlm {

Hierarchy buildHierarchyDevice(cudaStream_t stream, int nCells, int nInternal, const int32_t* own, const int32_t* nei,
                               const double* magSf, const double* ndc, int mergeLevels, int nCoarsest = 64);

}  // namespace vlm
