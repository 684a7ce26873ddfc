// Host-side construction of the shared-memory coarse tail's images (k_vcycle_tail_smem).
#pragma once

#include <cstdint>
#include <vector>

#include "devtypes.h"
#include "plan.h"

namespace vlm {

struct TailImages {
    std::vector<TailImg> imgs;       // per tail system
    std::vector<int32_t> codes;      // value-image gather codes (k_tail_values)
    std::vector<uint16_t> str;       // structure images
    size_t bytes64 = 0, bytes32 = 0; // dynamic shared memory of the largest system, FP64 / FP32
};

// Builds the images of every system of `ts` (levels first..coarsest): false when a system starts at
// level 0, a level exceeds the 16-bit local indices, or a system's FP64 images and vectors exceed
// `budget` bytes of shared memory.
bool buildTailImages(const BatchPlan& plan, const std::vector<TailSys>& ts, size_t budget, TailImages& out);

}  // namespace vlm
