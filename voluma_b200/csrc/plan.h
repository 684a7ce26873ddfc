// Device layout plan of a batch of LDU systems and their GAMG hierarchies.
//
// Every level of every system is laid out in "solver order": the rows of one system are
// contiguous; inside a system that still smooths on this level the rows are grouped by
// colour (greedy colouring, natural order inside a colour); every group is padded to a
// multiple of 32 rows so a SELL-32 slice (one warp) never mixes colours or systems.
// Systems are ordered by number of levels (descending), so on each level the systems
// that smooth form a prefix of the rows.
#pragma once

#include <cstdint>
#include <functional>
#include <vector>

#include "box.h"
#include "common.h"
#include "hierarchy.h"

namespace vlm {

struct SysTopo {
    int nCells = 0, nInternal = 0;
    const int32_t* own = nullptr;
    const int32_t* nei = nullptr;
    const double* magSf = nullptr;
    const double* ndc = nullptr;
};

// Block-hybrid Gauss-Seidel: rows of a smoothing system are cut into blocks of kBlockRows
// consecutive natural rows (kBlockRows, common.h); each block is one CTA that runs Gauss-Seidel
// over its rows in block-local colour order, reading neighbours outside the block from the
// previous sweep.
// Level 0 keeps a global multicolour Gauss-Seidel when its graph needs at most this many colours.
constexpr int kMaxGlobalColours = 4;

struct LevelPlan {
    bool blockGS = false;  // block-hybrid layout (else global colour-major)
    int nrows = 0;         // padded rows
    int nfaces = 0;        // faces of the systems present (level 0: user mesh faces)
    int nActiveRows = 0;   // rows of systems that smooth on this level
    int nSteps = 0;        // colour steps of a multicolour sweep (max colours over systems)
    int maxColours = 0;
    // SELL-32 structure: entry k of row r at slPtr[r/32] + 32*k + r%32, k < rlen[r]
    std::vector<int32_t> slPtr, rlen, col, src;  // src >= 0: upper[src]; src < 0: lower[~src]
    std::vector<std::vector<Chunk>> fwd, rev;     // colour step t chunks (forward / reversed)
    std::vector<Chunk> active;                    // all rows of smoothing systems
    std::vector<Chunk> all;                       // all rows (sys/slot set); level 0: kWideRows per chunk
    std::vector<Chunk> blocks;                    // block-hybrid GS blocks (count <= kBlockRows, slot = colours)
    std::vector<int8_t> rowColour;                // block-local colour of each row (block levels)
    std::vector<int32_t> natural;                 // row -> natural index in its system (-1 padding)
    std::vector<int32_t> rowSys;                  // row -> system (batch order), -1 padding
    std::vector<int32_t> sysRow;                  // system -> first row of its block
    std::vector<int32_t> sysFace;                 // system -> first face in this level's face arrays
    // transfer to the next level (defined on rows of smoothing systems)
    std::vector<int32_t> agg;                     // row -> next-level row (-1: padding)
    std::vector<int32_t> childPtr, child;         // next-level row -> rows, ascending natural index
    std::vector<int32_t> intraPtr, intraFace;     // next-level row -> this-level faces inside it
    std::vector<int32_t> cfacePtr, cfaceSrc;      // next-level face -> this-level faces | flip<<31
    // level 0 of a batch of box meshes (box.h): per batch position its descriptor, and per
    // direction d and solver row the user face to the row's +d neighbour (-1: none)
    bool box = false;
    std::vector<BoxSys> boxes;
    std::vector<int32_t> boxFace;                 // [d * nrows + row]
};

struct CoarsePlan {
    int level, rowStart, n, invOffset, sys;
};

struct BatchPlan {
    int nsys = 0;
    std::vector<int> order;        // batch position -> input system index
    std::vector<int> nLevels;      // per batch position
    std::vector<Hierarchy> H;      // per batch position
    std::vector<LevelPlan> levels;
    std::vector<CoarsePlan> coarse;  // per batch position
    int invTotal = 0;              // doubles of all coarse inverses
    // level-0 <-> user arrays (user arrays are concatenations in INPUT order)
    std::vector<int32_t> perm0;    // level-0 row -> user cell (-1 padding)
    std::vector<int64_t> userCellBase, userFaceBase;  // per input system
    int64_t userCells = 0, userFaces = 0;
    std::vector<int32_t> sysSlotBegin, sysSlotEnd;   // level-0 reduction slots per batch position
    std::vector<int32_t> sysCells;                   // real cells per batch position
    int nSlots = 0;
};

// useBox: lay level 0 out for the structured box kernels when every system is a box mesh whose
// natural-order colouring is the red-black parity colouring.
// hierarchy: builds one system's agglomeration hierarchy instead of buildHierarchy (the device
// agglomeration; called for one system at a time).
BatchPlan buildPlan(const std::vector<SysTopo>& systems, int mergeLevels, bool useBox = true,
                    const std::function<Hierarchy(const SysTopo&)>& hierarchy = {});

}  // namespace vlm
