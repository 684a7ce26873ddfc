// Level schedule of the DIC/DILU preconditioner (LinearSolver.cpp:28-112) on the device.
//
// The reference factorises and applies DILU in natural cell order over the faces sorted by
// (upper cell, lower cell): rD[u] -= A_lu A_ul / rD[l], then a forward sweep
// w[u] -= rD[u] A_ul w[l] and a backward sweep w[l] -= rD[l] A_lu w[u].  Each is a recurrence
// along the natural-order dependency graph (l -> u for every face), so rows can be updated in
// parallel exactly when they sit on the same level of that graph: level[u] = 1 + max level[l]
// over its lower neighbours.  Inside a row the terms are applied in the reference's order
// (forward: lower neighbours by ascending (l, face); backward: upper neighbours by descending
// (u, face)), so the device result is the reference's, bit for bit.
#pragma once

#include <cstdint>
#include <vector>

#include "plan.h"

namespace vlm {

// One system's part of the schedule (batch position `sys`): levels [levBegin, levBegin + nLev) of
// the concatenated level table.
struct DiluSys {
    int sys, levBegin, nLev, rowBegin, rowCount;  // rows [rowBegin, rowBegin + rowCount) of level 0
    int slotBegin, slotEnd;                       // its slots: levRows[slotBegin .. slotEnd)
    int loBegin, loEnd, upBegin, upEnd;           // its entries of the streamed schedule
};

// One level of the streamed schedule: slots [s0, s0 + width) of levRows; entry j of slot s0 + q at
// lo + j * width + q (j < mlo, lower neighbours in forward order) and up + j * width + q (j < mup,
// upper neighbours in backward order).  A row with fewer entries pads its column with -1.  A level's
// rows, scalars and entries are contiguous, so a CTA can stream them into shared memory levels ahead
// of the sweep without looking anything up.
struct DiluLevel {
    int s0, width, lo, mlo, up, mup;
};

struct DiluPlan {
    // per level-0 row (solver order): lower neighbours (forward order) and upper neighbours
    // (backward order); face = user face index | ownerIsL << 31
    std::vector<int32_t> loPtr, loCol, loFace;
    std::vector<int32_t> upPtr, upCol, upFace;
    // level schedule: levPtr[levBegin + t] .. levPtr[levBegin + t + 1] index levRows (solver rows);
    // padding rows are on level 0 of their system
    std::vector<int32_t> levPtr, levRows;
    std::vector<DiluSys> sys;
    // streamed schedule (per level of levPtr): slot -> row - rowBegin, entries (local column or -1,
    // face as loFace)
    std::vector<DiluLevel> lev;
    std::vector<int32_t> slotRow;
    std::vector<int32_t> sLoCol, sLoFace, sUpCol, sUpFace;
    int maxEnt = 0;    // largest mlo / mup of any level
    int maxWidth = 0;  // widest level over all systems
    int maxLevels = 0;
    int maxRows = 0;   // largest system (level-0 rows incl. padding)
};

// systems: input order; P: the batch plan (solver order, perm0).
DiluPlan buildDiluPlan(const std::vector<SysTopo>& systems, const BatchPlan& P);

}  // namespace vlm
