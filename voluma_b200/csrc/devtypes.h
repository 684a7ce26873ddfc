// Plain structs shared by the host orchestration and the device kernels.
#pragma once

#include <cstdint>

#include "common.h"

namespace vlm {

// Per-system solver state, resident on the device.
struct SysState {
    double normFactor, initialResidual, finalResidual, residualSum;
    double wArA, wArAold, alpha, beta, omega, rho, rhoOld, s0, s1;
    double innerInit, innerFinal;  // mixed precision inner solve (FP32 L1 norms)
    int iterations, converged, done, status;
    int innerIterations, innerDone, outer, pad;
};

// Solve controls as seen by the device.
struct DevCtrl {
    double tolerance, relTol, innerRelTol;
    int maxIter, minIter, maxInner;
};

// Double-double accumulator of the compensated reductions.
struct DD {
    double hi, lo;
};

// Reduction context: per-CTA partial slots and per-system completion counters.
struct RedCtx {
    DD* partials;           // [slot * NV + q]
    long long* xbins;       // exact sums: [slot][NV][bins + flags]
    int* counters;          // per system
    const int* slotBegin;   // per system
    const int* slotEnd;
};

// SELL-32 structure of one level.
struct Sell {
    const int32_t* slPtr;
    const int32_t* rlen;
    const int32_t* col;
};

// Coarsest-level solve of one system.
struct CoarseDev {
    int rowStart, n, invOffset, sys;
};

// Arrays of one level as the coarse-tail kernel sees them (one table per precision).
template <class T>
struct TailLevel {
    Sell S;
    const T* val;
    const T* diag;
    T* r;                   // null on level 0 (the V-cycle's own input is passed instead)
    T* x;                   // null on level 0 (the V-cycle's own output)
    T* x2;                  // Jacobi ping-pong vector
    const int32_t* agg;     // row -> next-level row (-1: padding)
    const int32_t* cptr;    // next-level row -> its children on this level
    const int32_t* child;
};

// One system's part of the coarse tail: levels first..coarsest of the V-cycle run in one
// thread-block cluster.
constexpr int kTailMaxLevels = 32;
struct TailSys {
    int sys, first, coarsest;  // batch position; first tail level; coarsest level
    int coarseN, invOffset;
    int rowStart[kTailMaxLevels], rowCount[kTailMaxLevels];
    // level 0 in the tail (first == 0) with global multicolour Gauss-Seidel: the system's colour
    // groups (padded row ranges) and whether the batch runs the two-colour fused schedule
    int nColours, two;
    int grpStart[4], grpCount[4];
};

}  // namespace vlm
