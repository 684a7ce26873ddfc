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
    // defect correction around a reference row (the one row of A with a non-zero row sum): A =
    // L + refC e_ref e_ref^T with L's rows summing to zero; sumR = sum of the outer residual,
    // innerMu = mean of the inner iteration's preconditioned residual
    double refC, sumR, innerMu;
    int iterations, converged, done, status;
    int innerIterations, innerDone, outer, pad;
    int refRow, refCount;  // refRow < 0: no single reference row (no projection)
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

// One system's coarse tail in shared memory (k_vcycle_tail_smem): the Jacobi levels first..coarsest-1
// as ELL rows with 16-bit local columns, the coarsest level's dense inverse, and every level's
// vectors.  t* are element offsets into the T region of shared memory (the value image, then the
// vectors), u* into the uint16 region (structure image).
#ifdef __CUDACC__
#define VLM_HD __host__ __device__
#else
#define VLM_HD
#endif
VLM_HD constexpr size_t tail_align16(size_t b) { return (b + 15) & ~size_t(15); }

// Shared-memory bytes of one system's tail: the T region, the coarsest inverse (doubles), the
// uint16 region, each starting on a 16-byte boundary.
VLM_HD inline size_t tail_smem_bytes(size_t tsize, int tCount, int nc, int strCount) {
    return tail_align16(size_t(tCount) * tsize) + tail_align16(size_t(nc) * nc * sizeof(double)) +
           tail_align16(size_t(strCount) * sizeof(uint16_t));
}

struct TailImg {
    int sys, first, coarsest, nc, invOffset;
    int valOff, strOff;              // offsets of this system's images in the batch's image buffers
    int valCount, tCount, strCount;  // value-image T count; T count in shared memory; uint16 count
    int n[kTailMaxLevels], W[kTailMaxLevels], rowStart[kTailMaxLevels];
    int tDiag[kTailMaxLevels], tVal[kTailMaxLevels], tR[kTailMaxLevels], tX[kTailMaxLevels], tX2[kTailMaxLevels];
    int uRlen[kTailMaxLevels], uCol[kTailMaxLevels], uAgg[kTailMaxLevels], uCptr[kTailMaxLevels],
        uChild[kTailMaxLevels];
};

}  // namespace vlm
