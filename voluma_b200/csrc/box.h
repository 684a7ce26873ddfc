// Structured level 0 of box meshes.
//
// The meshes of every pressure case here are boxes (generateBox, src/fvm/mesh/RawMesh.cpp:391-502):
// cell (i,j,k) = i + nx(j + ny k), internal faces in owner order (+x, +y, +z of each cell), then the
// cyclic pairs of the periodic directions (x, then y, then z; owner on the min side).  On such a
// mesh the two-colour (red-black) Gauss-Seidel order of level 0 has a closed form, so the level-0
// row kernels find every neighbour by index arithmetic and read each face coefficient from one
// array per direction (stored once, at the cell on the face's minus side), instead of walking a
// SELL row of column indices and per-row copies of the coefficients.
//
// Solver-row layout of a box system on level 0 (colour C = parity of i+j+k; greedy natural-order
// colouring gives exactly this on a box whose periodic extents are even):
//   colour group C starts at row base[C]; slot s of the group is the cell
//   (i, j, k) with q = s / H, m = s % H, j = q % ny, k = q / ny, i = 2m + ((j + k + C) & 1),
//   H = ceil(nx / 2); a slot with i >= nx (odd nx) is a padding row.
// Inside a colour the cells keep natural order, so for even nx this is the colour-major layout of
// the general plan.
#pragma once

#include <cstdint>

namespace vlm {

struct Chunk;

// Shape of a box mesh as its face arrays define it.
struct BoxShape {
    int n[3] = {0, 0, 0};
    int per[3] = {0, 0, 0};  // 1: periodic (cyclic faces) in that direction
};

// Whether (own, nei) are exactly the internal faces of a generateBox mesh, and of which shape.
// Requires nx, ny >= 2 and at least 3 cells along every periodic direction (with 2, the cyclic and
// the internal face would join the same pair of cells).
bool detectBox(int nCells, int nInternal, const int32_t* own, const int32_t* nei, BoxShape* out);

// Whether the level-0 colouring of a box (greedy natural order: `colour`, `nColours` colours) is the
// red-black parity colouring the box layout assumes; periodic extents must also be even, so every
// face joins cells of opposite parity.
bool boxParityColouring(const BoxShape& S, const int* colour, int nColours);

// Division of a non-negative 31-bit n by a fixed d >= 1 as a multiply and a shift (Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994, Theorem 4.2 with N = 31):
// l = ceil(log2 d), m = ceil(2^(31+l) / d) < 2^32, n / d = umulhi(n, m) >> (l - 1); d = 1 has
// shift -1 (the quotient is n).
struct FastDiv {
    uint32_t m;
    int32_t shift;
};
FastDiv makeFastDiv(uint32_t d);

// Level-0 descriptor of one box system, as the row kernels read it (48 bytes, three int4 loads).
struct BoxSys {
    int nx, ny, nz, H;  // H = slots per x-row of one colour
    int per;            // bit d: periodic in direction d
    int base0, base1;   // first solver row of colour group 0 and 1
    int slots;          // H * ny * nz
    FastDiv divH, divNy;
};

// Rows of one launch: a chunk list (any batch; CTA b takes chunk b, whose system gives the
// descriptor, and skips systems that are done), or - a batch of one system - a row range taken by
// arithmetic with the descriptor passed by value, so the first loads of a thread are its data.  The
// range form skips the state check: the loop stops once its one system is done, and a V-cycle that
// still runs in that last pass (after a breakdown found earlier in the pass) only rewrites the
// preconditioner's scratch vectors, which nothing reads afterwards.
// Counters of the fused two-colour level-0 sweep: piece tickets, finished CTAs, launch epoch, and an
// error word for a wait that gave up.
struct SweepSync {
    unsigned ticket, finished, epoch, err;
};

struct BoxRows {
    const Chunk* ch;  // null: the range form
    const BoxSys* boxes;
    BoxSys one;
    int begin, end;
};

}  // namespace vlm
