// Box-mesh detection from the face arrays (host, once per mesh).
#include "box.h"

#include <vector>

namespace vlm {

namespace {

// Appends the internal faces a box of shape S has, in generateBox order: raw internal faces in
// owner order (+x, +y, +z per cell), then the cyclic pairs x, y, z (xMin patch: k outer, j inner;
// yMin: k outer, i inner; zMin: j outer, i inner), owner on the min side.  Compares on the fly.
bool matches(const BoxShape& S, int nInternal, const int32_t* own, const int32_t* nei) {
    const int nx = S.n[0], ny = S.n[1], nz = S.n[2];
    int64_t f = 0;
    auto take = [&](int o, int n) {
        if (f >= nInternal || own[f] != o || nei[f] != n) return false;
        ++f;
        return true;
    };
    for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const int c = i + nx * (j + ny * k);
                if (i + 1 < nx && !take(c, c + 1)) return false;
                if (j + 1 < ny && !take(c, c + nx)) return false;
                if (k + 1 < nz && !take(c, c + nx * ny)) return false;
            }
    if (S.per[0])
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j) {
                const int c = nx * (j + ny * k);
                if (!take(c, c + nx - 1)) return false;
            }
    if (S.per[1])
        for (int k = 0; k < nz; ++k)
            for (int i = 0; i < nx; ++i) {
                const int c = i + nx * ny * k;
                if (!take(c, c + nx * (ny - 1))) return false;
            }
    if (S.per[2])
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const int c = i + nx * j;
                if (!take(c, c + nx * ny * (nz - 1))) return false;
            }
    return f == nInternal;
}

}  // namespace

bool detectBox(int nCells, int nInternal, const int32_t* own, const int32_t* nei, BoxShape* out) {
    // cell 0 owns the first faces: +x (neighbour 1), +y (neighbour nx), and +z (neighbour nx*ny)
    // when the box is more than one cell thick
    if (nCells < 4 || nInternal < 3) return false;
    if (own[0] != 0 || nei[0] != 1 || own[1] != 0) return false;
    const int64_t nx = nei[1];
    if (nx < 2 || nCells % nx != 0) return false;
    int64_t ny, nz;
    if (own[2] == 0) {
        const int64_t nxny = nei[2];
        if (nxny % nx != 0) return false;
        ny = nxny / nx;
        if (ny < 2 || nCells % nxny != 0) return false;
        nz = nCells / nxny;
    } else {
        ny = nCells / nx;
        nz = 1;
    }
    if (ny < 2 || nx * ny * nz != nCells) return false;
    const int64_t raw = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1);
    const int64_t cyc[3] = {ny * nz, nx * nz, nx * ny};
    const int64_t n[3] = {nx, ny, nz};
    for (int mask = 0; mask < 8; ++mask) {
        int64_t cnt = raw;
        bool ok = true;
        for (int d = 0; d < 3; ++d)
            if (mask >> d & 1) {
                cnt += cyc[d];
                if (n[d] < 3) ok = false;
            }
        if (!ok || cnt != nInternal) continue;
        BoxShape S;
        for (int d = 0; d < 3; ++d) {
            S.n[d] = int(n[d]);
            S.per[d] = mask >> d & 1;
        }
        if (matches(S, nInternal, own, nei)) {
            *out = S;
            return true;
        }
    }
    return false;
}

FastDiv makeFastDiv(uint32_t d) {
    if (d <= 1) return FastDiv{0u, -1};
    int l = 0;
    while ((uint64_t(1) << l) < d) ++l;
    const uint64_t num = uint64_t(1) << (31 + l);
    return FastDiv{uint32_t((num + d - 1) / d), l - 1};
}

bool boxParityColouring(const BoxShape& S, const int* colour, int nColours) {
    for (int d = 0; d < 3; ++d)
        if (S.per[d] && S.n[d] % 2 != 0) return false;
    if (nColours != 2) return false;
    const int nx = S.n[0], ny = S.n[1], nz = S.n[2];
    for (int k = 0, c = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i, ++c)
                if (colour[c] != ((i + j + k) & 1)) return false;
    return true;
}

}  // namespace vlm
