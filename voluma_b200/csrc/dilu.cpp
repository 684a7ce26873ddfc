// Host construction of the DIC/DILU level schedule (see dilu.h).
#include "dilu.h"

#include <algorithm>
#include <array>
#include <stdexcept>

namespace vlm {

DiluPlan buildDiluPlan(const std::vector<SysTopo>& systems, const BatchPlan& P) {
    const LevelPlan& L0 = P.levels[0];
    const int nrows = L0.nrows;
    DiluPlan D;
    // user cell -> level-0 row
    std::vector<int32_t> rowOf(static_cast<size_t>(P.userCells), -1);
    for (int r = 0; r < nrows; ++r)
        if (P.perm0[r] >= 0) rowOf[P.perm0[r]] = r;
    std::vector<std::vector<std::array<int32_t, 3>>> lo(static_cast<size_t>(nrows)), up(static_cast<size_t>(nrows));
    D.levPtr.push_back(0);
    for (int b = 0; b < P.nsys; ++b) {
        const int s = P.order[b];
        const SysTopo& T = systems[s];
        const int64_t cb = P.userCellBase[s], fb = P.userFaceBase[s];
        // faces whose two cells are distinct cells of this system (LinearSolver.cpp:34-42)
        std::vector<std::array<int32_t, 3>> faces;  // (u, l, f)
        faces.reserve(size_t(T.nInternal));
        for (int f = 0; f < T.nInternal; ++f) {
            const int o = T.own[f], n = T.nei[f];
            if (o >= T.nCells || n >= T.nCells || o == n) continue;
            faces.push_back({std::max(o, n), std::min(o, n), f});
        }
        std::sort(faces.begin(), faces.end());
        for (const auto& t : faces) {
            const int u = t[0], l = t[1], f = t[2];
            const int32_t flag = T.own[f] == l ? int32_t(1u << 31) : 0;
            const int32_t face = int32_t(fb + f) | flag;
            const int32_t ru = rowOf[cb + u], rl = rowOf[cb + l];
            lo[ru].push_back({ru, rl, face});  // appended in ascending (l, f) for this u
            up[rl].push_back({rl, ru, face});  // ascending (u, f) for this l: reversed below
        }
        // levels in natural order
        std::vector<int32_t> level(static_cast<size_t>(T.nCells), 0);
        int nLev = 1;
        for (int c = 0; c < T.nCells; ++c) {
            int lv = 0;
            for (const auto& e : lo[rowOf[cb + c]]) {
                // e[1] is a solver row; its natural cell is perm0 - cb
                lv = std::max(lv, level[P.perm0[e[1]] - cb] + 1);
            }
            level[c] = lv;
            nLev = std::max(nLev, lv + 1);
        }
        std::vector<std::vector<int32_t>> byLevel(static_cast<size_t>(nLev));
        for (int c = 0; c < T.nCells; ++c) byLevel[level[c]].push_back(rowOf[cb + c]);
        // padding rows of this system: level 0 (no neighbours, diag 1, r 0)
        for (int r = L0.sysRow[b]; r < L0.sysRow[b + 1]; ++r)
            if (P.perm0[r] < 0) byLevel[0].push_back(r);
        DiluSys ds;
        ds.sys = b;
        ds.levBegin = int(D.levPtr.size()) - 1;
        ds.nLev = nLev;
        ds.rowBegin = L0.sysRow[b];
        ds.rowCount = L0.sysRow[b + 1] - L0.sysRow[b];
        ds.slotBegin = int(D.levRows.size());
        ds.loBegin = int(D.sLoCol.size());
        ds.upBegin = int(D.sUpCol.size());
        D.maxRows = std::max(D.maxRows, ds.rowCount);
        for (auto& v : byLevel) {
            std::sort(v.begin(), v.end());
            const int width = int(v.size());
            D.maxWidth = std::max(D.maxWidth, width);
            DiluLevel lv;
            lv.s0 = int(D.levRows.size());
            lv.width = width;
            lv.mlo = lv.mup = 0;
            for (int r : v) {
                lv.mlo = std::max(lv.mlo, int(lo[r].size()));
                lv.mup = std::max(lv.mup, int(up[r].size()));
                D.slotRow.push_back(r - ds.rowBegin);
            }
            D.maxEnt = std::max({D.maxEnt, lv.mlo, lv.mup});
            lv.lo = int(D.sLoCol.size());
            for (int j = 0; j < lv.mlo; ++j)
                for (int r : v) {
                    const bool has = j < int(lo[r].size());
                    D.sLoCol.push_back(has ? lo[r][j][1] - ds.rowBegin : -1);
                    D.sLoFace.push_back(has ? lo[r][j][2] : 0);
                }
            lv.up = int(D.sUpCol.size());
            for (int j = 0; j < lv.mup; ++j)
                for (int r : v) {
                    const int nu = int(up[r].size());
                    const bool has = j < nu;  // backward order: descending (u, f)
                    D.sUpCol.push_back(has ? up[r][nu - 1 - j][1] - ds.rowBegin : -1);
                    D.sUpFace.push_back(has ? up[r][nu - 1 - j][2] : 0);
                }
            D.lev.push_back(lv);
            D.levRows.insert(D.levRows.end(), v.begin(), v.end());
            D.levPtr.push_back(int32_t(D.levRows.size()));
        }
        ds.slotEnd = int(D.levRows.size());
        ds.loEnd = int(D.sLoCol.size());
        ds.upEnd = int(D.sUpCol.size());
        D.maxLevels = std::max(D.maxLevels, nLev);
        D.sys.push_back(ds);
    }
    D.loPtr.assign(size_t(nrows) + 1, 0);
    D.upPtr.assign(size_t(nrows) + 1, 0);
    for (int r = 0; r < nrows; ++r) {
        D.loPtr[r + 1] = D.loPtr[r] + int32_t(lo[r].size());
        D.upPtr[r + 1] = D.upPtr[r] + int32_t(up[r].size());
        for (const auto& e : lo[r]) {
            D.loCol.push_back(e[1]);
            D.loFace.push_back(e[2]);
        }
        for (auto it = up[r].rbegin(); it != up[r].rend(); ++it) {
            D.upCol.push_back((*it)[1]);
            D.upFace.push_back((*it)[2]);
        }
    }
    return D;
}

}  // namespace vlm
