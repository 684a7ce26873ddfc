// Builds the device layout plan of a batch (see plan.h).  Host-only, once per mesh set.
#include "plan.h"

#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <thread>

namespace vlm {

namespace {

// Greedy colouring of rows [s0, s1) considering only edges inside the block.
std::vector<int> blockColour(const HLevel& L, int s0, int s1, int* nColours) {
    std::vector<int> colour(size_t(s1 - s0), -1);
    std::vector<int> mark;
    int nc = 0;
    for (int i = s0; i < s1; ++i) {
        for (int k = L.off[i]; k < L.off[i + 1]; ++k) {
            const int j = L.adjCell[k];
            if (j < s0 || j >= s1) continue;
            const int c = colour[j - s0];
            if (c >= 0) {
                if (size_t(c) >= mark.size()) mark.resize(size_t(c) + 1, -1);
                mark[c] = i;
            }
        }
        int c = 0;
        while (size_t(c) < mark.size() && mark[c] == i) ++c;
        colour[i - s0] = c;
        nc = std::max(nc, c + 1);
    }
    *nColours = nc;
    return colour;
}

void appendChunks(std::vector<Chunk>& out, int start, int len, int sys, int* slot, int width = kRowsPerCta) {
    for (int s = 0; s < len; s += width) {
        Chunk c;
        c.start = start + s;
        c.count = std::min(width, len - s);
        c.sys = sys;
        c.slot = slot ? (*slot)++ : 0;
        out.push_back(c);
    }
}

}  // namespace

BatchPlan buildPlan(const std::vector<SysTopo>& systems, int mergeLevels, bool useBox,
                    const std::function<Hierarchy(const SysTopo&)>& hierarchy) {
    BatchPlan P;
    const int ns = int(systems.size());
    if (ns == 0) throw std::invalid_argument("empty batch");
    P.nsys = ns;
    P.userCellBase.resize(ns);
    P.userFaceBase.resize(ns);
    for (int s = 0; s < ns; ++s) {
        P.userCellBase[s] = P.userCells;
        P.userFaceBase[s] = P.userFaces;
        P.userCells += systems[s].nCells;
        P.userFaces += systems[s].nInternal;
    }
    if (P.userCells >= (int64_t(1) << 31) - 1 || P.userFaces >= (int64_t(1) << 31) - 1)
        throw std::invalid_argument("batch exceeds 2^31 cells/faces");

    std::vector<Hierarchy> Hin(ns);
    for (int s = 0; s < ns; ++s)
        if (systems[s].nCells <= 0) throw std::invalid_argument("system with no cells");
    if (hierarchy) {
        for (int s = 0; s < ns; ++s) Hin[s] = hierarchy(systems[s]);
    } else {
    // the systems' hierarchies are independent: built by a pool of host threads, each taking the
    // next system (largest first keeps the pool busy to the end)
        std::vector<int> byCells(ns);
        std::iota(byCells.begin(), byCells.end(), 0);
        std::stable_sort(byCells.begin(), byCells.end(),
                         [&](int a, int b) { return systems[a].nCells > systems[b].nCells; });
        std::atomic<int> next{0};
        std::exception_ptr err;
        std::mutex errMutex;
        auto work = [&] {
            for (int q = next++; q < ns; q = next++) {
                const SysTopo& t = systems[byCells[q]];
                try {
                    Hin[byCells[q]] = buildHierarchy(t.nCells, t.nInternal, t.own, t.nei, t.magSf, t.ndc, mergeLevels);
                } catch (...) {
                    std::lock_guard<std::mutex> lock(errMutex);
                    if (!err) err = std::current_exception();
                }
            }
        };
        const int nt = std::max(1, std::min(ns, int(std::min(32u, std::max(1u, std::thread::hardware_concurrency())))));
        std::vector<std::thread> pool;
        for (int k = 1; k < nt; ++k) pool.emplace_back(work);
        work();
        for (auto& t : pool) t.join();
        if (err) std::rethrow_exception(err);
    }
    P.order.resize(ns);
    std::iota(P.order.begin(), P.order.end(), 0);
    std::stable_sort(P.order.begin(), P.order.end(),
                     [&](int a, int b) { return Hin[a].levels.size() > Hin[b].levels.size(); });
    P.H.resize(ns);
    P.nLevels.resize(ns);
    P.sysCells.resize(ns);
    for (int b = 0; b < ns; ++b) {
        P.H[b] = std::move(Hin[P.order[b]]);
        P.nLevels[b] = int(P.H[b].levels.size());
        P.sysCells[b] = P.H[b].levels[0].n;
    }
    const int Lmax = P.nLevels[0];
    P.levels.resize(Lmax);

    // ---------------------------------------------------------------- box level 0
    // Every system a box mesh with even periodic extents that smooths on level 0 (a one-level system
    // solves level 0 directly, in natural row order), and its natural-order colouring the parity
    // colouring: level 0 takes the box layout (box.h).
    std::vector<BoxShape> shapes(ns);
    bool boxMode = useBox;
    for (int b = 0; b < ns && boxMode; ++b) {
        const SysTopo& T = systems[P.order[b]];
        BoxShape& S = shapes[b];
        if (!detectBox(T.nCells, T.nInternal, T.own, T.nei, &S)) {
            boxMode = false;
            break;
        }
        for (int d = 0; d < 3; ++d)
            if (S.per[d] && S.n[d] % 2 != 0) boxMode = false;
        if (P.nLevels[b] <= 1) boxMode = false;
        if (!boxMode) continue;
        int nc = 0;
        const std::vector<int> colour = greedyColour(P.H[b].levels[0], &nc);
        boxMode = boxParityColouring(S, colour.data(), nc);
    }

    // ---------------------------------------------------------------- row layout per level
    // rowOf[k][b][natural] -> solver row
    std::vector<std::vector<std::vector<int32_t>>> rowOf(Lmax, std::vector<std::vector<int32_t>>(ns));
    std::vector<std::vector<std::vector<std::pair<int, int>>>> groups(Lmax, std::vector<std::vector<std::pair<int, int>>>(ns));
    for (int k = 0; k < Lmax; ++k) {
        LevelPlan& LP = P.levels[k];
        int row = 0;
        int present = 0, active = 0;
        if (k > 0) {
            LP.blockGS = true;
        } else if (boxMode) {
            LP.box = true;
        } else {
            // level 0: global multicolour GS if every smoothing system needs few colours
            for (int b = 0; b < ns; ++b) {
                if (P.nLevels[b] <= 1) continue;
                int nc = 0;
                greedyColour(P.H[b].levels[0], &nc);
                if (nc > kMaxGlobalColours) LP.blockGS = true;
            }
        }
        for (int b = 0; b < ns; ++b) {
            if (P.nLevels[b] > k) present = b + 1;
            if (P.nLevels[b] - 1 > k) active = b + 1;
        }
        LP.sysRow.assign(size_t(present) + 1, 0);
        LP.sysFace.assign(size_t(present) + 1, 0);
        int64_t faceCount = 0;
        for (int b = 0; b < present; ++b) {
            const HLevel& L = P.H[b].levels[k];
            LP.sysRow[b] = row;
            LP.sysFace[b] = k == 0 ? int32_t(P.userFaceBase[P.order[b]]) : int32_t(faceCount);
            faceCount += int64_t(L.l.size());
            auto& ro = rowOf[k][b];
            ro.assign(size_t(L.n), -1);
            auto place = [&](int i) {
                ro[i] = row;
                LP.natural.push_back(i);
                LP.rowSys.push_back(b);
                ++row;
            };
            auto pad = [&]() {
                while (row % kSlice) {
                    LP.natural.push_back(-1);
                    LP.rowSys.push_back(-1);
                    ++row;
                }
            };
            if (LP.box) {
                // colour groups in slot order (box.h); slots past the x-row's end are padding
                const BoxShape& S = shapes[b];
                const int nx = S.n[0], ny = S.n[1], nz = S.n[2], H = (nx + 1) / 2;
                BoxSys bs;
                bs.nx = nx;
                bs.ny = ny;
                bs.nz = nz;
                bs.H = H;
                bs.per = S.per[0] | S.per[1] << 1 | S.per[2] << 2;
                bs.slots = H * ny * nz;
                bs.divH = makeFastDiv(uint32_t(H));
                bs.divNy = makeFastDiv(uint32_t(ny));
                for (int C = 0; C < 2; ++C) {
                    const int g0 = row;
                    (C == 0 ? bs.base0 : bs.base1) = row;
                    for (int q = 0; q < ny * nz; ++q) {
                        const int j = q % ny, kk = q / ny;
                        for (int m = 0; m < H; ++m) {
                            const int i = 2 * m + ((j + kk + C) & 1);
                            if (i < nx) {
                                place(i + nx * q);
                            } else {
                                LP.natural.push_back(-1);
                                LP.rowSys.push_back(-1);
                                ++row;
                            }
                        }
                    }
                    pad();
                    if (b < active) groups[k][b].push_back({g0, row - g0});
                }
                if (b < active) LP.maxColours = std::max(LP.maxColours, 2);
                LP.boxes.push_back(bs);
            } else if (b < active && !LP.blockGS) {
                int nc = 0;
                const std::vector<int> colour = greedyColour(L, &nc);
                LP.maxColours = std::max(LP.maxColours, nc);
                std::vector<std::vector<int>> byColour(static_cast<size_t>(nc));
                for (int i = 0; i < L.n; ++i) byColour[colour[i]].push_back(i);
                for (int c = 0; c < nc; ++c) {
                    const int g0 = row;
                    for (int i : byColour[c]) place(i);
                    pad();
                    groups[k][b].push_back({g0, row - g0});
                }
            } else if (b < active) {
                // blocks of consecutive natural rows, each ordered by its block-local colouring
                for (int s0 = 0; s0 < L.n; s0 += kBlockRows) {
                    const int s1 = std::min(L.n, s0 + kBlockRows);
                    int nc = 0;
                    const std::vector<int> colour = blockColour(L, s0, s1, &nc);
                    LP.maxColours = std::max(LP.maxColours, nc);
                    Chunk blk;
                    blk.start = row;
                    blk.count = s1 - s0;
                    blk.sys = b;
                    blk.slot = nc;
                    // inside a colour the rows are independent (block Gauss-Seidel and Jacobi update
                    // each from other colours' or the previous iterate's values), so they are
                    // ordered by decreasing row length: SELL slices of rows of equal length pad
                    // less (1.28x -> 1.11x the entries on the coarse levels at 128^3)
                    std::vector<int> grp;
                    for (int c = 0; c < nc; ++c) {
                        grp.clear();
                        for (int i = s0; i < s1; ++i)
                            if (colour[i - s0] == c) grp.push_back(i);
                        std::stable_sort(grp.begin(), grp.end(), [&L](int a, int b2) {
                            return L.off[a + 1] - L.off[a] > L.off[b2 + 1] - L.off[b2];
                        });
                        for (int i : grp) {
                            place(i);
                            LP.rowColour.push_back(int8_t(c));
                        }
                    }
                    LP.blocks.push_back(blk);
                }
                const int before = row;
                pad();
                LP.rowColour.resize(LP.rowColour.size() + size_t(row - before), int8_t(-1));
            } else {
                for (int i = 0; i < L.n; ++i) place(i);
                const int before = row;
                pad();
                if (LP.blockGS) LP.rowColour.resize(LP.rowColour.size() + size_t(row - before + L.n), int8_t(-1));
            }
        }
        LP.sysRow[present] = row;
        LP.sysFace[present] = k == 0 ? int32_t(P.userFaces) : int32_t(faceCount);
        LP.nrows = row;
        LP.nfaces = k == 0 ? int(P.userFaces) : int(faceCount);
        LP.nActiveRows = LP.sysRow[active];
        LP.sysRow.resize(size_t(present) + 1);
        // chunks
        int slot = 0;
        for (int b = 0; b < present; ++b) {
            const int s0 = LP.sysRow[b], len = LP.sysRow[b + 1] - LP.sysRow[b];
            if (k == 0) P.sysSlotBegin.push_back(slot);
            appendChunks(LP.all, s0, len, b, &slot, k == 0 ? kWideRows : kRowsPerCta);
            if (k == 0) P.sysSlotEnd.push_back(slot);
            if (b < active) appendChunks(LP.active, s0, len, b, nullptr);
        }
        if (k == 0) P.nSlots = slot;
        int nSteps = 0;
        for (int b = 0; b < active; ++b) nSteps = std::max(nSteps, int(groups[k][b].size()));
        LP.nSteps = nSteps;
        LP.fwd.assign(size_t(nSteps), {});
        LP.rev.assign(size_t(nSteps), {});
        for (int t = 0; t < nSteps; ++t)
            for (int b = 0; b < active; ++b) {
                const auto& g = groups[k][b];
                const int nc = int(g.size());
                if (t < nc) {
                    appendChunks(LP.fwd[t], g[t].first, g[t].second, b, nullptr);
                    appendChunks(LP.rev[t], g[nc - 1 - t].first, g[nc - 1 - t].second, b, nullptr);
                }
            }
    }

    // ---------------------------------------------------------------- box face map
    if (P.levels[0].box) {
        LevelPlan& LP = P.levels[0];
        const size_t nr = size_t(LP.nrows);
        LP.boxFace.assign(3 * nr, -1);
        for (int b = 0; b < int(LP.sysRow.size()) - 1; ++b) {
            const SysTopo& T = systems[P.order[b]];
            const BoxShape& S = shapes[b];
            const int nx = S.n[0], nxny = S.n[0] * S.n[1];
            for (int f = 0; f < T.nInternal; ++f) {
                const int o = T.own[f], n = T.nei[f];
                const int io = o % nx, jo = (o / nx) % S.n[1], ko = o / nxny;
                const int in = n % nx, jn = (n / nx) % S.n[1], kn = n / nxny;
                int d, minus;
                if (jo == jn && ko == kn) {
                    d = 0;
                    minus = in == io + 1 ? o : n;  // cyclic: the max-side cell is the minus side
                } else if (io == in && ko == kn) {
                    d = 1;
                    minus = jn == jo + 1 ? o : n;
                } else {
                    d = 2;
                    minus = kn == ko + 1 ? o : n;
                }
                LP.boxFace[size_t(d) * nr + size_t(rowOf[0][b][minus])] = LP.sysFace[b] + f;
            }
        }
    }

    // ---------------------------------------------------------------- SELL-32 structure
    for (int k = 0; k < Lmax; ++k) {
        LevelPlan& LP = P.levels[k];
        const int nsl = LP.nrows / kSlice;
        LP.rlen.assign(size_t(LP.nrows), 0);
        LP.slPtr.assign(size_t(nsl) + 1, 0);
        for (int r = 0; r < LP.nrows; ++r) {
            const int b = LP.rowSys[r];
            if (b < 0) continue;
            const HLevel& L = P.H[b].levels[k];
            const int i = LP.natural[r];
            LP.rlen[r] = L.off[i + 1] - L.off[i];
        }
        for (int s = 0; s < nsl; ++s) {
            int w = 0;
            for (int q = 0; q < kSlice; ++q) w = std::max(w, LP.rlen[s * kSlice + q]);
            LP.slPtr[s + 1] = LP.slPtr[s] + w * kSlice;
        }
        LP.col.assign(size_t(LP.slPtr[nsl]), 0);
        LP.src.assign(size_t(LP.slPtr[nsl]), 0);
        for (int r = 0; r < LP.nrows; ++r) {
            const int b = LP.rowSys[r];
            if (b < 0) {
                continue;
            }
            const HLevel& L = P.H[b].levels[k];
            const int i = LP.natural[r];
            const int base = LP.slPtr[r / kSlice] + (r % kSlice);
            const int32_t fb = LP.sysFace[b];
            const SysTopo& T = systems[P.order[b]];
            for (int e = L.off[i]; e < L.off[i + 1]; ++e) {
                const int q = e - L.off[i];
                const int f = L.adjFace[e];
                LP.col[size_t(base) + size_t(q) * kSlice] = rowOf[k][b][L.adjCell[e]];
                bool useUpper;
                if (k == 0)
                    useUpper = T.own[f] == i;  // user arrays are owner-oriented
                else
                    useUpper = L.adjIsL[e] != 0;
                const int32_t g = fb + f;
                LP.src[size_t(base) + size_t(q) * kSlice] = useUpper ? g : ~g;
            }
        }
        // padding rows point at themselves (never read: rlen = 0)
    }

    // ---------------------------------------------------------------- transfer maps
    for (int k = 0; k + 1 < Lmax; ++k) {
        LevelPlan& LP = P.levels[k];
        const LevelPlan& NP = P.levels[k + 1];
        LP.agg.assign(size_t(LP.nrows), -1);
        LP.childPtr.assign(size_t(NP.nrows) + 1, 0);
        LP.intraPtr.assign(size_t(NP.nrows) + 1, 0);
        LP.cfacePtr.assign(size_t(NP.nfaces) + 1, 0);
        const int activeSys = int(NP.sysRow.size()) - 1;  // systems present on k+1 = active on k
        // CSR lists by counting sort: a counting pass, prefix sums, then a filling pass in the same
        // order (systems, cells / faces ascending), so each list keeps that order
        for (int pass = 0; pass < 2; ++pass) {
            std::vector<int32_t> ck, ci, cc;  // fill cursors
            if (pass == 1) {
                for (int R = 0; R < NP.nrows; ++R) {
                    LP.childPtr[R + 1] += LP.childPtr[R];
                    LP.intraPtr[R + 1] += LP.intraPtr[R];
                }
                for (int c = 0; c < NP.nfaces; ++c) LP.cfacePtr[c + 1] += LP.cfacePtr[c];
                LP.child.resize(size_t(LP.childPtr[NP.nrows]));
                LP.intraFace.resize(size_t(LP.intraPtr[NP.nrows]));
                LP.cfaceSrc.resize(size_t(LP.cfacePtr[NP.nfaces]));
                ck.assign(LP.childPtr.begin(), LP.childPtr.end() - 1);
                ci.assign(LP.intraPtr.begin(), LP.intraPtr.end() - 1);
                cc.assign(LP.cfacePtr.begin(), LP.cfacePtr.end() - 1);
            }
            for (int b = 0; b < activeSys; ++b) {
                const HLevel& L = P.H[b].levels[k];
                const int32_t fb = LP.sysFace[b], nfb = NP.sysFace[b];
                const std::vector<int32_t>& rk = rowOf[k][b];
                const std::vector<int32_t>& rk1 = rowOf[k + 1][b];
                for (int i = 0; i < L.n; ++i) {
                    const int R = rk1[L.agg[i]];
                    if (pass == 0) {
                        LP.agg[rk[i]] = R;
                        ++LP.childPtr[R + 1];
                    } else {
                        LP.child[size_t(ck[R]++)] = rk[i];
                    }
                }
                const bool lev0 = k == 0;
                for (size_t f = 0; f < L.l.size(); ++f) {
                    const int c = L.faceMap[f];
                    const int32_t g = fb + int32_t(f);
                    if (c < 0) {
                        const int R = rk1[L.agg[L.l[f]]];
                        if (pass == 0)
                            ++LP.intraPtr[R + 1];
                        else
                            LP.intraFace[size_t(ci[R]++)] = g;
                    } else {
                        const size_t C = size_t(nfb + c);
                        if (pass == 0) {
                            ++LP.cfacePtr[C + 1];
                        } else {
                            bool flip = L.faceFlip[f] != 0;
                            if (lev0 && !P.H[b].ownerIsL[f]) flip = !flip;
                            LP.cfaceSrc[size_t(cc[C]++)] = int32_t(uint32_t(g) | (flip ? 0x80000000u : 0u));
                        }
                    }
                }
            }
        }
    }

    // ---------------------------------------------------------------- coarse solves, level-0 map
    P.coarse.resize(ns);
    int inv = 0;
    for (int b = 0; b < ns; ++b) {
        const int Lc = P.nLevels[b] - 1;
        CoarsePlan c;
        c.level = Lc;
        c.rowStart = P.levels[Lc].sysRow[b];
        c.n = P.H[b].levels[Lc].n;
        c.invOffset = inv;
        c.sys = b;
        inv += c.n * c.n;
        P.coarse[b] = c;
    }
    P.invTotal = inv;
    const LevelPlan& L0 = P.levels[0];
    P.perm0.assign(size_t(L0.nrows), -1);
    for (int r = 0; r < L0.nrows; ++r)
        if (L0.rowSys[r] >= 0)
            P.perm0[r] = int32_t(P.userCellBase[P.order[L0.rowSys[r]]] + L0.natural[r]);
    return P;
}

}  // namespace vlm
