// Images of the shared-memory coarse tail: per system, the Jacobi levels first..coarsest-1 as ELL
// rows (values gathered per solve through `codes`, structure with 16-bit local indices), then the
// vectors of every level; offsets as TailImg describes them.
#include "tailplan.h"

#include <algorithm>
#include <cstring>

namespace vlm {

bool buildTailImages(const BatchPlan& plan, const std::vector<TailSys>& ts, size_t budget, TailImages& out) {
    std::vector<TailImg>& imgs = out.imgs;
    std::vector<int32_t>& codes = out.codes;
    std::vector<uint16_t>& str = out.str;
    imgs.assign(ts.size(), TailImg{});
    codes.clear();
    str.clear();
    size_t max64 = 0, max32 = 0;
    for (size_t b = 0; b < ts.size(); ++b) {
        const TailSys& s = ts[b];
        const int f = s.first, c = s.coarsest;
        if (f < 1 || c >= kTailMaxLevels || c > 31) return false;
        TailImg& I = imgs[b];
        std::memset(&I, 0, sizeof I);
        I.sys = s.sys;
        I.first = f;
        I.coarsest = c;
        I.nc = s.coarseN;
        I.invOffset = s.invOffset;
        for (int k = f; k <= c; ++k) {
            I.n[k] = s.rowCount[k];
            I.rowStart[k] = s.rowStart[k];
            if (I.n[k] >= 0xffff) return false;
        }
        if (I.nc > I.n[c]) return false;
        // value image: per Jacobi level the diagonal, then the ELL values (entry q of row i at q n + i)
        I.valOff = int(codes.size());
        int tc = 0;
        for (int k = f; k < c; ++k) {
            const LevelPlan& P = plan.levels[k];
            const int n = I.n[k], rs = I.rowStart[k];
            if (P.col.empty() || P.rlen.size() < size_t(rs + n)) return false;  // host structure released
            int W = 0;
            for (int i = 0; i < n; ++i) W = std::max(W, P.rlen[size_t(rs + i)]);
            I.W[k] = W;
            I.tDiag[k] = tc;
            for (int i = 0; i < n; ++i) codes.push_back((k << 26) | (1 << 25) | (rs + i));
            tc += n;
            I.tVal[k] = tc;
            for (int q = 0; q < W; ++q)
                for (int i = 0; i < n; ++i) {
                    const int row = rs + i;
                    if (q < P.rlen[size_t(row)]) {
                        const int e = P.slPtr[size_t(row / kSlice)] + kSlice * q + row % kSlice;
                        if (e >= (1 << 25)) return false;
                        codes.push_back((k << 26) | e);
                    } else {
                        codes.push_back(-1);
                    }
                }
            tc += W * n;
        }
        while (tc % 4) {  // whole 16-byte words in both precisions
            codes.push_back(-1);
            ++tc;
        }
        I.valCount = tc;
        for (int k = f; k <= c; ++k) {
            I.tR[k] = tc;
            tc += I.n[k];
            I.tX[k] = tc;
            tc += I.n[k];
            if (k < c) {
                I.tX2[k] = tc;
                tc += I.n[k];
            }
        }
        tc = (tc + 3) & ~3;
        I.tCount = tc;
        // structure image: row lengths, local columns, aggregates, children of the next level
        I.strOff = int(str.size());
        int su = 0;
        auto push = [&](int v) {
            str.push_back(uint16_t(v));
            ++su;
        };
        for (int k = f; k < c; ++k) {
            const LevelPlan& P = plan.levels[k];
            const int n = I.n[k], rs = I.rowStart[k], n1 = I.n[k + 1], rs1 = I.rowStart[k + 1];
            I.uRlen[k] = su;
            for (int i = 0; i < n; ++i) push(P.rlen[size_t(rs + i)]);
            I.uCol[k] = su;
            for (int q = 0; q < I.W[k]; ++q)
                for (int i = 0; i < n; ++i) {
                    const int row = rs + i;
                    int cl = 0;
                    if (q < P.rlen[size_t(row)]) {
                        cl = P.col[size_t(P.slPtr[size_t(row / kSlice)] + kSlice * q + row % kSlice)] - rs;
                        if (cl < 0 || cl >= n) return false;
                    }
                    push(cl);
                }
            I.uAgg[k] = su;
            for (int i = 0; i < n; ++i) {
                const int a = P.agg[size_t(rs + i)];
                if (a >= 0 && (a - rs1 < 0 || a - rs1 >= n1)) return false;
                push(a < 0 ? 0xffff : a - rs1);
            }
            const int c0 = P.childPtr[size_t(rs1)];
            I.uCptr[k] = su;
            for (int R = 0; R <= n1; ++R) {
                const int v = P.childPtr[size_t(rs1 + R)] - c0;
                if (v >= 0xffff) return false;
                push(v);
            }
            I.uChild[k] = su;
            for (int q = c0; q < P.childPtr[size_t(rs1 + n1)]; ++q) {
                const int v = P.child[size_t(q)] - rs;
                if (v < 0 || v >= n) return false;
                push(v);
            }
        }
        while (su % 8) push(0);
        I.strCount = su;
        const size_t b64 = tail_smem_bytes(sizeof(double), I.tCount, I.nc, I.strCount);
        const size_t b32 = tail_smem_bytes(sizeof(float), I.tCount, I.nc, I.strCount);
        if (b64 > budget) return false;
        max64 = std::max(max64, b64);
        max32 = std::max(max32, b32);
    }
    if (imgs.empty()) return false;
    out.bytes64 = max64;
    out.bytes32 = max32;
    return true;
}

}  // namespace vlm
