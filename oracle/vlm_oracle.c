/* CPU restatement of the reference's LDU solve path — TEST INFRASTRUCTURE ONLY (the checker of
 * the CUDA path; never linked into the product).  See vlm_oracle.h.
 *
 * Compiled with -ffp-contract=off like the reference, and every loop keeps the reference's
 * operation order, so for the reference's own algorithms (natural-order Gauss-Seidel GAMG,
 * LU coarse solve, plain or exact sums) the results are bit-identical to the reference.
 */
#include "vlm_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define VSMALL 1.0e-300
#define GREAT 1.0e15
#define VO_BLOCK_ROWS 512       /* block size of the device's block-hybrid Gauss-Seidel */
#define VO_MAX_GLOBAL_COLOURS 4 /* level 0 keeps global multicolour GS up to this many colours */

/* ======================================================================= ExactSum */
#define NBINS 72
typedef struct {
    int64_t bins[NBINS];
    int64_t pending;
    int nonFinite;
    double nonFiniteValue;
} es_t;

static void es_clear(es_t* s) { memset(s, 0, sizeof(*s)); }

static void es_normalize(int64_t* b, int n) {
    for (int k = 0; k < n - 1; ++k) {
        const int64_t carry = b[k] >> 32;
        b[k] -= carry * ((int64_t)1 << 32);
        b[k + 1] += carry;
    }
}

/* Comm.h:65-93: v = ±M 2^(max(ex,1)-1075) split over three 32-bit bins */
static void es_add(es_t* s, double v) {
    uint64_t bits;
    memcpy(&bits, &v, sizeof bits);
    const int ex = (int)((bits >> 52) & 0x7ff);
    if (ex == 0x7ff) {
        s->nonFinite = 1;
        s->nonFiniteValue += v;
        return;
    }
    int64_t M = (int64_t)(bits & (((uint64_t)1 << 52) - 1));
    if (ex != 0) M |= (int64_t)1 << 52;
    if (M == 0) return;
    const int p = (ex == 0 ? 1 : ex) - 1;
    const int i = p >> 5, sh = p & 31;
    const int64_t sgn = -(int64_t)(bits >> 63);
    int64_t lo = (M & (((int64_t)1 << (32 - sh)) - 1)) << sh;
    const int64_t r = M >> (32 - sh);
    int64_t mid = r & 0xFFFFFFFF;
    int64_t hi = r >> 32;
    lo = (lo ^ sgn) - sgn;
    mid = (mid ^ sgn) - sgn;
    hi = (hi ^ sgn) - sgn;
    s->bins[i] += lo;
    s->bins[i + 1] += mid;
    s->bins[i + 2] += hi;
    if (++s->pending >= ((int64_t)1 << 29)) {
        es_normalize(s->bins, NBINS);
        s->pending = 0;
    }
}

/* Comm.cpp:135-164 binsToDouble / value */
static double es_value(const es_t* s) {
    if (s->nonFinite) return s->nonFiniteValue;
    int64_t b[NBINS];
    memcpy(b, s->bins, sizeof b);
    es_normalize(b, NBINS);
    double sign = 1.0;
    if (b[NBINS - 1] < 0) {
        sign = -1.0;
        for (int k = 0; k < NBINS; ++k) b[k] = -b[k];
        es_normalize(b, NBINS);
    }
    double r = 0.0;
    for (int k = NBINS - 1; k >= 0; --k)
        if (b[k] != 0) r += ldexp((double)b[k], 32 * k - 1074);
    return sign * r;
}

double vo_exact_sum(const double* v, long n) {
    es_t s;
    es_clear(&s);
    for (long i = 0; i < n; ++i) es_add(&s, v[i]);
    return es_value(&s);
}

/* SumAcc (Comm.h:96-116): exact or plain double accumulation */
typedef struct {
    int exact;
    es_t ex;
    double plain;
} sum_t;

static void sum_init(sum_t* s, int exact) {
    s->exact = exact;
    s->plain = 0.0;
    if (exact) es_clear(&s->ex);
}
static void sum_add(sum_t* s, double v) {
    if (s->exact)
        es_add(&s->ex, v);
    else
        s->plain += v;
}
static double sum_get(const sum_t* s) { return s->exact ? es_value(&s->ex) : s->plain; }

static double gSumProd(const double* a, const double* b, int n, int exact) {
    sum_t s;
    sum_init(&s, exact);
    for (int c = 0; c < n; ++c) sum_add(&s, a[c] * b[c]);
    return sum_get(&s);
}

static double gSumMag(const double* a, int n, int exact) {
    sum_t s;
    sum_init(&s, exact);
    for (int c = 0; c < n; ++c) sum_add(&s, fabs(a[c]));
    return sum_get(&s);
}

/* ======================================================================= amul */
void vo_amul(int n, int nf, const int* own, const int* nei, const double* diag, const double* upper,
             const double* lower, const double* x, double* y) {
    if (!lower) lower = upper;
    for (int c = 0; c < n; ++c) y[c] = diag[c] * x[c];
    for (int f = 0; f < nf; ++f) {
        y[own[f]] += upper[f] * x[nei[f]];
        y[nei[f]] += lower[f] * x[own[f]];
    }
}

/* ======================================================================= hierarchy */
typedef struct {
    int n, nf;
    int *l, *u;
    double* weight;
    int *off, *adjCell, *adjFace;
    signed char* adjIsL;
    int *agg, *faceMap; /* agg == NULL on the coarsest level */
    signed char* faceFlip;
} vo_level;

struct vo_hier {
    int nL;
    vo_level lev[40];
    signed char* ownerIsL;
};

static void level_free(vo_level* L) {
    free(L->l);
    free(L->u);
    free(L->weight);
    free(L->off);
    free(L->adjCell);
    free(L->adjFace);
    free(L->adjIsL);
    free(L->agg);
    free(L->faceMap);
    free(L->faceFlip);
    memset(L, 0, sizeof *L);
}

/* GAMG.cpp:15-37 */
static void build_adjacency(vo_level* L) {
    free(L->off);
    free(L->adjCell);
    free(L->adjFace);
    free(L->adjIsL);
    L->off = (int*)calloc((size_t)L->n + 1, sizeof(int));
    for (int f = 0; f < L->nf; ++f) {
        L->off[L->l[f] + 1]++;
        L->off[L->u[f] + 1]++;
    }
    for (int i = 0; i < L->n; ++i) L->off[i + 1] += L->off[i];
    const int nnz = L->off[L->n];
    L->adjCell = (int*)malloc(sizeof(int) * (size_t)(nnz ? nnz : 1));
    L->adjFace = (int*)malloc(sizeof(int) * (size_t)(nnz ? nnz : 1));
    L->adjIsL = (signed char*)malloc((size_t)(nnz ? nnz : 1));
    int* fill = (int*)malloc(sizeof(int) * (size_t)(L->n ? L->n : 1));
    for (int i = 0; i < L->n; ++i) fill[i] = L->off[i];
    for (int f = 0; f < L->nf; ++f) {
        int k = fill[L->l[f]]++;
        L->adjCell[k] = L->u[f];
        L->adjFace[k] = f;
        L->adjIsL[k] = 1;
        k = fill[L->u[f]]++;
        L->adjCell[k] = L->l[f];
        L->adjFace[k] = f;
        L->adjIsL[k] = 0;
    }
    free(fill);
}

/* open-addressing map (lo,hi) -> coarse face, first-occurrence numbering */
typedef struct {
    uint64_t* key;
    int* val;
    size_t cap;
} fmap_t;

static void fmap_init(fmap_t* m, size_t n) {
    size_t cap = 16;
    while (cap < 2 * n + 16) cap <<= 1;
    m->cap = cap;
    m->key = (uint64_t*)malloc(sizeof(uint64_t) * cap);
    m->val = (int*)malloc(sizeof(int) * cap);
    for (size_t i = 0; i < cap; ++i) m->key[i] = UINT64_MAX;
}
static void fmap_free(fmap_t* m) {
    free(m->key);
    free(m->val);
}
/* returns pointer to value slot; *found tells whether the key existed */
static int* fmap_get(fmap_t* m, uint64_t k, int* found) {
    size_t h = (size_t)((k * 0x9E3779B97F4A7C15ull) >> 17) & (m->cap - 1);
    while (m->key[h] != UINT64_MAX && m->key[h] != k) h = (h + 1) & (m->cap - 1);
    *found = m->key[h] == k;
    m->key[h] = k;
    return &m->val[h];
}

/* GAMG.cpp:40-94: one pairwise pass on L, returns the coarse topology */
static vo_level agglomerate(vo_level* L) {
    free(L->agg);
    L->agg = (int*)malloc(sizeof(int) * (size_t)(L->n ? L->n : 1));
    for (int i = 0; i < L->n; ++i) L->agg[i] = -1;
    int nc = 0;
    for (int i = 0; i < L->n; ++i) {
        if (L->agg[i] >= 0) continue;
        int best = -1;
        double bw = -1;
        for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
            const int j = L->adjCell[k];
            if (L->agg[j] < 0 && j != i && L->weight[L->adjFace[k]] > bw) {
                bw = L->weight[L->adjFace[k]];
                best = j;
            }
        }
        if (best >= 0) {
            L->agg[i] = L->agg[best] = nc++;
            continue;
        }
        for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
            if (L->weight[L->adjFace[k]] > bw) {
                bw = L->weight[L->adjFace[k]];
                best = L->adjCell[k];
            }
        }
        L->agg[i] = best >= 0 ? L->agg[best] : nc++;
    }
    vo_level C;
    memset(&C, 0, sizeof C);
    C.n = nc;
    free(L->faceMap);
    free(L->faceFlip);
    L->faceMap = (int*)malloc(sizeof(int) * (size_t)(L->nf ? L->nf : 1));
    L->faceFlip = (signed char*)calloc((size_t)(L->nf ? L->nf : 1), 1);
    C.l = (int*)malloc(sizeof(int) * (size_t)(L->nf ? L->nf : 1));
    C.u = (int*)malloc(sizeof(int) * (size_t)(L->nf ? L->nf : 1));
    C.weight = (double*)malloc(sizeof(double) * (size_t)(L->nf ? L->nf : 1));
    fmap_t fm;
    fmap_init(&fm, (size_t)L->nf);
    for (int f = 0; f < L->nf; ++f) {
        L->faceMap[f] = -1;
        const int a = L->agg[L->l[f]], b = L->agg[L->u[f]];
        if (a == b) continue;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        int found;
        int* slot = fmap_get(&fm, ((uint64_t)(uint32_t)lo << 32) | (uint64_t)(uint32_t)hi, &found);
        int cf;
        if (!found) {
            cf = C.nf++;
            *slot = cf;
            C.l[cf] = lo;
            C.u[cf] = hi;
            C.weight[cf] = 0.0;
        } else {
            cf = *slot;
        }
        L->faceMap[f] = cf;
        L->faceFlip[f] = (signed char)(a != lo);
        C.weight[cf] += L->weight[f];
    }
    fmap_free(&fm);
    return C;
}

/* The device agglomeration's parallel handshake matching (voluma_b200/csrc/aggl.cu), restated
 * with synchronous rounds: every unpaired cell names its heaviest unpaired neighbour (weight, then
 * the SplitMix64 hash of the cell pair, Steele, Lea and Flood, OOPSLA 2014), mutual names pair up,
 * until no pair forms; a cell left alone joins its heaviest neighbour's aggregate, a cell without
 * neighbours is an aggregate of its own; aggregates numbered by their first cell; coarse faces in
 * (lower, upper) order with weights summed in fine-face order. */
static uint64_t pair_hash(int a, int b) {
    const uint32_t lo = (uint32_t)(a < b ? a : b), hi = (uint32_t)(a < b ? b : a);
    uint64_t z = (((uint64_t)lo << 32) | hi) + 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static int heavier(double w, uint64_t h, double bw, uint64_t bh) { return w > bw || (w == bw && h > bh); }

typedef struct {
    uint64_t key;
    int face;
} keyface_t;

static int cmp_keyface(const void* a, const void* b) {
    const keyface_t* x = (const keyface_t*)a;
    const keyface_t* y = (const keyface_t*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->face < y->face ? -1 : (x->face > y->face ? 1 : 0);
}

static vo_level agglomerate_matching(vo_level* L) {
    const int n = L->n;
    int* match = (int*)malloc(sizeof(int) * (size_t)(n ? n : 1));
    int* pref = (int*)malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int i = 0; i < n; ++i) match[i] = -1;
    for (;;) {
        for (int i = 0; i < n; ++i) {
            int best = -1;
            double bw = 0.0;
            uint64_t bh = 0;
            if (match[i] < 0)
                for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
                    const int j = L->adjCell[k];
                    if (match[j] >= 0) continue;
                    const double w = L->weight[L->adjFace[k]];
                    const uint64_t h = pair_hash(i, j);
                    if (best < 0 || heavier(w, h, bw, bh)) {
                        best = j;
                        bw = w;
                        bh = h;
                    }
                }
            pref[i] = best;
        }
        int paired = 0;
        for (int i = 0; i < n; ++i)
            if (match[i] < 0 && pref[i] >= 0 && pref[pref[i]] == i) {
                match[i] = pref[i];
                ++paired;
            }
        if (paired == 0) break;
    }
    int* id = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    int nc = 0;
    for (int i = 0; i < n; ++i) {
        id[i] = nc;
        const int lead = match[i] >= 0 ? (i < match[i]) : (L->off[i + 1] == L->off[i]);
        nc += lead;
    }
    free(L->agg);
    L->agg = (int*)malloc(sizeof(int) * (size_t)(n ? n : 1));
    for (int i = 0; i < n; ++i) {
        const int m = match[i];
        if (m >= 0) {
            L->agg[i] = id[i < m ? i : m];
        } else if (L->off[i + 1] == L->off[i]) {
            L->agg[i] = id[i];
        } else {
            int best = -1;
            double bw = 0.0;
            uint64_t bh = 0;
            for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
                const int j = L->adjCell[k];
                const double w = L->weight[L->adjFace[k]];
                const uint64_t h = pair_hash(i, j);
                if (best < 0 || heavier(w, h, bw, bh)) {
                    best = j;
                    bw = w;
                    bh = h;
                }
            }
            const int mb = match[best];
            L->agg[i] = id[best < mb ? best : mb];
        }
    }
    free(match);
    free(pref);
    free(id);
    vo_level C;
    memset(&C, 0, sizeof C);
    C.n = nc;
    free(L->faceMap);
    free(L->faceFlip);
    const size_t nfa = (size_t)(L->nf ? L->nf : 1);
    L->faceMap = (int*)malloc(sizeof(int) * nfa);
    L->faceFlip = (signed char*)calloc(nfa, 1);
    C.l = (int*)malloc(sizeof(int) * nfa);
    C.u = (int*)malloc(sizeof(int) * nfa);
    C.weight = (double*)malloc(sizeof(double) * nfa);
    keyface_t* kf = (keyface_t*)malloc(sizeof(keyface_t) * nfa);
    int m = 0;
    for (int f = 0; f < L->nf; ++f) {
        L->faceMap[f] = -1;
        const int a = L->agg[L->l[f]], b = L->agg[L->u[f]];
        if (a == b) continue;
        const int lo = a < b ? a : b, hi = a < b ? b : a;
        kf[m].key = ((uint64_t)(uint32_t)lo << 32) | (uint64_t)(uint32_t)hi;
        kf[m].face = f;
        ++m;
    }
    qsort(kf, (size_t)m, sizeof(keyface_t), cmp_keyface);
    for (int k = 0; k < m; ++k) {
        if (k == 0 || kf[k].key != kf[k - 1].key) {
            C.l[C.nf] = (int)(kf[k].key >> 32);
            C.u[C.nf] = (int)(kf[k].key & 0xffffffffu);
            C.weight[C.nf] = 0.0;
            C.nf++;
        }
        const int cf = C.nf - 1, f = kf[k].face;
        L->faceMap[f] = cf;
        L->faceFlip[f] = (signed char)(L->agg[L->l[f]] != C.l[cf]);
        C.weight[cf] += L->weight[f];
    }
    free(kf);
    return C;
}

static vo_hier* hier_build(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                           int mergeLevels, int nCoarsest, vo_level (*pass)(vo_level*));

vo_hier* vo_hier_build(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                       int mergeLevels, int nCoarsest) {
    return hier_build(n, nf, own, nei, magSf, ndc, mergeLevels, nCoarsest, agglomerate);
}

vo_hier* vo_hier_build_matching(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                                int mergeLevels, int nCoarsest) {
    return hier_build(n, nf, own, nei, magSf, ndc, mergeLevels, nCoarsest, agglomerate_matching);
}

static vo_hier* hier_build(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                           int mergeLevels, int nCoarsest, vo_level (*pass)(vo_level*)) {
    if (mergeLevels < 1) mergeLevels = 1;
    if (nCoarsest <= 0) nCoarsest = 64;
    vo_hier* H = (vo_hier*)calloc(1, sizeof(vo_hier));
    H->ownerIsL = (signed char*)malloc((size_t)(nf ? nf : 1));
    vo_level* L0 = &H->lev[0];
    L0->n = n;
    L0->l = (int*)malloc(sizeof(int) * (size_t)(nf ? nf : 1));
    L0->u = (int*)malloc(sizeof(int) * (size_t)(nf ? nf : 1));
    L0->weight = (double*)malloc(sizeof(double) * (size_t)(nf ? nf : 1));
    for (int f = 0; f < nf; ++f) {
        const int o = own[f], m = nei[f];
        if (o == m) continue; /* self-coupled faces are not part of level 0 (GAMG.cpp:212) */
        L0->l[L0->nf] = o < m ? o : m;
        L0->u[L0->nf] = o < m ? m : o;
        L0->weight[L0->nf] = magSf[f] * ndc[f];
        H->ownerIsL[L0->nf] = (signed char)(o < m);
        L0->nf++;
    }
    build_adjacency(L0);
    H->nL = 1;
    while (H->nL < 40) {
        vo_level* F = &H->lev[H->nL - 1];
        const int nF = F->n;
        if (nF <= nCoarsest) break;
        vo_level C = pass(F);
        for (int k = 1; k < mergeLevels && C.n > nCoarsest; ++k) {
            build_adjacency(&C);
            vo_level C2 = pass(&C);
            for (int i = 0; i < F->n; ++i) F->agg[i] = C.agg[F->agg[i]];
            for (int f = 0; f < F->nf; ++f) {
                const int cf = F->faceMap[f];
                if (cf < 0) continue;
                F->faceMap[f] = C.faceMap[cf];
                F->faceFlip[f] = (signed char)(F->faceFlip[f] != C.faceFlip[cf]);
            }
            level_free(&C);
            C = C2;
        }
        if (C.n >= nF) {
            free(F->agg);
            F->agg = NULL;
            level_free(&C);
            break;
        }
        build_adjacency(&C);
        H->lev[H->nL++] = C;
    }
    return H;
}

void vo_hier_free(vo_hier* h) {
    if (!h) return;
    for (int k = 0; k < h->nL; ++k) level_free(&h->lev[k]);
    free(h->ownerIsL);
    free(h);
}

int vo_hier_nlevels(const vo_hier* h) { return h->nL; }

void vo_hier_level(const vo_hier* h, int lev, int* sizes, int* l, int* u, double* weight, int* agg, int* faceMap,
                   signed char* faceFlip) {
    const vo_level* L = &h->lev[lev];
    const int hasAgg = L->agg != NULL && lev + 1 < h->nL;
    sizes[0] = L->n;
    sizes[1] = L->nf;
    sizes[2] = hasAgg ? L->n : 0;
    if (l) memcpy(l, L->l, sizeof(int) * (size_t)L->nf);
    if (u) memcpy(u, L->u, sizeof(int) * (size_t)L->nf);
    if (weight) memcpy(weight, L->weight, sizeof(double) * (size_t)L->nf);
    if (agg && hasAgg) memcpy(agg, L->agg, sizeof(int) * (size_t)L->n);
    if (faceMap && hasAgg) memcpy(faceMap, L->faceMap, sizeof(int) * (size_t)L->nf);
    if (faceFlip && hasAgg) memcpy(faceFlip, L->faceFlip, (size_t)L->nf);
}

/* greedy colouring in natural order: smallest colour not used by a coloured neighbour */
int vo_hier_colour(const vo_hier* h, int lev, int* colour) {
    const vo_level* L = &h->lev[lev];
    int nc = 0;
    int* mark = (int*)malloc(sizeof(int) * 256);
    int cap = 256;
    for (int c = 0; c < cap; ++c) mark[c] = -1;
    for (int i = 0; i < L->n; ++i) colour[i] = -1;
    for (int i = 0; i < L->n; ++i) {
        for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
            const int c = colour[L->adjCell[k]];
            if (c >= cap) {
                mark = (int*)realloc(mark, sizeof(int) * (size_t)(2 * c));
                for (int q = cap; q < 2 * c; ++q) mark[q] = -1;
                cap = 2 * c;
            }
            if (c >= 0) mark[c] = i;
        }
        int c = 0;
        while (c < cap && mark[c] == i) ++c;
        colour[i] = c;
        if (c + 1 > nc) nc = c + 1;
    }
    free(mark);
    return nc;
}

/* ======================================================================= GAMG preconditioner */
static void block_colour(const vo_level* L, int* colour);
typedef struct {
    const vo_hier* H;
    int nL;
    double** diag;
    double** up;
    double** lo;
    double* lu;    /* coarsest LU, row major */
    double* inv;   /* explicit inverse (coarse == 1) */
    int nc;
    int** colour;
    int* ncol;
    int* blockGS;  /* level uses the block-hybrid Gauss-Seidel of the device */
    int** bcol;    /* block-local colour of each row (block levels) */
    double** xb;
    double** rb;
    double** tb;
    double** x2;
    vo_gamg_opts opt;
} gamg_t;

static void gamg_free(gamg_t* g) {
    for (int k = 0; k < g->nL; ++k) {
        free(g->diag[k]);
        free(g->up[k]);
        free(g->lo[k]);
        free(g->colour[k]);
        free(g->xb[k]);
        free(g->rb[k]);
        free(g->tb[k]);
        free(g->x2[k]);
    }
    free(g->diag);
    free(g->up);
    free(g->lo);
    for (int k = 0; k < g->nL; ++k) free(g->bcol[k]);
    free(g->bcol);
    free(g->blockGS);
    free(g->colour);
    free(g->ncol);
    free(g->xb);
    free(g->rb);
    free(g->tb);
    free(g->x2);
    free(g->lu);
    free(g->inv);
}

/* GamgPreconditioner ctor (GAMG.cpp:263-353), serial */
static int gamg_init(gamg_t* g, const vo_hier* H, const double* diag, const double* upper, const double* lower,
                     const vo_gamg_opts* opt) {
    memset(g, 0, sizeof *g);
    g->H = H;
    g->opt = *opt;
    const int nL = H->nL;
    g->nL = nL;
    g->diag = (double**)calloc((size_t)nL, sizeof(double*));
    g->up = (double**)calloc((size_t)nL, sizeof(double*));
    g->lo = (double**)calloc((size_t)nL, sizeof(double*));
    g->colour = (int**)calloc((size_t)nL, sizeof(int*));
    g->ncol = (int*)calloc((size_t)nL, sizeof(int));
    g->blockGS = (int*)calloc((size_t)nL, sizeof(int));
    g->bcol = (int**)calloc((size_t)nL, sizeof(int*));
    g->xb = (double**)calloc((size_t)nL, sizeof(double*));
    g->rb = (double**)calloc((size_t)nL, sizeof(double*));
    g->tb = (double**)calloc((size_t)nL, sizeof(double*));
    g->x2 = (double**)calloc((size_t)nL, sizeof(double*));
    for (int k = 0; k < nL; ++k) {
        const vo_level* L = &H->lev[k];
        g->diag[k] = (double*)calloc((size_t)L->n + 1, sizeof(double));
        g->up[k] = (double*)calloc((size_t)L->nf + 1, sizeof(double));
        g->lo[k] = (double*)calloc((size_t)L->nf + 1, sizeof(double));
        g->xb[k] = (double*)calloc((size_t)L->n + 1, sizeof(double));
        g->rb[k] = (double*)calloc((size_t)L->n + 1, sizeof(double));
        g->tb[k] = (double*)calloc((size_t)L->n + 1, sizeof(double));
        g->x2[k] = (double*)calloc((size_t)L->n + 1, sizeof(double));
        g->colour[k] = (int*)calloc((size_t)L->n + 1, sizeof(int));
        g->ncol[k] = vo_hier_colour(H, k, g->colour[k]);
        /* device schedule: level 0 keeps a global multicolour GS when it needs <= 4 colours,
           every other level runs the block-hybrid GS */
        g->blockGS[k] = k > 0 || g->ncol[k] > VO_MAX_GLOBAL_COLOURS;
        g->bcol[k] = (int*)calloc((size_t)L->n + 1, sizeof(int));
        block_colour(L, g->bcol[k]);
    }
    {
        const vo_level* L = &H->lev[0];
        memcpy(g->diag[0], diag, sizeof(double) * (size_t)L->n);
        for (int k = 0; k < L->nf; ++k) {
            /* level-0 faces are the mesh faces in order (no self-coupled faces) */
            g->up[0][k] = H->ownerIsL[k] ? upper[k] : lower[k];
            g->lo[0][k] = H->ownerIsL[k] ? lower[k] : upper[k];
        }
    }
    for (int lev = 0; lev + 1 < nL; ++lev) {
        const vo_level* L = &H->lev[lev];
        double* Cd = g->diag[lev + 1];
        double* Cu = g->up[lev + 1];
        double* Cl = g->lo[lev + 1];
        for (int i = 0; i < L->n; ++i) Cd[L->agg[i]] += g->diag[lev][i];
        for (int f = 0; f < L->nf; ++f) {
            const int cf = L->faceMap[f];
            if (cf < 0) {
                Cd[L->agg[L->l[f]]] += g->up[lev][f] + g->lo[lev][f];
            } else if (!L->faceFlip[f]) {
                Cu[cf] += g->up[lev][f];
                Cl[cf] += g->lo[lev][f];
            } else {
                Cu[cf] += g->lo[lev][f];
                Cl[cf] += g->up[lev][f];
            }
        }
    }
    const vo_level* LC = &H->lev[nL - 1];
    const int n = LC->n;
    g->nc = n;
    double* A = (double*)calloc((size_t)n * n + 1, sizeof(double));
    g->lu = A;
    for (int i = 0; i < n; ++i) A[(size_t)i * n + i] = g->diag[nL - 1][i];
    for (int f = 0; f < LC->nf; ++f) {
        A[(size_t)LC->l[f] * n + LC->u[f]] += g->up[nL - 1][f];
        A[(size_t)LC->u[f] * n + LC->l[f]] += g->lo[nL - 1][f];
    }
    for (int k = 0; k < n; ++k) {
        const double piv = A[(size_t)k * n + k];
        if (fabs(piv) < VSMALL) return 4;
        for (int i = k + 1; i < n; ++i) {
            const double fct = A[(size_t)i * n + k] / piv;
            A[(size_t)i * n + k] = fct;
            if (fct == 0.0) continue;
            for (int j = k + 1; j < n; ++j) A[(size_t)i * n + j] -= fct * A[(size_t)k * n + j];
        }
    }
    if (opt->coarse == 1) {
        double* X = (double*)calloc((size_t)n * n + 1, sizeof(double));
        g->inv = X;
        for (int j = 0; j < n; ++j) {
            for (int i = 0; i < n; ++i) {
                double v = i == j ? 1.0 : 0.0;
                for (int k = 0; k < i; ++k) v -= A[(size_t)i * n + k] * X[(size_t)k * n + j];
                X[(size_t)i * n + j] = v;
            }
            /* U back substitution with the upper terms in descending k (the device kernel's
               right-looking order) */
            for (int i = n - 1; i >= 0; --i) {
                double v = X[(size_t)i * n + j];
                for (int k = n - 1; k > i; --k) v -= A[(size_t)i * n + k] * X[(size_t)k * n + j];
                X[(size_t)i * n + j] = v / A[(size_t)i * n + i];
            }
        }
    }
    return 0;
}

static double row_minus(const vo_level* L, const double* up, const double* lo, const double* x, int i, double s) {
    for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
        const int f = L->adjFace[k];
        s -= (L->adjIsL[k] ? up[f] : lo[f]) * x[L->adjCell[k]];
    }
    return s;
}

/* Greedy colouring of each block of VO_BLOCK_ROWS consecutive rows, in-block edges only. */
static void block_colour(const vo_level* L, int* colour) {
    int mark[256];
    for (int s0 = 0; s0 < L->n; s0 += VO_BLOCK_ROWS) {
        const int s1 = s0 + VO_BLOCK_ROWS < L->n ? s0 + VO_BLOCK_ROWS : L->n;
        for (int q = 0; q < 256; ++q) mark[q] = -1;
        for (int i = s0; i < s1; ++i) colour[i] = -1;
        for (int i = s0; i < s1; ++i) {
            for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
                const int j = L->adjCell[k];
                if (j < s0 || j >= s1) continue;
                if (colour[j] >= 0) mark[colour[j]] = i;
            }
            int c = 0;
            while (c < 256 && mark[c] == i) ++c;
            colour[i] = c;
        }
    }
}

/* GAMG.cpp:363-385 and the device smoothers */
static void gamg_smooth(gamg_t* g, int lev, const double* r, double* x, int forward) {
    const vo_level* L = &g->H->lev[lev];
    const double* D = g->diag[lev];
    const double* up = g->up[lev];
    const double* lo = g->lo[lev];
    if (g->opt.smoother == 3 && lev > 0) {
        double* xo = g->x2[lev];
        const double om = g->opt.omega;
        for (int i = 0; i < L->n; ++i) {
            const double v = row_minus(L, up, lo, x, i, r[i]) / D[i];
            xo[i] = om == 1.0 ? v : x[i] + om * (v - x[i]);
        }
        memcpy(x, xo, sizeof(double) * (size_t)L->n);
    } else if ((g->opt.smoother == 1 || g->opt.smoother == 3) && g->blockGS[lev]) {
        /* block-hybrid GS: Gauss-Seidel inside each block in block-local colour order; the terms
           of neighbours outside the block (previous sweep) are subtracted first, then the
           in-block terms, each group in face order */
        double* xi = g->x2[lev];
        memcpy(xi, x, sizeof(double) * (size_t)L->n);
        const int* bc = g->bcol[lev];
        for (int s0 = 0; s0 < L->n; s0 += VO_BLOCK_ROWS) {
            const int s1 = s0 + VO_BLOCK_ROWS < L->n ? s0 + VO_BLOCK_ROWS : L->n;
            int nc = 0;
            for (int i = s0; i < s1; ++i)
                if (bc[i] + 1 > nc) nc = bc[i] + 1;
            double* sout = g->tb[lev];  /* out-of-block partial sums of the block's rows */
            for (int i = s0; i < s1; ++i) {
                double sum = r[i];
                for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
                    const int j = L->adjCell[k];
                    if (j >= s0 && j < s1) continue;
                    const int f = L->adjFace[k];
                    sum -= (L->adjIsL[k] ? up[f] : lo[f]) * xi[j];
                }
                sout[i] = sum;
            }
            for (int t = 0; t < nc; ++t) {
                const int c = forward ? t : nc - 1 - t;
                for (int i = s0; i < s1; ++i) {
                    if (bc[i] != c) continue;
                    double sum = sout[i];
                    for (int k = L->off[i]; k < L->off[i + 1]; ++k) {
                        const int j = L->adjCell[k];
                        if (!(j >= s0 && j < s1)) continue;
                        const int f = L->adjFace[k];
                        sum -= (L->adjIsL[k] ? up[f] : lo[f]) * x[j];
                    }
                    x[i] = sum / D[i];
                }
            }
        }
    } else if (g->opt.smoother == 0) {
        if (forward)
            for (int i = 0; i < L->n; ++i) x[i] = row_minus(L, up, lo, x, i, r[i]) / D[i];
        else
            for (int i = L->n - 1; i >= 0; --i) x[i] = row_minus(L, up, lo, x, i, r[i]) / D[i];
    } else if (g->opt.smoother == 1 || g->opt.smoother == 3) {
        const int nc = g->ncol[lev];
        const int* col = g->colour[lev];
        for (int t = 0; t < nc; ++t) {
            const int c = forward ? t : nc - 1 - t;
            for (int i = 0; i < L->n; ++i)
                if (col[i] == c) x[i] = row_minus(L, up, lo, x, i, r[i]) / D[i];
        }
    } else {
        double* xo = g->x2[lev];
        const double om = g->opt.omega;
        for (int i = 0; i < L->n; ++i) {
            const double v = row_minus(L, up, lo, x, i, r[i]) / D[i];
            xo[i] = om == 1.0 ? v : x[i] + om * (v - x[i]);
        }
        memcpy(x, xo, sizeof(double) * (size_t)L->n);
    }
}

/* GAMG.cpp:387-401 */
static void gamg_residual(gamg_t* g, int lev, const double* r, const double* x, double* res) {
    const vo_level* L = &g->H->lev[lev];
    const double* D = g->diag[lev];
    for (int i = 0; i < L->n; ++i) res[i] = r[i] - D[i] * x[i];
    for (int f = 0; f < L->nf; ++f) {
        res[L->l[f]] -= g->up[lev][f] * x[L->u[f]];
        res[L->u[f]] -= g->lo[lev][f] * x[L->l[f]];
    }
}

/* GAMG.cpp:403-443 */
static void gamg_vcycle(gamg_t* g, int lev, const double* r, double* x) {
    const vo_level* L = &g->H->lev[lev];
    if (lev == g->nL - 1) {
        const int n = g->nc;
        if (g->opt.coarse == 1) {
            for (int i = 0; i < n; ++i) {
                double v = 0.0;
                for (int j = 0; j < n; ++j) v += g->inv[(size_t)i * n + j] * r[j];
                g->tb[lev][i] = v;
            }
            memcpy(x, g->tb[lev], sizeof(double) * (size_t)n);
            return;
        }
        double* v = g->tb[lev];
        for (int i = 0; i < n; ++i) v[i] = r[i];
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < i; ++k) v[i] -= g->lu[(size_t)i * n + k] * v[k];
        for (int i = n - 1; i >= 0; --i) {
            for (int k = i + 1; k < n; ++k) v[i] -= g->lu[(size_t)i * n + k] * v[k];
            v[i] /= g->lu[(size_t)i * n + i];
        }
        memcpy(x, v, sizeof(double) * (size_t)n);
        return;
    }
    for (int i = 0; i < L->n; ++i) x[i] = 0.0;
    for (int s = 0; s < 2; ++s) gamg_smooth(g, lev, r, x, 1);
    double* res = g->tb[lev];
    gamg_residual(g, lev, r, x, res);
    double* rc = g->rb[lev + 1];
    double* xc = g->xb[lev + 1];
    const vo_level* C = &g->H->lev[lev + 1];
    for (int i = 0; i < C->n; ++i) rc[i] = 0.0;
    for (int i = 0; i < L->n; ++i) rc[L->agg[i]] += res[i];
    gamg_vcycle(g, lev + 1, rc, xc);
    for (int i = 0; i < L->n; ++i) x[i] += xc[L->agg[i]];
    for (int s = 0; s < 2; ++s) gamg_smooth(g, lev, r, x, 0);
}

int vo_gamg_apply(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                  const double* diag, const double* upper, const double* lower, const double* r, double* w,
                  const vo_gamg_opts* opt) {
    vo_hier* H = (opt->matching ? vo_hier_build_matching : vo_hier_build)(n, nf, own, nei, magSf, ndc,
                                                                           opt->mergeLevels ? opt->mergeLevels : 2, 64);
    gamg_t g;
    const int st = gamg_init(&g, H, diag, upper, lower ? lower : upper, opt);
    if (st == 0) gamg_vcycle(&g, 0, r, w);
    gamg_free(&g);
    vo_hier_free(H);
    return st;
}

/* ======================================================================= DIC / DILU */
/* Faces of the DIC/DILU sweeps (LinearSolver.cpp:28-50): internal faces between two distinct
 * cells, (l, u) = (min, max), sorted by (u, l, face). */
typedef struct {
    int n, m;
    int *face, *l, *u;
    unsigned char* ownerIsL;
    double* rD;
} dilu_t;

static int cmp_ulf(const void* a, const void* b) {
    const int* x = (const int*)a;
    const int* y = (const int*)b;
    for (int q = 0; q < 3; ++q)
        if (x[q] != y[q]) return x[q] < y[q] ? -1 : 1;
    return 0;
}

/* LinearSolver.cpp:66-77: rD[u] -= A_lu A_ul / rD[l] over the sorted faces, then rD = 1 / rD */
static void dilu_init(dilu_t* P, int n, int nf, const int* own, const int* nei, const double* diag,
                      const double* upper, const double* lower) {
    int* t = (int*)malloc(sizeof(int) * 3 * (size_t)(nf > 0 ? nf : 1));
    int m = 0;
    for (int f = 0; f < nf; ++f) {
        const int o = own[f], q = nei[f];
        if (o >= n || q >= n || o == q) continue;
        t[3 * m] = o > q ? o : q;
        t[3 * m + 1] = o < q ? o : q;
        t[3 * m + 2] = f;
        ++m;
    }
    qsort(t, (size_t)m, sizeof(int) * 3, cmp_ulf);
    P->n = n;
    P->m = m;
    P->face = (int*)malloc(sizeof(int) * (size_t)(m + 1));
    P->l = (int*)malloc(sizeof(int) * (size_t)(m + 1));
    P->u = (int*)malloc(sizeof(int) * (size_t)(m + 1));
    P->ownerIsL = (unsigned char*)malloc((size_t)(m + 1));
    P->rD = (double*)malloc(sizeof(double) * (size_t)(n + 1));
    for (int k = 0; k < m; ++k) {
        P->u[k] = t[3 * k];
        P->l[k] = t[3 * k + 1];
        P->face[k] = t[3 * k + 2];
        P->ownerIsL[k] = own[P->face[k]] == P->l[k];
    }
    free(t);
    for (int c = 0; c < n; ++c) P->rD[c] = diag[c];
    for (int k = 0; k < m; ++k) {
        const int f = P->face[k];
        const double Alu = P->ownerIsL[k] ? upper[f] : lower[f];
        const double Aul = P->ownerIsL[k] ? lower[f] : upper[f];
        P->rD[P->u[k]] -= Alu * Aul / P->rD[P->l[k]];
    }
    for (int c = 0; c < n; ++c) P->rD[c] = 1.0 / P->rD[c];
}

/* LinearSolver.cpp:87-106: w = rD r, forward and backward substitution over the sorted faces */
static void dilu_apply(const dilu_t* P, const double* upper, const double* lower, const double* r, double* w) {
    for (int c = 0; c < P->n; ++c) w[c] = P->rD[c] * r[c];
    for (int k = 0; k < P->m; ++k) {
        const int f = P->face[k];
        const double Aul = P->ownerIsL[k] ? lower[f] : upper[f];
        w[P->u[k]] -= P->rD[P->u[k]] * Aul * w[P->l[k]];
    }
    for (int k = P->m; k-- > 0;) {
        const int f = P->face[k];
        const double Alu = P->ownerIsL[k] ? upper[f] : lower[f];
        w[P->l[k]] -= P->rD[P->l[k]] * Alu * w[P->u[k]];
    }
}

static void dilu_free(dilu_t* P) {
    free(P->face);
    free(P->l);
    free(P->u);
    free(P->ownerIsL);
    free(P->rD);
}

int vo_precond_apply(int n, int nf, const int* own, const int* nei, const double* diag, const double* upper,
                     const double* lower, const char* precond, const double* r, double* w) {
    if (!lower) lower = upper;
    if (strcmp(precond, "none") == 0) {
        memcpy(w, r, sizeof(double) * (size_t)n);
    } else if (strcmp(precond, "diagonal") == 0) {
        for (int c = 0; c < n; ++c) w[c] = 1.0 / diag[c] * r[c];
    } else if (strcmp(precond, "DIC") == 0 || strcmp(precond, "DILU") == 0) {
        dilu_t P;
        dilu_init(&P, n, nf, own, nei, diag, upper, lower);
        dilu_apply(&P, upper, lower, r, w);
        dilu_free(&P);
    } else {
        return 7;
    }
    return 0;
}

/* ======================================================================= solveLdu */
typedef struct {
    int kind; /* 0 none, 1 diagonal, 2 GAMG, 3 DIC/DILU */
    int n;
    double* rD;
    gamg_t g;
    vo_hier* H;
    dilu_t d;
    const double *up, *lo;
} prec_t;

static void prec_apply(prec_t* P, const double* r, double* w) {
    if (P->kind == 0) {
        memcpy(w, r, sizeof(double) * (size_t)P->n);
    } else if (P->kind == 1) {
        for (int c = 0; c < P->n; ++c) w[c] = P->rD[c] * r[c];
    } else if (P->kind == 3) {
        dilu_apply(&P->d, P->up, P->lo, r, w);
    } else {
        gamg_vcycle(&P->g, 0, r, P->g.xb[0]);
        memcpy(w, P->g.xb[0], sizeof(double) * (size_t)P->n);
    }
}

static int converged(double tol, double relTol, int minIter, int iters, double fin, double init) {
    if (iters < minIter) return 0;
    return fin < tol || (relTol > 0 && fin < relTol * init);
}

/* sweepCell of LinearSolver.cpp:245-259: the cell's faces in cellFaces order (ascending face,
 * a face listed twice when both its sides are the cell, Mesh.cpp:630-641) */
static double sweep_cell(int c, const int* cfOff, const int* cf, const int* own, const int* nei, const double* diag,
                         const double* upper, const double* lower, const double* b, const double* xs) {
    double r = b[c];
    for (int k = cfOff[c]; k < cfOff[c + 1]; ++k) {
        const int f = cf[k];
        if (own[f] == c && nei[f] == c)
            r -= (upper[f] + lower[f]) * xs[c];
        else if (own[f] == c)
            r -= upper[f] * xs[nei[f]];
        else
            r -= lower[f] * xs[own[f]];
    }
    return r / diag[c];
}

int vo_solve(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
             const double* diag, const double* upper, const double* lower, const double* b, double* x,
             const char* solver, const char* precond, double tol, double relTol, int maxIter, int minIter,
             int exactSums, const vo_gamg_opts* opt, double* perf) {
    return vo_solve_ex(n, nf, own, nei, magSf, ndc, diag, upper, lower, b, x, solver, precond, tol, relTol, maxIter,
                       minIter, 1, exactSums, opt, perf);
}

int vo_solve_ex(int n, int nf, const int* own, const int* nei, const double* magSf, const double* ndc,
                const double* diag, const double* upper, const double* lower, const double* b, double* x,
                const char* solver, const char* precond, double tol, double relTol, int maxIter, int minIter,
                int nSweeps, int exactSums, const vo_gamg_opts* opt, double* perf) {
    const int sym = lower == NULL || lower == upper;
    if (!lower) lower = upper;
    const int pcg = strcmp(solver, "PCG") == 0;
    const int bicg = strcmp(solver, "PBiCGStab") == 0;
    int gs = strcmp(solver, "GaussSeidel") == 0, sgs = strcmp(solver, "symGaussSeidel") == 0;
    int jac = strcmp(solver, "Jacobi") == 0;
    if (!pcg && !bicg && !gs && !sgs && !jac) return 7;
    if (pcg && !sym) return 7;
    if (exactSums && (gs || sgs)) { /* CFD_REPRODUCIBLE swap, LinearSolver.cpp:141 */
        gs = sgs = 0;
        jac = 1;
    }
    const int relax = gs || sgs || jac;
    if (relax && nSweeps < 1) return 1;
    prec_t P;
    memset(&P, 0, sizeof P);
    P.n = n;
    P.up = upper;
    P.lo = lower;
    if (relax || strcmp(precond, "none") == 0)
        P.kind = 0;
    else if (strcmp(precond, "diagonal") == 0)
        P.kind = 1;
    else if (strcmp(precond, "GAMG") == 0)
        P.kind = 2;
    else if (strcmp(precond, "DIC") == 0 || strcmp(precond, "DILU") == 0)
        P.kind = 3;
    else
        return 7;
    if (exactSums && P.kind != 0) P.kind = 1; /* CFD_REPRODUCIBLE swap, LinearSolver.cpp:138-148 */
    double* wA = (double*)calloc((size_t)n + 1, sizeof(double));
    double* rA = (double*)calloc((size_t)n + 1, sizeof(double));
    double* pA = (double*)calloc((size_t)n + 1, sizeof(double));
    double* xr = (double*)calloc((size_t)n + 1, sizeof(double));
    int status = 0;
    vo_amul(n, nf, own, nei, diag, upper, lower, x, wA);
    for (int c = 0; c < n; ++c) rA[c] = b[c] - wA[c];
    sum_t xs;
    sum_init(&xs, exactSums);
    for (int c = 0; c < n; ++c) sum_add(&xs, x[c]);
    const double xRef = sum_get(&xs) / (double)n;
    for (int c = 0; c < n; ++c) xr[c] = xRef;
    vo_amul(n, nf, own, nei, diag, upper, lower, xr, pA);
    sum_t nfs;
    sum_init(&nfs, exactSums);
    for (int c = 0; c < n; ++c) sum_add(&nfs, fabs(wA[c] - pA[c]) + fabs(b[c] - pA[c]));
    const double normFactor = sum_get(&nfs) + 1e-20;
    double residualSum = gSumMag(rA, n, exactSums);
    double init = residualSum / normFactor, fin = init;
    int it = 0;
    if (!(init < tol && minIter <= 0)) {
        if (P.kind == 1) {
            P.rD = (double*)malloc(sizeof(double) * (size_t)n);
            for (int c = 0; c < n; ++c) P.rD[c] = 1.0 / diag[c];
        } else if (P.kind == 2) {
            P.H = (opt->matching ? vo_hier_build_matching : vo_hier_build)(n, nf, own, nei, magSf, ndc,
                                                                           opt->mergeLevels ? opt->mergeLevels : 2, 64);
            status = gamg_init(&P.g, P.H, diag, upper, lower, opt);
        } else if (P.kind == 3) {
            dilu_init(&P.d, n, nf, own, nei, diag, upper, lower);
        }
        if (status == 0 && relax) {
            /* LinearSolver.cpp:238-278 */
            int* cfOff = (int*)calloc((size_t)n + 1, sizeof(int));
            for (int f = 0; f < nf; ++f) {
                if (own[f] < n) ++cfOff[own[f] + 1];
                if (nei[f] < n) ++cfOff[nei[f] + 1];
            }
            for (int c = 0; c < n; ++c) cfOff[c + 1] += cfOff[c];
            int* cf = (int*)malloc(sizeof(int) * (size_t)(cfOff[n] + 1));
            int* fill = (int*)malloc(sizeof(int) * (size_t)(n + 1));
            for (int c = 0; c < n; ++c) fill[c] = cfOff[c];
            for (int f = 0; f < nf; ++f) {
                if (own[f] < n) cf[fill[own[f]]++] = f;
                if (nei[f] < n) cf[fill[nei[f]]++] = f;
            }
            double* xOld = (double*)malloc(sizeof(double) * (size_t)(n + 1));
            do {
                for (int sw = 0; sw < nSweeps; ++sw) {
                    if (jac) {
                        memcpy(xOld, x, sizeof(double) * (size_t)n);
                        for (int c = 0; c < n; ++c)
                            x[c] = sweep_cell(c, cfOff, cf, own, nei, diag, upper, lower, b, xOld);
                    } else {
                        for (int c = 0; c < n; ++c) x[c] = sweep_cell(c, cfOff, cf, own, nei, diag, upper, lower, b, x);
                        if (sgs)
                            for (int c = n; c-- > 0;)
                                x[c] = sweep_cell(c, cfOff, cf, own, nei, diag, upper, lower, b, x);
                    }
                }
                it += nSweeps;
                vo_amul(n, nf, own, nei, diag, upper, lower, x, wA);
                for (int c = 0; c < n; ++c) rA[c] = b[c] - wA[c];
                fin = gSumMag(rA, n, exactSums) / normFactor;
            } while (it < maxIter && !converged(tol, relTol, minIter, it, fin, init));
            free(cfOff);
            free(cf);
            free(fill);
            free(xOld);
        } else if (status == 0 && pcg) {
            double* w = (double*)calloc((size_t)n + 1, sizeof(double));
            double* p = (double*)calloc((size_t)n + 1, sizeof(double));
            double wArA = GREAT, wArAold;
            do {
                wArAold = wArA;
                prec_apply(&P, rA, w);
                wArA = gSumProd(w, rA, n, exactSums);
                if (it == 0) {
                    for (int c = 0; c < n; ++c) p[c] = w[c];
                } else {
                    const double beta = wArA / wArAold;
                    for (int c = 0; c < n; ++c) p[c] = w[c] + beta * p[c];
                }
                vo_amul(n, nf, own, nei, diag, upper, lower, p, wA);
                const double wApA = gSumProd(wA, p, n, exactSums);
                if (fabs(wApA) < VSMALL) break;
                const double alpha = wArA / wApA;
                for (int c = 0; c < n; ++c) {
                    x[c] += alpha * p[c];
                    rA[c] -= alpha * wA[c];
                }
                fin = gSumMag(rA, n, exactSums) / normFactor;
                ++it;
            } while (it < maxIter && !converged(tol, relTol, minIter, it, fin, init));
            free(w);
            free(p);
        } else if (status == 0) {
            double* rA0 = (double*)malloc(sizeof(double) * (size_t)n + 8);
            double* p = (double*)calloc((size_t)n + 1, sizeof(double));
            double* y = (double*)calloc((size_t)n + 1, sizeof(double));
            double* Ay = (double*)calloc((size_t)n + 1, sizeof(double));
            double* s = (double*)calloc((size_t)n + 1, sizeof(double));
            double* z = (double*)calloc((size_t)n + 1, sizeof(double));
            double* t = (double*)calloc((size_t)n + 1, sizeof(double));
            memcpy(rA0, rA, sizeof(double) * (size_t)n);
            double rho = 0, alpha = 0, omega = 0;
            do {
                const double rhoOld = rho;
                rho = gSumProd(rA0, rA, n, exactSums);
                if (it == 0) {
                    for (int c = 0; c < n; ++c) p[c] = rA[c];
                } else {
                    if (fabs(rhoOld) < VSMALL || fabs(omega) < VSMALL) break;
                    const double beta = (rho / rhoOld) * (alpha / omega);
                    for (int c = 0; c < n; ++c) p[c] = rA[c] + beta * (p[c] - omega * Ay[c]);
                }
                prec_apply(&P, p, y);
                vo_amul(n, nf, own, nei, diag, upper, lower, y, Ay);
                const double r0Ay = gSumProd(rA0, Ay, n, exactSums);
                if (fabs(r0Ay) < VSMALL) break;
                alpha = rho / r0Ay;
                for (int c = 0; c < n; ++c) s[c] = rA[c] - alpha * Ay[c];
                ++it;
                fin = gSumMag(s, n, exactSums) / normFactor;
                if (converged(tol, relTol, minIter, it, fin, init)) {
                    for (int c = 0; c < n; ++c) x[c] += alpha * y[c];
                    break;
                }
                prec_apply(&P, s, z);
                vo_amul(n, nf, own, nei, diag, upper, lower, z, t);
                const double tt = gSumProd(t, t, n, exactSums);
                omega = tt > VSMALL ? gSumProd(t, s, n, exactSums) / tt : 0.0;
                for (int c = 0; c < n; ++c) {
                    x[c] += alpha * y[c] + omega * z[c];
                    rA[c] = s[c] - omega * t[c];
                }
                fin = gSumMag(rA, n, exactSums) / normFactor;
            } while (it < maxIter && !converged(tol, relTol, minIter, it, fin, init));
            free(rA0);
            free(p);
            free(y);
            free(Ay);
            free(s);
            free(z);
            free(t);
        }
        if (P.kind == 2) {
            gamg_free(&P.g);
            vo_hier_free(P.H);
        }
        if (P.kind == 3) dilu_free(&P.d);
        free(P.rD);
    }
    perf[0] = init;
    perf[1] = fin;
    perf[2] = residualSum;
    perf[3] = normFactor;
    perf[4] = it;
    perf[5] = converged(tol, relTol, minIter, it, fin, init);
    free(wA);
    free(rA);
    free(pA);
    free(xr);
    return status;
}
