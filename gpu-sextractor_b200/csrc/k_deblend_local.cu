// k_deblend_local.cu -- deblending of raw objects of at most 32767 pixels
// with a compact per-object state: in shared memory for objects of at most
// 256 pixels (one warp each), in a global arena of 48 B per pixel otherwise.
//
// Same algorithm and results as k_deblend_sweep / k_deblend_assign (one CTA
// per raw object, incremental union-find sweep from the top threshold down,
// MINCONT cut evaluated two levels at a time, replay sweep for ownership,
// preanalysis of the kept branches, gatherup), with three changes that only
// affect speed:
//
//  * the union-find forest, the component sizes, the branch fluxes, the
//    branch nodes of two consecutive levels and the level order of the pixels
//    are packed (16-bit element indices; about 45 B per pixel in the sweep,
//    34 B in the assignment); grids are persistent, sized to the resident
//    capacity, and take objects from a device-side cursor;
//  * for objects whose state lives in the global arena, the part of it on the
//    sweep's dependent chains -- the union-find parents and the pixel levels,
//    5 B per pixel -- is kept in shared memory instead (the "hybrid" form:
//    every find, link and activity test of the unions is an on-chip access;
//    sizes, fluxes and branch lists stay in the arena);
//  * a branch flux is one 64-bit fixed-scale integer (units of 2^(e0-23),
//    e0 the exponent of the detection threshold, every cd of the object being
//    at least that threshold).  The object's range is checked first: when
//    (exponent of its peak - e0) + 24 + bits(pixels) exceeds 63 the object is
//    handed to the global kernels (128-bit limbs) instead;
//  * levels at which no pixel of the object first passes the threshold are
//    skipped.  At such a level the components do not change, every branch has
//    one child (itself one level up), no branch is cut there and the ok-after
//    state carries over; the only thing that changes is the flag of each
//    branch, which depends on the threshold, so when the next populated level
//    L is reached the branches of the list are re-flagged at threshold L+1
//    before they act as L's children.
//
// Reference for the algorithm: src/cuda/cudadeblend.cu:199-217, :579-727,
// :1262-1360, :1425-1776; src/cuda/cudaanalyse.cu:1686-1903.
#include "common.cuh"
#include "kernels.cuh"

namespace sx {

#ifndef SX_DL_MID
#define SX_DL_MID 2048
#endif
#ifndef SX_DL_ARENA_MAX
#define SX_DL_ARENA_MAX 32767
#endif
constexpr int DL_CAP0 = 256;                   // shared-memory tier (one warp per object)
constexpr int DL_CAP1 = 64;                    // its small-object classes (more warps resident per SM)
constexpr int DL_CAP2 = 128;
constexpr int DL_MID = SX_DL_MID;              // arena tier with 64-thread CTAs up to here, 256 above
constexpr int DL_ARENA_MAX = SX_DL_ARENA_MAX;  // at most 32767: element indices are 16-bit
constexpr int DL_SWEEP_BYTES = 45;   // shared bytes per pixel, sweep
constexpr int DL_ASSIGN_BYTES = 34;  // shared bytes per pixel, assignment
constexpr int DL_ARENA_BYTES = 48;   // global arena bytes per pixel (either pass)

// ---- shared-memory union-find over the element indices of one object
// Path halving: a node's pointer is replaced by its grandparent.  Every
// pointer goes to a smaller element index and only roots are linked, so a
// halving store that races with a link of the same node can only drop that
// link to an ancestor; the linking thread then continues with the old parent,
// so no connection is lost.
// Plain (cached) loads: a stale pointer read is an older pointer to an
// ancestor, so a walk still ends at a root of the same tree, and a union that
// acted on a stale root sees it in the value atomicMin returns and retries.
__device__ __forceinline__ int sfind(int *par, int a, int cap, int *status) {
    for (int n = 0; n <= cap; n++) {
        int p = par[a];
        if (p == a) return a;
        int g = par[p];
        if (g != p) par[a] = g;
        a = g;
    }
    atomicOr(status, SX_ST_LOOP);
    return a;
}

// find with path compression; only used while no union is in flight, so every
// pointer written is the final root of the tree
__device__ __forceinline__ int sfind_c(int *par, int a, int cap, int *status) {
    int rt = sfind(par, a, cap, status);
    for (int n = 0; n <= cap; n++) {
        int p = par[a];
        if (p == rt || p == a) break;
        par[a] = rt;
        a = p;
    }
    return rt;
}

__device__ __forceinline__ void sunion(int *par, int a, int b, int cap, int *status) {
    for (int it = 0; it <= 2 * cap + 2; it++) {
        a = sfind(par, a, cap, status);
        b = sfind(par, b, cap, status);
        if (a == b) return;
        if (a < b) {
            int t = a;
            a = b;
            b = t;
        }
        int old = atomicMin(&par[a], b);
        if (old == a) return;
        a = old;
    }
    atomicOr(status, SX_ST_LOOP);
}

// the 64-bit fixed-scale flux is usable for this object
__device__ __forceinline__ bool dl_range_ok(float fdpeak, int e0, int P) {
    return fexpo(fdpeak) - e0 + 24 + (32 - __clz(P)) <= 63;
}

// flux of a branch: the exact fixed-scale sum rounded to double, then to
// float, as the 128-bit path rounds it
__device__ __forceinline__ float dl_flux(unsigned long long acc, int e0) {
    return (float)scalbn(__ull2double_rn(acc), e0 - 23);
}

__device__ __forceinline__ unsigned long long dl_term(float c, int e0) {
    unsigned u = __float_as_uint(c);
    int sh = (int)((u >> 23) & 0xff) - 127 - e0;
    return (unsigned long long)((u & 0x7fffffu) | 0x800000u) << sh;
}

// pixels first active at level L (their parents point at themselves since
// before the sweep): join each to its active neighbours
template <int NT>
__device__ __forceinline__ void dl_activate_union(const DebArgs &A, int off, int ucap, int L, int b0, int b1,
                                                  const unsigned short *order, int *par, const unsigned char *lev,
                                                  int *status) {
    for (int i = b0 + (int)threadIdx.x; i < b1; i += NT) {
        const int e = order[i];
        const int p = (int)A.rpix[off + e];
        const int y = (int)fdiv((unsigned)p, A.wdiv), x = p - y * A.w;
        // the eight neighbour lookups are independent: issue them together
        int nb[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int ddx[8] = {-1, 0, 1, -1, 1, -1, 0, 1}, ddy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
            const int nx = x + ddx[q], ny = y + ddy[q];
            nb[q] = (nx < 0 || ny < 0 || nx >= A.w || ny >= A.h) ? -1 : __ldg(A.pos2idx + (size_t)ny * A.w + nx);
        }
        bool act[8];
#pragma unroll
        for (int q = 0; q < 8; q++) act[q] = nb[q] >= 0 && lev[nb[q] - off] >= L;
#pragma unroll
        for (int q = 0; q < 8; q++)
            if (act[q]) sunion(par, e, nb[q] - off, ucap, status);
    }
    __syncthreads();
}

// deblending level of a filtered value: the highest L with c >= thr[L]
__device__ __forceinline__ int dl_level_of(float c, const float *thr, int N) {
    int lo = 0, hi = N - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (c >= thr[mid])
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// An object whose filtered values have a single local maximum (one pixel
// with no 8-neighbour in the object strictly above it) cannot be split:
// every superlevel set of it is connected, because each component of one
// holds a pixel with no neighbour above it (its maximum: neighbours inside
// the component are not above it, neighbours outside it are below the level
// or, being adjacent, would belong to it).  The sweep's result for such an
// object is the whole object, kept at level 0.  Neighbours in the object are
// those with a root-list index (pixels of two roots are never adjacent).
template <int NT>
__device__ __forceinline__ bool dl_single_peak(const DebArgs &A, int P, const unsigned *pix, int *s_cnt) {
    if (threadIdx.x == 0) *s_cnt = 0;
    __syncthreads();
    int n = 0;
    for (int k = threadIdx.x; k < P; k += NT) {
        const int p = (int)pix[k];
        const int y = (int)fdiv((unsigned)p, A.wdiv), x = p - y * A.w;
        const float c = A.cd[p];
        bool top = true;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int ddx[8] = {-1, 0, 1, -1, 1, -1, 0, 1}, ddy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
            const int nx = x + ddx[q], ny = y + ddy[q];
            if (nx >= 0 && ny >= 0 && nx < A.w && ny < A.h) {
                const size_t np = (size_t)ny * A.w + nx;
                if (__ldg(A.pos2idx + np) >= 0 && __ldg(A.cd + np) > c) top = false;
            }
        }
        n += top;
    }
    n = __reduce_add_sync(0xffffffffu, n);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(s_cnt, n);
    __syncthreads();
    return *s_cnt == 1;
}

// levels, level counts, level order (highest level first); cdv holds the
// filtered values of the elements, and every element's merge record starts
// as "active from its level, not absorbed"
template <int NT>
__device__ __forceinline__ void dl_levels(const DebArgs &A, int P, const float *cdv, const float *thr,
                                          unsigned char *lev, unsigned short *order, int *lvcnt, int *lvstart,
                                          int *lvcur, int *rec, bool count_levpix) {
    for (int i = threadIdx.x; i <= A.N; i += NT) {
        lvcnt[i] = 0;
        if (i < DB_MAXLEV) lvcur[i] = 0;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < P; k += NT) {
        const int lo = dl_level_of(cdv[k], thr, A.N);
        lev[k] = (unsigned char)lo;
        rec[k] = (lo << 24) | 0x00ffffff;
        atomicAdd(&lvcnt[lo], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        unsigned long long lp = 0;
        for (int L = A.N - 1; L >= 0; L--) {
            lvstart[L] = s;
            s += lvcnt[L];
            lp += (unsigned long long)L * lvcnt[L];
        }
        if (count_levpix) atomicAdd(&A.sc->levpix, lp);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < P; k += NT) {
        int L = lev[k];
        order[lvstart[L] + atomicAdd(&lvcur[L], 1)] = (unsigned short)k;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// sweep: branch tree, MINCONT cut, kept branches
// ---------------------------------------------------------------------------
// hyb: for an arena object, shared memory holding its union-find parents
// (4 B per pixel) and levels (1 B per pixel), or null
template <int NT>
__device__ __forceinline__ void dl_sweep_root(const DebArgs &A, const int r, unsigned char *base, int cap,
                                              int *glist, int *gcount, unsigned char *hyb) {
    __shared__ float thr[DB_MAXLEV];
    __shared__ int lvcnt[DB_MAXLEV + 1], lvstart[DB_MAXLEV + 1], lvcur[DB_MAXLEV];
    __shared__ int s_nrl[2], s_nn[2], s_nkept, s_npeak;
    __shared__ unsigned s_peak;
    __shared__ XSum s_part[NT / 32];
    __shared__ float s_fdflux;
    const int tid = threadIdx.x;
    const int off = A.R.off[r], P = A.R.size[r];
    const unsigned *pix = A.rpix + off;
    if (!base) {  // global-memory arena: 48 B per element at the root's offset
        base = A.D.arena + (size_t)off * DL_ARENA_BYTES;
        cap = P;
    }
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(base);
    int *par = reinterpret_cast<int *>(acc + cap);
    int *sz = par + cap;
    // two-level arrays: level slot s of X is X0 + s * cap (arithmetic, so
    // that no pointer table lands in local memory)
    int *const nds0 = sz + cap;
    unsigned *const nfl0 = reinterpret_cast<unsigned *>(sz + 3 * cap);
    unsigned short *const order = reinterpret_cast<unsigned short *>(sz + 5 * cap);
    unsigned short *const rl0 = order + cap;
    unsigned short *const nid = order + 3 * cap;
    unsigned short *const ndr0 = order + 4 * cap;
    unsigned char *lev = reinterpret_cast<unsigned char *>(order + 6 * cap);
    if (hyb) {
        par = reinterpret_cast<int *>(hyb);
        lev = hyb + 4 * (size_t)P;
    }
#define NDS(s) (nds0 + (s) * cap)
#define NFL(s) (nfl0 + (s) * cap)
#define RL(s) (rl0 + (s) * cap)
#define NDR(s) (ndr0 + (s) * cap)
    unsigned long long *kept = A.D.kept + off;
    // merge record of every element: (activation level << 24) |
    // (level at which it stopped being a root, 0xff if never << 16) | the root
    // that absorbed it; the assignment walks these instead of replaying
    int *rec = A.D.rec + off;
    const int e0 = A.sc->e0cd;
    int *status = &A.sc->status;
    // walk cap of the union-find: the object's size (no walk is longer), or
    // a smaller cap set for a failure test
    const int ucap = A.loop_cap > 0 ? min(P, A.loop_cap) : P;

    // fdpeak, exact fdflux, completion keys (as k_deblend_sweep)
    if (tid == 0) {
        s_peak = 0u;
        s_nkept = 0;
        s_nrl[0] = s_nrl[1] = s_nn[0] = s_nn[1] = 0;
    }
    __syncthreads();
    XSum xs;
    xs_init(xs);
    unsigned pk = 0u;
    // every element's parent, size and flux term as the component it starts
    // when it becomes active (nothing reads or links them before), and its
    // filtered value for the levels, kept in the branch-count area until the
    // sweep needs it
    float *const cdv = reinterpret_cast<float *>(nds0);
    for (int k = tid; k < P; k += NT) {
        float c = A.cd[pix[k]];
        xs_add(xs, c);
        pk = max(pk, f2ord(c));
        par[k] = k;
        sz[k] = 1;
        acc[k] = dl_term(c, e0);
        cdv[k] = c;
    }
    xs = xs_warp_sum(xs);
    if ((tid & 31) == 0) s_part[tid >> 5] = xs;
    atomicMax(&s_peak, pk);
    {
        const int ymax = (int)fdiv(pix[P - 1], A.wdiv);
        for (int k = tid; k < P; k += NT) {
            const int y = (int)fdiv(pix[k], A.wdiv);
            if (y == ymax && (k == 0 || (int)fdiv(pix[k - 1], A.wdiv) < ymax)) {
                A.R.ymax[r] = ymax;
                A.R.lastx[r] = (int)pix[k] - ymax * A.w;
            }
        }
    }
    __syncthreads();
    if (tid == 0) {
        XSum t = s_part[0];
        for (int k = 1; k < NT / 32; k++) xs_merge(t, s_part[k]);
        if (t.ovf) atomicOr(status, SX_ST_RANGE);
        s_fdflux = xs_float(t);
        A.R.fdflux[r] = s_fdflux;
        A.R.fdpeak[r] = ord2f(s_peak);
        A.R.first[r] = (int)pix[0];
    }
    __syncthreads();
    const float fdpeak = ord2f(s_peak);
    if (!dl_range_ok(fdpeak, e0, P)) {
        if (tid == 0) glist[atomicAdd(gcount, 1)] = r;
        return;
    }
    const double value0 = (double)s_fdflux * A.mincont;
    block_thresholds(A, A.R.dthresh[r], fdpeak, thr);
    __syncthreads();
    if (dl_single_peak<NT>(A, P, pix, &s_npeak)) {
        // no split possible: the levels only count towards the summary
        unsigned ls = 0;
        for (int k = tid; k < P; k += NT) ls += (unsigned)dl_level_of(cdv[k], thr, A.N);
        ls = __reduce_add_sync(0xffffffffu, ls);
        if ((tid & 31) == 0 && ls) atomicAdd(&A.sc->levpix, (unsigned long long)ls);
        if (tid == 0) {
            kept[0] = 0ull;
            A.R.nkept[r] = 1;
        }
        return;
    }
    dl_levels<NT>(A, P, cdv, thr, lev, order, lvcnt, lvstart, lvcur, rec, true);
    int cur = 0, lastL = -1;
    for (int L = A.N - 1; L >= 0; L--) {
        const int cnt = lvcnt[L];
        if (cnt == 0) continue;
        const int prv = cur ^ 1, cl = L + 1;
        const int b0 = lvstart[L], b1 = b0 + cnt;
        const int nold = lastL >= 0 ? s_nrl[prv] : 0;
        const int nprev = lastL >= 0 ? s_nn[prv] : 0;
        // (a) the children re-flagged at level L+1 when the levels since the
        // last populated one were empty (the new pixels' sizes, flux terms and
        // records were set before the sweep)
        if (lastL > cl)
            for (int i = tid; i < nprev; i += NT) {
                const int c = NDR(prv)[i];
                const float lhs = dl_flux(acc[c], e0) - thr[cl] * (float)(unsigned)sz[c];
                NFL(prv)[i] = (NFL(prv)[i] & ~1u) | (lhs > value0 ? 1u : 0u);
            }
        // (b) activation and unions
        dl_activate_union<NT>(A, off, ucap, L, b0, b1, order, par, lev, status);
        // (c) roots that joined another component hand over size and flux
        for (int i = tid; i < nold + cnt; i += NT) {
            const int c = i < nold ? RL(prv)[i] : order[b0 + i - nold];
            if (par[c] != c) {
                const int rt = sfind_c(par, c, ucap, status);
                atomicAdd(&sz[rt], sz[c]);
                atomicAdd(&acc[rt], acc[c]);
                rec[c] = (lev[c] << 24) | (L << 16) | rt;  // absorbed at level L by rt
            } else {
                RL(cur)[atomicAdd(&s_nrl[cur], 1)] = (unsigned short)c;
            }
        }
        __syncthreads();
        // (d) this level's branches
        const int nr = s_nrl[cur];
        for (int i = tid; i < nr; i += NT) {
            const int c = RL(cur)[i], s = sz[c];
            if (s >= A.debminarea) {
                const int k = atomicAdd(&s_nn[cur], 1);
                NDR(cur)[k] = (unsigned short)c;
                nid[c] = (unsigned short)k;
                const float lhs = dl_flux(acc[c], e0) - thr[L] * (float)(unsigned)s;
                NFL(cur)[k] = (lhs > value0 ? 1u : 0u) | 2u;
                NDS(cur)[k] = 0;
            }
        }
        __syncthreads();
        // (e) children report to their parent
        for (int i = tid; i < nprev; i += NT) {
            const int p = nid[sfind_c(par, NDR(prv)[i], ucap, status)];
            const unsigned f = NFL(prv)[i];
            NDS(prv)[i] = p;
            if (f & 1u) atomicAdd(&NDS(cur)[p], 1);
            if (!(f & 4u)) atomicAnd(&NFL(cur)[p], ~2u);
        }
        __syncthreads();
        // (f) cut decisions for the children; (g) ok-after for this level
        for (int i = tid; i < nprev; i += NT) {
            const unsigned f = NFL(prv)[i];
            if ((f & 5u) == 5u && NDS(cur)[NDS(prv)[i]] > 1) {
                const int k = atomicAdd(&s_nkept, 1);
                kept[k] = ((unsigned long long)cl << 32) | NDR(prv)[i];
            }
        }
        const int ncur = s_nn[cur];
        for (int i = tid; i < ncur; i += NT) {
            const unsigned f = NFL(cur)[i];
            if ((f & 2u) && NDS(cur)[i] <= 1) NFL(cur)[i] = f | 4u;
        }
        if (tid == 0) {
            s_nrl[prv] = 0;
            s_nn[prv] = 0;
        }
        __syncthreads();
        lastL = L;
        cur = prv;
    }
    // level 0: the whole object is one branch
    const int fin = cur ^ 1;
    if (tid == 0) {
        int nk = s_nkept;
        for (int i = 0; i < s_nn[fin]; i++)
            if (NFL(fin)[i] & 4u) kept[nk++] = (unsigned long long)NDR(fin)[i];
        A.R.nkept[r] = nk;
    }
#undef NDS
#undef NFL
#undef RL
#undef NDR
}

// ---------------------------------------------------------------------------
// assignment: ownership of the kept branches, their preanalysis, gatherup
// ---------------------------------------------------------------------------
// gtab: shared memory for the centres and shapes of up to gcap kept
// branches (32 B each), staged for the gatherup; null when the kernel has none
template <int NT>
__device__ __forceinline__ void dl_assign_root(const DebArgs &A, const int r, unsigned char *base, int cap,
                                               unsigned char *gtab, int gcap) {
    __shared__ float thr[DB_MAXLEV];
    const int tid = threadIdx.x, lane = tid & 31;
    const int off = A.R.off[r], P = A.R.size[r];
    const float fdpeak = A.R.fdpeak[r];
    const int e0 = A.sc->e0cd;
    if (!dl_range_ok(fdpeak, e0, P)) return;  // done by the global kernels
    const int K = A.R.nkept[r], ob = A.R.objbase[r];
    const unsigned *pix = A.rpix + off;
    const unsigned long long *kept = A.D.kept + off;
    const int *rec = A.D.rec + off;
    if (!base) {
        base = A.D.arena + (size_t)off * DL_ARENA_BYTES;
        cap = P;
    }
    unsigned long long *kept2 = reinterpret_cast<unsigned long long *>(base);
    int *bcnt = reinterpret_cast<int *>(kept2 + cap), *bstart = bcnt + cap, *bcur = bstart + cap;
    unsigned short *blist = reinterpret_cast<unsigned short *>(bcur + cap);
    short *own = reinterpret_cast<short *>(blist + cap);
    unsigned short *kidx = reinterpret_cast<unsigned short *>(own + cap);
    unsigned char *kl = reinterpret_cast<unsigned char *>(kidx + cap);
    int *status = &A.sc->status;

    // one kept branch that is the whole object at level 0 (nothing split
    // off): every pixel is its own, in list order; of the thresholds only
    // the lowest (the object's own) is used
    const bool whole = K == 1 && (kept[0] >> 32) == 0;
    if (!whole) block_thresholds(A, A.R.dthresh[r], fdpeak, thr);
    if (whole) {
        if (tid == 0) {
            thr[0] = A.R.dthresh[r];
            kept2[0] = kept[0];
            bcnt[0] = P;
            bstart[0] = 0;
        }
        __syncthreads();
    } else {
        for (int k = tid; k < P; k += NT) kl[k] = 0xff;
        for (int k = tid; k < K; k += NT) bcnt[k] = bcur[k] = 0;
        __syncthreads();
        // kept list in (level, element) order
        for (int i = tid; i < K; i += NT) {
            const unsigned long long key = kept[i];
            int rank = 0;
            for (int j = 0; j < K; j++) rank += kept[j] < key;
            kept2[rank] = key;
        }
        __syncthreads();
        for (int i = tid; i < K; i += NT) {
            const unsigned long long key = kept2[i];
            kl[(int)(key & 0xffffffffu)] = (unsigned char)(key >> 32);
            kidx[(int)(key & 0xffffffffu)] = (unsigned short)i;
        }
        __syncthreads();
        // Owner of each pixel: its component at level L is the node of its
        // merge chain e -> up(e) -> ... that covers L (node x covers the levels
        // above the one at which it was absorbed, down from where the previous
        // node was absorbed); a kept branch (L, c) owns the pixel when c covers
        // L on the chain.  Absorption levels fall strictly along a chain.
        for (int e = tid; e < P; e += NT) {
            int x = e, hi = rec[e] >> 24, o = -1;
            for (int step = 0; step <= DB_MAXLEV + 1; step++) {
                const int rx = rec[x], m = (rx >> 16) & 0xff;
                const int lo = m == 0xff ? -1 : m;
                const int kx = kl[x];
                if (kx != 0xff && kx > lo && kx <= hi) {
                    o = kidx[x];
                    break;
                }
                if (m == 0xff) break;
                if (step == DB_MAXLEV + 1) atomicOr(status, SX_ST_LOOP);
                hi = lo;
                x = rx & 0xffff;
            }
            own[e] = (short)o;
            if (o >= 0) atomicAdd(&bcnt[o], 1);
        }
        __syncthreads();
        if (tid == 0) {
            int s = 0;
            for (int k = 0; k < K; k++) {
                bstart[k] = s;
                s += bcnt[k];
            }
        }
        __syncthreads();
        for (int e = tid; e < P; e += NT) {
            const int k = own[e];
            if (k >= 0) blist[bstart[k] + atomicAdd(&bcur[k], 1)] = (unsigned short)e;
        }
        __syncthreads();
    }
    // preanalysis of each kept branch over its own pixels, one warp per branch
    for (int k = tid >> 5; k < K; k += NT / 32) {
        const int o = ob + k, L = (int)(kept2[k] >> 32), nb = bcnt[k], bb = bstart[k];
        int xmin = 0x7fffffff, xmax = -1, ymin = 0x7fffffff, ymax = -1;
        unsigned pk = 0u, cpk = 0u;
        // exact sums in double bins (hint: the raw object's filtered peak),
        // or with XSum when a term falls outside them or the branch is large
        const bool binned = nb <= BS_MAX_TERMS;
        bool ok = binned;
        BinSum brv;
        bs_init(brv);
        const int top_c = bs_order(fdpeak);
        for (int i = lane; i < nb; i += 32) {
            const unsigned p = pix[whole ? i : blist[bb + i]];
            const int y = (int)fdiv(p, A.wdiv), x = (int)p - y * A.w;
            xmin = min(xmin, x);
            xmax = max(xmax, x);
            ymin = min(ymin, y);
            ymax = max(ymax, y);
            pk = max(pk, f2ord(A.sub[p]));
            const float c = A.cd[p];
            cpk = max(cpk, f2ord(c));
            if (binned) ok &= bs_add(brv, c, top_c);
        }
        for (int d = 16; d > 0; d >>= 1) {
            xmin = min(xmin, __shfl_xor_sync(0xffffffffu, xmin, d));
            xmax = max(xmax, __shfl_xor_sync(0xffffffffu, xmax, d));
            ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, d));
            ymax = max(ymax, __shfl_xor_sync(0xffffffffu, ymax, d));
            pk = max(pk, __shfl_xor_sync(0xffffffffu, pk, d));
            cpk = max(cpk, __shfl_xor_sync(0xffffffffu, cpk, d));
        }
        XSum srv;
        if (__all_sync(0xffffffffu, ok)) {
            srv = bs_to_xsum(bs_warp_sum(brv));
        } else {
            xs_init(srv);
            for (int i = lane; i < nb; i += 32) xs_add(srv, A.cd[pix[whole ? i : blist[bb + i]]]);
            srv = xs_warp_sum(srv);
        }
        const float peak = ord2f(pk);
        const double dthresh = thr[L], dthresh2 = (dthresh + peak) / 2.0;
        // second pass: the moments' terms are below the filtered peak times
        // the box sides
        const int bx = 32 - __clz(xmax - xmin), by = 32 - __clz(ymax - ymin), tc = bs_order(ord2f(cpk)) + 1;
        const int tv_top = bs_order(peak);
        BinSum bmx, bmy, bmx2, bmy2, bmxy, btv;
        bs_init(bmx);
        bs_init(bmy);
        bs_init(bmx2);
        bs_init(bmy2);
        bs_init(bmxy);
        bs_init(btv);
        ok = binned;
        int dnpix = 0, area2 = 0;
        for (int i = lane; i < nb; i += 32) {
            const unsigned p = pix[whole ? i : blist[bb + i]];
            const int yy = (int)fdiv(p, A.wdiv), x = (int)p - yy * A.w - xmin, y = yy - ymin;
            const float cval = A.cd[p], val = A.sub[p];
            dnpix += val > dthresh;
            area2 += val > dthresh2;
            if (binned) {
                ok &= bs_add(bmx, cval * x, tc + bx);
                ok &= bs_add(bmy, cval * y, tc + by);
                ok &= bs_add(bmx2, cval * x * x, tc + 2 * bx);
                ok &= bs_add(bmy2, cval * y * y, tc + 2 * by);
                ok &= bs_add(bmxy, cval * x * y, tc + bx + by);
                ok &= bs_add(btv, val, tv_top);
            }
        }
        for (int d = 16; d > 0; d >>= 1) {
            dnpix += __shfl_xor_sync(0xffffffffu, dnpix, d);
            area2 += __shfl_xor_sync(0xffffffffu, area2, d);
        }
        XSum smx, smy, smx2, smy2, smxy, stv;
        if (__all_sync(0xffffffffu, ok)) {
            smx = bs_to_xsum(bs_warp_sum(bmx));
            smy = bs_to_xsum(bs_warp_sum(bmy));
            smx2 = bs_to_xsum(bs_warp_sum(bmx2));
            smy2 = bs_to_xsum(bs_warp_sum(bmy2));
            smxy = bs_to_xsum(bs_warp_sum(bmxy));
            stv = bs_to_xsum(bs_warp_sum(btv));
        } else {
            Moments6 m;
            moments_xsum(A.cd, A.sub, pix, whole ? nullptr : blist, bb, nb, A.wdiv, A.w, xmin, ymin, &m);
            smx = m.mx;
            smy = m.my;
            smx2 = m.mx2;
            smy2 = m.my2;
            smxy = m.mxy;
            stv = m.tv;
        }
        if (lane != 0) continue;
        if (srv.ovf | smx.ovf | smy.ovf | smx2.ovf | smy2.ovf | smxy.ovf | stv.ovf) atomicOr(status, SX_ST_RANGE);
        int flag = 0;
        if (L > 0) flag |= SX_OBJ_MERGED;
        if (xmin == 0 || xmax == A.w - 1 || ymin == 0 || ymax == A.h - 1) flag |= SX_OBJ_TRUNC;
        const float rv = xs_float(srv);
        const double rvd = rv;
        const double mx = xs_double(smx), my = xs_double(smy);
        const double mx2 = xs_double(smx2), my2 = xs_double(smy2), mxy = xs_double(smxy);
        const double xm = mx / rvd, ym = my / rvd;
        double xm2 = mx2 / rvd - xm * xm, ym2 = my2 / rvd - ym * ym, xym = mxy / rvd - xm * ym;
        double temp, temp2, theta, pmx2, pmy2, darea, t1t2;
        int singu = 0;
        if ((temp2 = xm2 * ym2 - xym * xym) < 0.00694) {
            xm2 += 0.0833333;
            ym2 += 0.0833333;
            temp2 = xm2 * ym2 - xym * xym;
            singu = 1;
        }
        if ((fabs(temp = xm2 - ym2)) > 0.0)
            theta = atan2(2.0 * xym, temp) / 2.0;
        else
            theta = SX_PI / 4.0;
        temp = sqrt(0.25 * temp * temp + xym * xym);
        pmy2 = pmx2 = 0.5 * (xm2 + ym2);
        pmx2 += temp;
        pmy2 -= temp;
        const float fa = (float)sqrt(pmx2), fb = (float)sqrt(pmy2);
        float abcor;
        darea = (double)area2 - dnpix;
        t1t2 = dthresh / dthresh2;
        if (t1t2 > 0.0) {
            abcor = (darea < 0.0 ? darea : -1.0) / (2 * SX_PI * log(t1t2 < 1.0 ? t1t2 : 0.99) * fa * fb);
            if (abcor > 1.0) abcor = 1.0;
        } else
            abcor = 1.0;
        A.O.root[o] = r;
        A.O.level[o] = L;
        A.O.node_dthresh[o] = thr[L];
        A.O.dthr[o] = A.R.dthresh[r];
        A.O.athr[o] = A.R.thresh[r];
        A.O.xmin[o] = xmin;
        A.O.xmax[o] = xmax;
        A.O.ymin[o] = ymin;
        A.O.ymax[o] = ymax;
        A.O.flags[o] = flag;
        A.O.singu[o] = singu;
        A.O.dnpix[o] = dnpix;
        A.O.fdflux[o] = rv;
        A.O.dflux[o] = xs_float(stv);
        A.O.fdpeak[o] = ord2f(cpk);
        A.O.dpeak[o] = peak;
        A.O.mx[o] = xm + xmin;
        A.O.my[o] = ym + ymin;
        A.O.mx2[o] = xm2;
        A.O.my2[o] = ym2;
        A.O.mxy[o] = xym;
        A.O.a[o] = fa;
        A.O.b[o] = fb;
        A.O.theta[o] = theta * 180.0 / SX_PI;
        A.O.cxx[o] = (float)(ym2 / temp2);
        A.O.cyy[o] = (float)(xm2 / temp2);
        A.O.cxy[o] = (float)(-2 * xym / temp2);
        A.O.abcor[o] = abcor;
        A.O.n[o] = bcnt[k];
    }
    __syncthreads();
    // the kept branches' centres and shapes in shared memory for the
    // gatherup, when there is room (the same values and types as the columns)
    const bool staged = gtab != nullptr && K <= gcap;
    double *gmx = reinterpret_cast<double *>(gtab), *gmy = gmx + gcap;
    float *gcxx = reinterpret_cast<float *>(gmy + gcap), *gcyy = gcxx + gcap, *gcxy = gcyy + gcap,
          *gabc = gcxy + gcap;
    if (staged && !whole) {
        for (int i = tid; i < K; i += NT) {
            gmx[i] = A.O.mx[ob + i];
            gmy[i] = A.O.my[ob + i];
            gcxx[i] = A.O.cxx[ob + i];
            gcyy[i] = A.O.cyy[ob + i];
            gcxy[i] = A.O.cxy[ob + i];
            gabc[i] = A.O.abcor[ob + i];
        }
        __syncthreads();
    }
    // gatherup (cudadeblend.cu:1262-1360): the nearest kept branch in the
    // elliptical metric, first in order on ties
    for (int e = tid; e < P; e += NT) {
        int k = whole ? 0 : own[e];
        const unsigned p = pix[e];
        if (k < 0) {
            const int y = (int)fdiv(p, A.wdiv), x = (int)p - y * A.w;
            int iclst = 0;
            float distmin = 1e+31f, dx, dy, dist;
            if (staged) {
                for (int i = 0; i < K; i++) {
                    dx = x - gmx[i];
                    dy = y - gmy[i];
                    dist = 0.5 * (gcxx[i] * dx * dx + gcyy[i] * dy * dy + gcxy[i] * dx * dy) / gabc[i];
                    if (dist < distmin) {
                        distmin = dist;
                        iclst = i;
                    }
                }
            } else {
                for (int i = 0; i < K; i++) {
                    const int o = ob + i;
                    dx = x - A.O.mx[o];
                    dy = y - A.O.my[o];
                    dist = 0.5 * (A.O.cxx[o] * dx * dx + A.O.cyy[o] * dy * dy + A.O.cxy[o] * dx * dy) / A.O.abcor[o];
                    if (dist < distmin) {
                        distmin = dist;
                        iclst = i;
                    }
                }
            }
            k = iclst;
            atomicAdd(&A.O.n[ob + k], 1);
        }
        A.alloc[p] = ob + k;
        A.objkey[off + e] = (unsigned)(ob + k);
    }
}

// Persistent CTAs: each takes the next root of its list from a device
// cursor until the list is exhausted, so the grid is sized to the resident
// capacity rather than to the (device-side) length of the list.
// cap > 0: per-object state in dynamic shared memory of cap elements;
// cap == 0: in the global arena
// Up to three lists of objects taken in order through one device cursor
// (the larger size classes first, so the longest objects start earliest).
struct RootLists {
    const int *list[3];
    const int *count[3];
};

__device__ __forceinline__ int rl_item(const RootLists &L, int c) {
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (!L.list[k]) return -1;
        const int n = *L.count[k];
        if (c < n) return L.list[k][c];
        c -= n;
    }
    return -1;
}

// cap > 0: per-object state in dynamic shared memory of cap elements;
// cap == 0: in the global arena, with the parents and levels of objects of
// at most hyb pixels in dynamic shared memory (5 * hyb bytes) when hyb > 0
template <int NT>
__global__ void __launch_bounds__(NT) k_dl_sweep(const __grid_constant__ DebArgs A, const RootLists L, int *cursor,
                                                 int cap, int *glist, int *gcount, int hyb) {
    extern __shared__ __align__(16) unsigned char dl_smem[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = rl_item(L, atomicAdd(cursor, 1));
        __syncthreads();
        const int r = s_item;
        __syncthreads();
        if (r < 0) break;
        unsigned char *h = (!cap && hyb > 0 && A.R.size[r] <= hyb) ? dl_smem : nullptr;
        dl_sweep_root<NT>(A, r, cap ? dl_smem : nullptr, cap, glist, gcount, h);
        __syncthreads();
    }
}

// at most 64 registers (32 one-warp, 16 two-warp, 4 eight-warp or one
// 32-warp CTAs per SM): the assignment waits on its chain walks and gathers,
// so residency pays more than the registers it costs.
// cap > 0: per-object state in dynamic shared memory of cap elements;
// cap == 0: in the global arena, with the gatherup's table of up to gcap
// kept branches in dynamic shared memory (DL_GTAB_BYTES each) when gcap > 0
template <int NT>
__global__ void __launch_bounds__(NT, NT == 32 ? 32 : NT == 64 ? 16 : NT == 256 ? 4 : 1)
    k_dl_assign(const __grid_constant__ DebArgs A, const RootLists L, int *cursor, int cap, int gcap) {
    extern __shared__ __align__(16) unsigned char dl_smem[];
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = rl_item(L, atomicAdd(cursor, 1));
        __syncthreads();
        const int r = s_item;
        __syncthreads();
        if (r < 0) break;
        dl_assign_root<NT>(A, r, cap ? dl_smem : nullptr, cap, (!cap && gcap > 0) ? dl_smem : nullptr, gcap);
        __syncthreads();
    }
}

// Size classes (list k at lists + k * n, n the number of roots or the
// capacity the launches were sized for; its length in counts[k]):
//   8  <= 64 pixels              shared memory, one warp
//   9  (64, 128]                 shared memory, one warp
//   0  (128, 256]                shared memory, one warp
//   1  (1024, 2048]   2 (256, 1024]       arena (hybrid), 64 threads
//   4  (4096, 8192]   5 (2048, 4096]      arena (hybrid), 256 threads
//   3  (8192, 32767]             arena (hybrid), 1024 threads
//   6  > 32767 pixels            128-bit global kernels
//   7  objects the compact sweeps hand over (flux range beyond 64 bits)
// Every list holds its objects largest first (a stable sort of the roots by
// size), so that the persistent grids start the longest objects first and
// end on short ones.  counts[DL_NLISTS + k] and counts[2 * DL_NLISTS + k]
// are the cursors of the sweep and the assignment kernel that takes list k
// first; counts[3 * DL_NLISTS ...] hold the class boundaries in sorted order.
constexpr int DL_NLISTS = 10;

__device__ __forceinline__ int dl_class(int s) {
    if (s <= DL_CAP1) return 8;
    if (s <= DL_CAP2) return 9;
    if (s <= DL_CAP0) return 0;
    if (s <= DL_MID) return s > DL_MID / 2 ? 1 : 2;
    if (s <= DL_ARENA_MAX) return s > 4 * DL_MID ? 3 : s > 2 * DL_MID ? 4 : 5;
    return 6;
}

// sort keys: larger objects first (sizes above 65535 tie, all in class 6)
__global__ void k_root_keys(const int *size, int n, const int *n_dev, unsigned *keys, unsigned *vals) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= sx_count(n, n_dev)) return;
    keys[r] = 65535u - (unsigned)min(size[r], 65535);
    vals[r] = (unsigned)r;
}

// first and last sorted position of every size class present
__global__ void k_class_bounds(const int *size, const unsigned *sorted, int n, const int *n_dev, int *bnd) {
    n = sx_count(n, n_dev);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int t = dl_class(size[sorted[i]]);
    if (i == 0 || dl_class(size[sorted[i - 1]]) != t) bnd[t] = i;
    if (i == n - 1 || dl_class(size[sorted[i + 1]]) != t) bnd[DL_NLISTS + t] = i;
}

__global__ void k_class_fill(const int *size, const unsigned *sorted, int n, const int *n_dev, const int *bnd,
                             int *lists, int *counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sx_count(n, n_dev)) return;
    const int t = dl_class(size[sorted[i]]);
    lists[(size_t)t * n + (i - bnd[t])] = (int)sorted[i];
    if (i == bnd[DL_NLISTS + t]) counts[t] = i - bnd[t] + 1;
}

// resident CTAs of a kernel on this device (cached per kernel and device; the
// first launch on a device also raises the kernel's dynamic shared memory
// limit to smem when that is above the default 48 KB)
template <typename K>
static int dl_grid(K kernel, int nt, size_t smem, DevCache &cache) {
    return sx_share(cache.get([&](int dev) {
        int nsm = 0, per = 0;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, nt, smem);
        return max(1, nsm) * max(1, per);
    }));
}

static RootLists dl_lists(const int *lists, int *counts, size_t n, int a, int b = -1, int c = -1) {
    RootLists L;
    const int k[3] = {a, b, c};
    for (int i = 0; i < 3; i++) {
        L.list[i] = k[i] >= 0 ? lists + (size_t)k[i] * n : nullptr;
        L.count[i] = k[i] >= 0 ? counts + k[i] : nullptr;
    }
    return L;
}

// keys, vals, kalt, valt: scratch of nroots elements each; tmp: sort scratch.
// nroots_dev (device, or null): the number of roots, at most nroots, when
// only the device knows it; nroots is then the capacity (the list stride).
void launch_deblend_split(const int *size, int nroots, const int *nroots_dev, int *lists, int *counts,
                          unsigned *keys, unsigned *vals, unsigned *kalt, unsigned *valt, int *tmp, cudaStream_t st) {
    cudaMemsetAsync(counts, 0, 3 * DL_NLISTS * sizeof(int), st);
    if (nroots <= 0) return;
    const unsigned g = (unsigned)((nroots + 255) / 256);
    k_root_keys<<<g, 256, 0, st>>>(size, nroots, nroots_dev, keys, vals);
    radix_sort_pairs(keys, vals, kalt, valt, nroots, 16, tmp, st, nroots_dev);
    k_class_bounds<<<g, 256, 0, st>>>(size, vals, nroots, nroots_dev, counts + 3 * DL_NLISTS);
    k_class_fill<<<g, 256, 0, st>>>(size, vals, nroots, nroots_dev, counts + 3 * DL_NLISTS, lists, counts);
}

int deblend_split_launches(int nroots) { return nroots > 0 ? 3 + radix_launches(16, nroots) : 0; }

static void dl_fork(const DebStreams &S) {
    cudaEventRecord(S.fork, S.main);
    for (int i = 0; i < DL_SIDE; i++) cudaStreamWaitEvent(S.side[i], S.fork, 0);
}

static void dl_join(const DebStreams &S) {
    for (int i = 0; i < DL_SIDE; i++) {
        cudaEventRecord(S.join[i], S.side[i]);
        cudaStreamWaitEvent(S.main, S.join[i], 0);
    }
}

#define DL_SCUR(k) (counts + DL_NLISTS + (k))
#define DL_ACUR(k) (counts + 2 * DL_NLISTS + (k))

// Three streams run the size classes side by side, placed by their measured
// times on a 4096 x 4096 frame of 35,000 raw objects: side stream 0 the
// 128-bit global class and classes 4-5, side stream 1 the largest objects
// (class 3), the main stream classes 1-2 and then the shared-memory classes
// (classes 1-2 after class 3 on side stream 1 measured slower: the classes
// compete for the same SMs, so the sum of their times counts more than the
// balance of the streams).  The objects handed over by the compact sweeps
// are swept last, after the join.
// hybrid tiers: largest object of each arena kernel (its parents and levels
// take 5 B per pixel of shared memory)
constexpr int DL_HYB3 = DL_ARENA_MAX;  // class 3: 1024-thread CTAs, about 160 KB
constexpr int DL_HYB45 = 4 * DL_MID;   // classes 4, 5: 256-thread CTAs, 40 KB
constexpr int DL_HYB12 = DL_MID;       // classes 1, 2: 64-thread CTAs, 10 KB
constexpr int DL_HYB_BYTES = 5;

void launch_deblend_sweep(const DebArgs &A, const int *lists, int *counts, int nroots, const DebStreams &S) {
    if (nroots <= 0) return;
    static DevCache g0, g1, g2, g3, g4, g5, g6;
    const size_t n = (size_t)nroots;
    int *glist = const_cast<int *>(lists) + 7 * n;
    const size_t m0 = DL_CAP0 * DL_SWEEP_BYTES, m1 = DL_CAP1 * DL_SWEEP_BYTES, m2 = DL_CAP2 * DL_SWEEP_BYTES;
    const size_t h3 = (size_t)DL_HYB3 * DL_HYB_BYTES, h45 = (size_t)DL_HYB45 * DL_HYB_BYTES,
                 h12 = (size_t)DL_HYB12 * DL_HYB_BYTES;
    dl_fork(S);
    const int grid3 = min(nroots, dl_grid(k_deblend_sweep, DB_THREADS, 0, g3));
    k_deblend_sweep<<<grid3, DB_THREADS, 0, S.side[0]>>>(A, lists + 6 * n, counts + 6, DL_SCUR(6));
    k_dl_sweep<256><<<min(nroots, dl_grid(k_dl_sweep<256>, 256, h45, g2)), 256, h45, S.side[0]>>>(
        A, dl_lists(lists, counts, n, 4, 5), DL_SCUR(4), 0, glist, counts + 7, DL_HYB45);
    k_dl_sweep<1024><<<min(nroots, dl_grid(k_dl_sweep<1024>, 1024, h3, g5)), 1024, h3, S.side[1]>>>(
        A, dl_lists(lists, counts, n, 3), DL_SCUR(3), 0, glist, counts + 7, DL_HYB3);
    k_dl_sweep<64><<<min(nroots, dl_grid(k_dl_sweep<64>, 64, h12, g1)), 64, h12, S.main>>>(
        A, dl_lists(lists, counts, n, 1, 2), DL_SCUR(1), 0, glist, counts + 7, DL_HYB12);
    k_dl_sweep<32><<<min(nroots, dl_grid(k_dl_sweep<32>, 32, m0, g0)), 32, m0, S.main>>>(
        A, dl_lists(lists, counts, n, 0), DL_SCUR(0), DL_CAP0, glist, counts + 7, 0);
    k_dl_sweep<32><<<min(nroots, dl_grid(k_dl_sweep<32>, 32, m2, g6)), 32, m2, S.main>>>(
        A, dl_lists(lists, counts, n, 9), DL_SCUR(9), DL_CAP2, glist, counts + 7, 0);
    k_dl_sweep<32><<<min(nroots, dl_grid(k_dl_sweep<32>, 32, m1, g4)), 32, m1, S.main>>>(
        A, dl_lists(lists, counts, n, 8), DL_SCUR(8), DL_CAP1, glist, counts + 7, 0);
    dl_join(S);
    k_deblend_sweep<<<grid3, DB_THREADS, 0, S.main>>>(A, glist, counts + 7, DL_SCUR(7));
}

// kept branches whose centres and shapes the gatherup stages in shared
// memory (more go through global memory)
constexpr int DL_GTAB_BYTES = 32;
constexpr int DL_GTAB_BIG = 1024;  // classes 3, 4, 5: 32 KB
constexpr int DL_GTAB_MID = 128;   // classes 1, 2: 4 KB

void launch_deblend_assign(const DebArgs &A, const int *lists, int *counts, int nroots, const DebStreams &S) {
    if (nroots <= 0) return;
    static DevCache g0, g1, g2, g3, g4, g5, g6;
    const size_t n = (size_t)nroots;
    const size_t m0 = DL_CAP0 * DL_ASSIGN_BYTES, m1 = DL_CAP1 * DL_ASSIGN_BYTES, m2 = DL_CAP2 * DL_ASSIGN_BYTES;
    const size_t tb = (size_t)DL_GTAB_BIG * DL_GTAB_BYTES, tm = (size_t)DL_GTAB_MID * DL_GTAB_BYTES;
    dl_fork(S);
    const int grid3 = min(nroots, dl_grid(k_deblend_assign, DB_THREADS, 0, g3));
    k_deblend_assign<<<grid3, DB_THREADS, 0, S.side[0]>>>(A, lists + 6 * n, counts + 6, DL_ACUR(6));
    k_deblend_assign<<<grid3, DB_THREADS, 0, S.side[0]>>>(A, lists + 7 * n, counts + 7, DL_ACUR(7));
    k_dl_assign<256><<<min(nroots, dl_grid(k_dl_assign<256>, 256, tb, g2)), 256, tb, S.side[0]>>>(
        A, dl_lists(lists, counts, n, 4, 5), DL_ACUR(4), 0, DL_GTAB_BIG);
    k_dl_assign<1024><<<min(nroots, dl_grid(k_dl_assign<1024>, 1024, tb, g5)), 1024, tb, S.side[1]>>>(
        A, dl_lists(lists, counts, n, 3), DL_ACUR(3), 0, DL_GTAB_BIG);
    k_dl_assign<64><<<min(nroots, dl_grid(k_dl_assign<64>, 64, tm, g1)), 64, tm, S.main>>>(
        A, dl_lists(lists, counts, n, 1, 2), DL_ACUR(1), 0, DL_GTAB_MID);
    k_dl_assign<32><<<min(nroots, dl_grid(k_dl_assign<32>, 32, m0, g0)), 32, m0, S.main>>>(
        A, dl_lists(lists, counts, n, 0), DL_ACUR(0), DL_CAP0, 0);
    k_dl_assign<32><<<min(nroots, dl_grid(k_dl_assign<32>, 32, m2, g6)), 32, m2, S.main>>>(
        A, dl_lists(lists, counts, n, 9), DL_ACUR(9), DL_CAP2, 0);
    k_dl_assign<32><<<min(nroots, dl_grid(k_dl_assign<32>, 32, m1, g4)), 32, m1, S.main>>>(
        A, dl_lists(lists, counts, n, 8), DL_ACUR(8), DL_CAP1, 0);
    dl_join(S);
}

}  // namespace sx
