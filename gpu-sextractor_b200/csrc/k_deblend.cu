// k_deblend.cu -- multi-threshold deblending of every raw object.
//
// Reference: src/cuda/cudadeblend.cu:199-217 (thresholds), :579-727 (one
// global CCL per sub-threshold level with host synchronisation), :1425-1776
// (cut_branch: MINCONT pruning, level by level with count read-backs),
// :1262-1360 (gatherup), src/cuda/cudaanalyse.cu:1686-1903 (preanalysis of the
// kept branches).
//
// Here one CTA owns one raw object.  It sweeps the N-1 thresholds from the
// highest down with an incremental union-find over the object's pixel list:
// at level L the pixels whose filtered value first passes t_L are activated
// and joined to their active 8-neighbours, and the components with at least
// deb_minarea pixels are that level's branches.  Branch sizes and exact flux
// sums are carried at the union-find roots and merged when components join.
// The pruning rule of decidePrune1/2 only couples a level with the one above,
// so it is evaluated during the same sweep; the kept branches come out
// directly.  A second sweep assigns the pixels of each kept branch, then the
// branches are pre-analysed and the remaining pixels gathered up.
#include "common.cuh"
#include "kernels.cuh"

namespace sx {

constexpr int DB_THREADS = 256;
constexpr int DB_MAXLEV = 64;

__device__ __forceinline__ int lfind(const int *par, int a) {
    for (int n = 0; n < (1 << 26); n++) {
        int p = par[a];
        if (p == a) break;
        a = p;
    }
    return a;
}

__device__ __forceinline__ void lunion(int *par, int a, int b, int *status) {
    for (int it = 0; it < (1 << 20); it++) {
        a = lfind(par, a);
        b = lfind(par, b);
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



// the raw object's detection threshold d0 (its pixels' smallest) and the
// N-1 thresholds above it (src/cuda/cudadeblend.cu:199-217)
__device__ __forceinline__ void block_thresholds(const DebArgs &A, float d0, float fdpeak, float *thr) {
    for (int i = threadIdx.x; i < A.N; i += blockDim.x) {
        if (i == 0)
            thr[0] = d0;
        else {
            double dt0 = d0, dp = fdpeak;
            thr[i] = dt0 * pow(dp / dt0, (double)i / A.N);
        }
    }
}

// activation + unions of the pixels first active at level L
__device__ __forceinline__ void activate_and_union(const DebArgs &A, int off, int L, int b0, int b1,
                                                   const int *order, int *par, const int *lev) {
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        int e = order[i];
        par[e] = e;
    }
    __syncthreads();
    for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        int e = order[i];
        int p = (int)A.rpix[off + e];
        int x = p % A.w, y = p / A.w;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const int ddx[8] = {-1, 0, 1, -1, 1, -1, 0, 1}, ddy[8] = {-1, -1, -1, 0, 0, 1, 1, 1};
            int nx = x + ddx[q], ny = y + ddy[q];
            if (nx < 0 || ny < 0 || nx >= A.w || ny >= A.h) continue;
            int j = A.pos2idx[(size_t)ny * A.w + nx];
            if (j < 0) continue;
            int qi = j - off;
            if (lev[qi] >= L) lunion(par, e, qi, &A.sc->status);
        }
    }
    __syncthreads();
}

// first sweep: branch tree, MINCONT pruning, kept branches
__device__ __forceinline__ void deblend_sweep_root(const DebArgs &A, const int r) {
    __shared__ float thr[DB_MAXLEV];
    __shared__ int lvcnt[DB_MAXLEV + 1], lvstart[DB_MAXLEV + 1], lvcur[DB_MAXLEV];
    __shared__ int s_nrl[2], s_nn[2], s_nkept;
    __shared__ unsigned s_peak;
    __shared__ XSum s_part[DB_THREADS / 32];
    __shared__ float s_fdflux;
    const int off = A.R.off[r], P = A.R.size[r];
    const unsigned *pix = A.rpix + off;
    int *par = A.D.par + off, *lev = A.D.lev + off, *sz = A.D.sz + off, *order = A.D.order + off;
    unsigned long long *acc = A.D.acc + (size_t)off * 4;
    int *rl[2] = {A.D.rl0 + off, A.D.rl1 + off};
    int *nid[2] = {A.D.nid0 + off, A.D.nid1 + off};
    int *ndr[2] = {A.D.nd_root0 + off, A.D.nd_root1 + off};
    int *ndf[2] = {A.D.nd_flag0 + off, A.D.nd_flag1 + off};
    int *nds[2] = {A.D.nd_nson0 + off, A.D.nd_nson1 + off};
    int *ndc[2] = {A.D.nd_okc0 + off, A.D.nd_okc1 + off};
    int *nda[2] = {A.D.nd_oka0 + off, A.D.nd_oka1 + off};
    unsigned long long *kept = A.D.kept + off;
    const int e0 = A.sc->e0cd;
    int *status = &A.sc->status;

    // fdpeak, exact fdflux, completion keys
    if (threadIdx.x == 0) {
        s_peak = 0u;
        s_nkept = 0;
        s_nrl[0] = s_nrl[1] = s_nn[0] = s_nn[1] = 0;
    }
    for (int i = threadIdx.x; i <= A.N; i += blockDim.x) {
        lvcnt[i] = 0;
        if (i < DB_MAXLEV) lvcur[i] = 0;
    }
    __syncthreads();
    XSum xs;
    xs_init(xs);
    unsigned pk = 0u;
    for (int k = threadIdx.x; k < P; k += blockDim.x) {
        float c = A.cd[pix[k]];
        xs_add(xs, c);
        pk = max(pk, f2ord(c));
    }
    xs = xs_warp_reduce(xs);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = xs;
    atomicMax(&s_peak, pk);
    {
        int ymax = (int)(pix[P - 1] / A.w);
        for (int k = threadIdx.x; k < P; k += blockDim.x)
            if ((int)(pix[k] / A.w) == ymax && (k == 0 || (int)(pix[k - 1] / A.w) < ymax)) {
                A.R.ymax[r] = ymax;
                A.R.lastx[r] = (int)(pix[k] % A.w);
            }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        XSum t = s_part[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) xs_merge(t, s_part[k]);
        if (t.ovf) atomicOr(status, SX_ST_RANGE);
        s_fdflux = xs_float(t);
        A.R.fdflux[r] = s_fdflux;
        A.R.fdpeak[r] = ord2f(s_peak);
        A.R.first[r] = (int)pix[0];
    }
    __syncthreads();
    const float fdpeak = ord2f(s_peak);
    const double value0 = (double)s_fdflux * A.mincont;
    block_thresholds(A, A.R.dthresh[r], fdpeak, thr);
    __syncthreads();
    // level of every pixel: largest i with cd >= thr[i]
    for (int k = threadIdx.x; k < P; k += blockDim.x) {
        float c = A.cd[pix[k]];
        int lo = 0, hi = A.N - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (c >= thr[mid])
                lo = mid;
            else
                hi = mid - 1;
        }
        lev[k] = lo;
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
        atomicAdd(&A.sc->levpix, lp);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < P; k += blockDim.x) {
        int L = lev[k];
        order[lvstart[L] + atomicAdd(&lvcur[L], 1)] = k;
    }
    __syncthreads();

    int cur = 0;
    for (int L = A.N - 1; L >= 0; L--) {
        const int prv = cur ^ 1;
        const int b0 = lvstart[L], b1 = lvstart[L] + lvcnt[L];
        // (a)+(b) activation and unions
        for (int i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
            int e = order[i];
            sz[e] = 1;
            unsigned int lim[4];
            bool neg;
            int bad = 0;
            limbs_term(A.cd[pix[e]], e0, lim, neg, bad);
            if (bad) atomicOr(status, SX_ST_RANGE);
#pragma unroll
            for (int q = 0; q < 4; q++) acc[(size_t)e * 4 + q] = lim[q];
        }
        activate_and_union(A, off, L, b0, b1, order, par, lev);
        // (c) roots that joined another component hand over their size and sum
        const int nold = s_nrl[prv];
        for (int i = threadIdx.x; i < nold + (b1 - b0); i += blockDim.x) {
            int c = i < nold ? rl[prv][i] : order[b0 + i - nold];
            if (par[c] != c) {
                int rt = lfind(par, c);
                atomicAdd(&sz[rt], sz[c]);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    unsigned long long v = acc[(size_t)c * 4 + q];
                    if (v) atomicAdd(&acc[(size_t)rt * 4 + q], v);
                }
            } else {
                rl[cur][atomicAdd(&s_nrl[cur], 1)] = c;
            }
        }
        __syncthreads();
        // (d) this level's branches
        const int nr = s_nrl[cur];
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            int c = rl[cur][i];
            int s = sz[c];
            if (s >= A.debminarea) {
                int k = atomicAdd(&s_nn[cur], 1);
                ndr[cur][k] = c;
                nid[cur][c] = k;
                XSum t = limbs_to_xsum(acc + (size_t)c * 4, e0);
                float fdflux = xs_float(t);
                float lhs = fdflux - thr[L] * (float)(unsigned)s;
                ndf[cur][k] = (lhs > value0) ? 1 : 0;
                nds[cur][k] = 0;
                ndc[cur][k] = 1;
            }
        }
        __syncthreads();
        // (e) children of the level above report to their parent
        const int nprev = (L < A.N - 1) ? s_nn[prv] : 0;
        for (int i = threadIdx.x; i < nprev; i += blockDim.x) {
            int c = ndr[prv][i];
            int p = nid[cur][lfind(par, c)];
            nds[prv][i] = p;  // the child's nson slot is free now: keep its parent there
            if (ndf[prv][i]) atomicAdd(&nds[cur][p], 1);
            if (!nda[prv][i]) atomicAnd(&ndc[cur][p], 0);
        }
        __syncthreads();
        // (f) final decision for the level above; ok-after for this level
        for (int i = threadIdx.x; i < nprev; i += blockDim.x) {
            int p = nds[prv][i];
            if (nds[cur][p] > 1 && nda[prv][i] && ndf[prv][i]) {
                int k = atomicAdd(&s_nkept, 1);
                kept[k] = ((unsigned long long)(L + 1) << 32) | (unsigned)ndr[prv][i];
            }
        }
        __syncthreads();
        const int ncur = s_nn[cur];
        for (int i = threadIdx.x; i < ncur; i += blockDim.x) nda[cur][i] = (ndc[cur][i] && nds[cur][i] <= 1) ? 1 : 0;
        __syncthreads();
        if (threadIdx.x == 0) {
            s_nrl[prv] = 0;
            s_nn[prv] = 0;
        }
        __syncthreads();
        cur = prv;
    }
    // level 0: the whole object is one branch
    const int fin = cur ^ 1;
    if (threadIdx.x == 0) {
        for (int i = 0; i < s_nn[fin]; i++)
            if (nda[fin][i]) kept[s_nkept++] = (unsigned long long)(unsigned)ndr[fin][i];
        A.R.nkept[r] = s_nkept;
    }
}

// ---------------------------------------------------------------------------
// second pass: ownership of the kept branches, preanalysis, gatherup
// ---------------------------------------------------------------------------
#define PI_XMIN 0
#define PI_XMAX 1
#define PI_YMIN 2
#define PI_YMAX 3
#define PI_PEAK 4
#define PI_CPEAK 5
#define PI_DNPIX 6
#define PI_AREA2 7
#define PA_RV 0
#define PA_MX 1
#define PA_MY 2
#define PA_MX2 3
#define PA_MY2 4
#define PA_MXY 5
#define PA_TV 6

__device__ __forceinline__ void lacc_add(unsigned long long *a, float f, int e0, int *status) {
    limbs_atomic_add_term(a, f, e0, status);
}

__device__ __forceinline__ void deblend_assign_root(const DebArgs &A, const int r) {
    __shared__ float thr[DB_MAXLEV];
    __shared__ int lvcnt[DB_MAXLEV + 1], lvstart[DB_MAXLEV + 1], lvkept[DB_MAXLEV];
    const int off = A.R.off[r], P = A.R.size[r], K = A.R.nkept[r], ob = A.R.objbase[r];
    const unsigned *pix = A.rpix + off;
    int *par = A.D.par + off, *lev = A.D.lev + off, *order = A.D.order + off;
    int *own = A.D.own + off, *kl = A.D.kl + off, *kidx = A.D.kidx + off;
    unsigned long long *kept = A.D.kept + off;
    unsigned long long *kept2 = A.D.acc + (size_t)off * 4;  // this root's acc is free now: sorted kept list
    int *pint = A.D.pint + (size_t)off * 8;
    int *status = &A.sc->status;
    const float fdpeak = A.R.fdpeak[r];
    block_thresholds(A, A.R.dthresh[r], fdpeak, thr);
    for (int i = threadIdx.x; i <= A.N; i += blockDim.x) {
        lvcnt[i] = 0;
        if (i < DB_MAXLEV) lvkept[i] = 0;
    }
    for (int k = threadIdx.x; k < P; k += blockDim.x) {
        own[k] = -1;
        kl[k] = -1;
    }
    __syncthreads();
    // kept list in (level, label) order
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        unsigned long long key = kept[i];
        int rank = 0;
        for (int j = 0; j < K; j++) rank += kept[j] < key;
        kept2[rank] = key;
    }
    for (int k = threadIdx.x; k < P; k += blockDim.x) atomicAdd(&lvcnt[lev[k]], 1);
    __syncthreads();
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
        unsigned long long key = kept2[i];
        int L = (int)(key >> 32), c = (int)(key & 0xffffffffu);
        kl[c] = L;
        kidx[c] = i;
        atomicAdd(&lvkept[L], 1);
    }
    if (threadIdx.x == 0) {
        int s = 0;
        for (int L = A.N - 1; L >= 0; L--) {
            lvstart[L] = s;
            s += lvcnt[L];
        }
    }
    __syncthreads();
    // replay of the sweep; at levels with kept branches label their pixels
    for (int L = A.N - 1; L >= 0; L--) {
        const int b0 = lvstart[L], b1 = lvstart[L] + lvcnt[L];
        activate_and_union(A, off, L, b0, b1, order, par, lev);
        if (lvkept[L]) {
            for (int i = threadIdx.x; i < b1; i += blockDim.x) {
                int e = order[i];
                int rt = lfind(par, e);
                if (kl[rt] == L) own[e] = kidx[rt];
            }
            __syncthreads();
        }
    }
    // preanalysis of each kept branch over its own pixels
    // (cudaanalyse.cu:1686-1903).  The owned pixels are grouped by branch with
    // a counting sort, then one warp reduces each branch with exact sums.
    int *bcnt = pint, *bstart = pint + K, *bcur = pint + 2 * K, *blist = pint + 3 * K;
    for (int k = threadIdx.x; k < K; k += blockDim.x) bcnt[k] = bcur[k] = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < P; e += blockDim.x)
        if (own[e] >= 0) atomicAdd(&bcnt[own[e]], 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int k = 0; k < K; k++) {
            bstart[k] = s;
            s += bcnt[k];
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < P; e += blockDim.x) {
        int k = own[e];
        if (k >= 0) blist[bstart[k] + atomicAdd(&bcur[k], 1)] = e;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
    for (int k = threadIdx.x >> 5; k < K; k += nwarp) {
        const int o = ob + k, L = (int)(kept2[k] >> 32), nb = bcnt[k], b0 = bstart[k];
        int xmin = 0x7fffffff, xmax = -1, ymin = 0x7fffffff, ymax = -1;
        unsigned pk = 0u, cpk = 0u;
        XSum srv;
        xs_init(srv);
        for (int i = lane; i < nb; i += 32) {
            int p = (int)pix[blist[b0 + i]], x = p % A.w, y = p / A.w;
            xmin = min(xmin, x);
            xmax = max(xmax, x);
            ymin = min(ymin, y);
            ymax = max(ymax, y);
            pk = max(pk, f2ord(A.sub[p]));
            float c = A.cd[p];
            cpk = max(cpk, f2ord(c));
            xs_add(srv, c);
        }
        for (int d = 16; d > 0; d >>= 1) {
            xmin = min(xmin, __shfl_xor_sync(0xffffffffu, xmin, d));
            xmax = max(xmax, __shfl_xor_sync(0xffffffffu, xmax, d));
            ymin = min(ymin, __shfl_xor_sync(0xffffffffu, ymin, d));
            ymax = max(ymax, __shfl_xor_sync(0xffffffffu, ymax, d));
            pk = max(pk, __shfl_xor_sync(0xffffffffu, pk, d));
            cpk = max(cpk, __shfl_xor_sync(0xffffffffu, cpk, d));
        }
        srv = xs_warp_reduce(srv);
        const float peak = ord2f(pk);
        const double dthresh = thr[L], dthresh2 = (dthresh + peak) / 2.0;
        XSum smx, smy, smx2, smy2, smxy, stv;
        xs_init(smx);
        xs_init(smy);
        xs_init(smx2);
        xs_init(smy2);
        xs_init(smxy);
        xs_init(stv);
        int dnpix = 0, area2 = 0;
        for (int i = lane; i < nb; i += 32) {
            int p = (int)pix[blist[b0 + i]];
            int x = p % A.w - xmin, y = p / A.w - ymin;
            float cval = A.cd[p], val = A.sub[p];
            dnpix += val > dthresh;
            area2 += val > dthresh2;
            xs_add(smx, cval * x);
            xs_add(smy, cval * y);
            xs_add(smx2, cval * x * x);
            xs_add(smy2, cval * y * y);
            xs_add(smxy, cval * x * y);
            xs_add(stv, val);
        }
        for (int d = 16; d > 0; d >>= 1) {
            dnpix += __shfl_xor_sync(0xffffffffu, dnpix, d);
            area2 += __shfl_xor_sync(0xffffffffu, area2, d);
        }
        smx = xs_warp_reduce(smx);
        smy = xs_warp_reduce(smy);
        smx2 = xs_warp_reduce(smx2);
        smy2 = xs_warp_reduce(smy2);
        smxy = xs_warp_reduce(smxy);
        stv = xs_warp_reduce(stv);
        if (lane != 0) continue;
        if (srv.ovf | smx.ovf | smy.ovf | smx2.ovf | smy2.ovf | smxy.ovf | stv.ovf) atomicOr(status, SX_ST_RANGE);
        int flag = 0;
        if (L > 0) flag |= SX_OBJ_MERGED;
        if (xmin == 0 || xmax == A.w - 1 || ymin == 0 || ymax == A.h - 1) flag |= SX_OBJ_TRUNC;
        float rv = xs_float(srv);
        double rvd = rv;
        double mx = xs_double(smx), my = xs_double(smy);
        double mx2 = xs_double(smx2), my2 = xs_double(smy2), mxy = xs_double(smxy);
        double xm = mx / rvd, ym = my / rvd;
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
        float fa = (float)sqrt(pmx2), fb = (float)sqrt(pmy2), abcor;
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
        A.O.n[o] = 0;
    }
    __syncthreads();
    // gatherup (cudadeblend.cu:1262-1360): the nearest kept branch in the
    // elliptical metric, first in order on ties
    for (int e = threadIdx.x; e < P; e += blockDim.x) {
        int k = own[e];
        int p = (int)pix[e];
        if (k < 0) {
            int x = p % A.w, y = p / A.w, iclst = 0;
            float distmin = 1e+31f, dx, dy, dist;
            for (int i = 0; i < K; i++) {
                int o = ob + i;
                dx = x - A.O.mx[o];
                dy = y - A.O.my[o];
                dist = 0.5 * (A.O.cxx[o] * dx * dx + A.O.cyy[o] * dy * dy + A.O.cxy[o] * dx * dy) / A.O.abcor[o];
                if (dist < distmin) {
                    distmin = dist;
                    iclst = i;
                }
            }
            k = iclst;
        }
        A.alloc[p] = ob + k;
        A.objkey[off + e] = (unsigned)(ob + k);
        atomicAdd(&A.O.n[ob + k], 1);
    }
}

// persistent CTAs over a device-side list of raw objects (see
// k_deblend_local.cu); these take the objects too large for shared memory
__global__ void __launch_bounds__(DB_THREADS) k_deblend_sweep(const __grid_constant__ DebArgs A, const int *roots,
                                                              const int *nroots, int *cursor) {
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(cursor, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= *nroots) break;
        deblend_sweep_root(A, roots[item]);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(DB_THREADS) k_deblend_assign(const __grid_constant__ DebArgs A, const int *roots,
                                                               const int *nroots, int *cursor) {
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(cursor, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= *nroots) break;
        deblend_assign_root(A, roots[item]);
        __syncthreads();
    }
}

}  // namespace sx
