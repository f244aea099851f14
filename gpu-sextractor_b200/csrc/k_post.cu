// k_post.cu -- CLEAN, merging of cleaned objects, photometry and FLAGS of
// the surviving objects, catalogue order and output.
//
// Reference: src/clean.c:89-180 (the CLEAN test) and :234-287 (mergeobject);
// src/cuda/cudaclean.cu:120-175 (pairwise form); src/cuda/cudaanalyse.cu:62-98
// (isocor), :104-287 (aperture), :293-592 (Kron/AUTO with OBJ_CROWDED and
// OBJ_APERT_PB), :2874 (OBJ_SATUR); catalogue numbering src/scan.c:148-157.
#include "common.cuh"
#include "kernels.cuh"
#include "sexgpu.h"

namespace sx {

// ---------------------------------------------------------------------------
// CLEAN
// ---------------------------------------------------------------------------
constexpr float CL_CELL = 32.0f;

// per-object CLEAN record, stored in cell order so that a cell's objects are
// contiguous (src/clean.c:105-107 for amp and alpha)
struct CleanObj {
    double mx, my, amp, alpha;
    float a, fdflux, cxx, cyy, cxy, mthresh;
    int idx, pad;
};

__device__ __forceinline__ int clean_cell(double mx, double my, int gx, int gy) {
    int cx = (int)floor(mx / CL_CELL), cy = (int)floor(my / CL_CELL);
    cx = min(max(cx, 0), gx - 1);
    cy = min(max(cy, 0), gy - 1);
    return cy * gx + cx;
}

__global__ void k_clean_count(ObjBufs O, int n, const int *n_dev, int *cellcnt, int gx, int gy) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sx_count(n, n_dev)) return;
    O.master[i] = 0x7fffffff;
    atomicAdd(&cellcnt[clean_cell(O.mx[i], O.my[i], gx, gy)], 1);
}

__global__ void k_clean_pack(ObjBufs O, int n, const int *n_dev, double beta, const int *cellstart, int *cellcur,
                             CleanObj *packed, int gx, int gy) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sx_count(n, n_dev)) return;
    CleanObj c;
    double unitarea = SX_PI * O.a[i] * O.b[i];
    c.amp = O.fdflux[i] / (2 * unitarea * O.abcor[i]);
    double q = c.amp / O.dthr[i];
    c.alpha = ((beta == 1.0 ? q : pow(q, 1.0 / beta)) - 1) * unitarea / O.fdnpix[i];
    c.mx = O.mx[i];
    c.my = O.my[i];
    c.a = O.a[i];
    c.fdflux = O.fdflux[i];
    c.cxx = O.cxx[i];
    c.cyy = O.cyy[i];
    c.cxy = O.cxy[i];
    c.mthresh = O.mthresh[i];
    c.idx = i;
    c.pad = 0;
    int cell = clean_cell(c.mx, c.my, gx, gy);
    packed[cellstart[cell] + atomicAdd(&cellcur[cell], 1)] = c;
}

// src/clean.c:108-132 on the pair (p, q) with p.idx < q.idx (the kernel's
// orientation, src/cuda/cudaclean.cu:140-170)
__device__ __forceinline__ void clean_test(const CleanObj &p, const CleanObj &q, double beta, int *master) {
    float dx, dy, rlim;
    double val;
    dx = p.mx - q.mx;
    dy = p.my - q.my;
    rlim = p.a + q.a;
    rlim *= rlim;
    if (!(dx * dx + dy * dy < rlim * SX_CLEAN_ZONE * SX_CLEAN_ZONE)) return;
    if (p.fdflux < q.fdflux) {
        val = 1 + q.alpha * (q.cxx * dx * dx + q.cyy * dy * dy + q.cxy * dx * dy);
        if (val > 1.0 && ((float)(val < 1e10 ? q.amp * (beta == 1.0 ? 1.0 / val : pow(val, -beta)) : 0.0)
                          > p.mthresh))
            atomicMin(&master[p.idx], q.idx);
    } else {
        val = 1 + p.alpha * (p.cxx * dx * dx + p.cyy * dy * dy + p.cxy * dx * dy);
        if (val > 1.0 && ((float)(val < 1e10 ? p.amp * (beta == 1.0 ? 1.0 / val : pow(val, -beta)) : 0.0)
                          > q.mthresh))
            atomicMin(&master[q.idx], p.idx);
    }
}

// every pair closer than CLEAN_ZONE*(a_i+a_j) is tested once, by the object
// of larger a (lower index on ties), which searches 20*a around itself.  The
// objects are packed by cell in row-major cell order, so the cells of one row
// of the search box hold one contiguous range of objects: the lanes of a warp
// stride over that range (coalesced, balanced).  One block of CL_PAIR_WARPS
// warps per object, the warps taking the rows of its search box in turn, so
// that the few objects with large boxes do not leave one warp running long
// after the others.
constexpr int CL_PAIR_WARPS = 4;

__global__ void __launch_bounds__(CL_PAIR_WARPS * 32) k_clean_pairs(const CleanObj *__restrict__ packed, int n,
                                                                    const int *n_dev, double beta,
                                                                    const int *__restrict__ cellstart,
                                                                    int *master, int gx, int gy) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = blockIdx.x;
    if (k >= sx_count(n, n_dev)) return;
    const CleanObj me = packed[k];
    const double rad = 20.0 * me.a * 1.001 + 2.0;
    int x0 = max((int)floor((me.mx - rad) / CL_CELL), 0), x1 = min((int)floor((me.mx + rad) / CL_CELL), gx - 1);
    int y0 = max((int)floor((me.my - rad) / CL_CELL), 0), y1 = min((int)floor((me.my + rad) / CL_CELL), gy - 1);
    for (int cy = y0 + wid; cy <= y1; cy += CL_PAIR_WARPS) {
        const int t1 = __ldg(cellstart + cy * gx + x1 + 1);
        for (int t = __ldg(cellstart + cy * gx + x0) + lane; t < t1; t += 32) {
            const CleanObj o = packed[t];
            if (o.idx == me.idx) continue;
            if (o.a < me.a || (o.a == me.a && o.idx > me.idx)) {
                if (me.idx < o.idx)
                    clean_test(me, o, beta, master);
                else
                    clean_test(o, me, beta, master);
            }
        }
    }
}

// end of the master chain; victims with a master get sort keys for merging
// the chain of masters of a victim ends at a survivor after fewer than n
// steps (masters have smaller indices); cap: a smaller bound set for a
// failure test (0: n); running out sets SX_ST_LOOP
__global__ void k_clean_chain(ObjBufs O, int n, const int *n_dev, unsigned *vkey, unsigned *vval, int *nvict,
                              int *status, int cap) {
    n = sx_count(n, n_dev);
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int m = O.master[i];
    if (m == 0x7fffffff) {
        O.fmaster[i] = -1;
        return;
    }
    const int lim = cap > 0 && cap < n ? cap : n;
    int it = 0;
    for (; it < lim && O.master[m] != 0x7fffffff; it++) m = O.master[m];
    if (O.master[m] != 0x7fffffff) atomicOr(status, SX_ST_LOOP);
    O.fmaster[i] = m;
    int k = atomicAdd(nvict, 1);
    vkey[k] = (unsigned)m;
    vval[k] = (unsigned)i;
}

// victims in (master, index) order: one block sorts the (master << 32 |
// index) keys, all distinct, in shared memory (bitonic network); larger
// victim lists go through two stable radix sorts instead.  With the count on
// the device (nv_dev), a list too long for the block is left alone and its
// length written to *big (0 otherwise): the count of the radix sorts.
constexpr int CL_SORT_MAX = 4096;

__global__ void __launch_bounds__(1024) k_victim_sort(unsigned *vkey, unsigned *vval, int nv, const int *nv_dev,
                                                      int *big) {
    __shared__ unsigned long long s[CL_SORT_MAX];
    nv = sx_count(nv, nv_dev);
    if (big && threadIdx.x == 0) *big = nv > CL_SORT_MAX ? nv : 0;
    if (nv > CL_SORT_MAX) return;
    int n2 = 1;
    while (n2 < nv) n2 <<= 1;
    for (int i = threadIdx.x; i < n2; i += blockDim.x)
        s[i] = i < nv ? ((unsigned long long)vkey[i] << 32) | vval[i] : ~0ull;
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n2; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const unsigned long long a = s[i], b = s[l];
                    if ((a > b) == ((i & k) == 0)) {
                        s[i] = b;
                        s[l] = a;
                    }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < nv; i += blockDim.x) {
        vkey[i] = (unsigned)(s[i] >> 32);
        vval[i] = (unsigned)s[i];
    }
}

// victims sorted by (master, index): each segment head merges its segment
__global__ void k_clean_merge(ObjBufs O, const unsigned *vkey, const unsigned *vval, int nv, const int *nv_dev) {
    nv = sx_count(nv, nv_dev);
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nv) return;
    if (k > 0 && vkey[k - 1] == vkey[k]) return;
    int m = (int)vkey[k];
    for (int j = k; j < nv && (int)vkey[j] == m; j++) {
        int s = (int)vval[j];
        O.fdnpix[m] += O.fdnpix[s];
        O.dnpix[m] += O.dnpix[s];
        O.fdflux[m] += O.fdflux[s];
        O.dflux[m] += O.dflux[s];
        O.flux[m] += O.flux[s];
        O.fluxerr[m] += O.fluxerr[s];
        if (O.fdpeak[s] > O.fdpeak[m]) {
            O.fdpeak[m] = O.fdpeak[s];
            O.peakx[m] = O.peakx[s];
            O.peaky[m] = O.peaky[s];
        }
        if (O.dpeak[s] > O.dpeak[m]) O.dpeak[m] = O.dpeak[s];
        if (O.peak[s] > O.peak[m]) O.peak[m] = O.peak[s];
        if (O.xmin[s] < O.xmin[m]) O.xmin[m] = O.xmin[s];
        if (O.xmax[s] > O.xmax[m]) O.xmax[m] = O.xmax[s];
        if (O.ymin[s] < O.ymin[m]) O.ymin[m] = O.ymin[s];
        if (O.ymax[s] > O.ymax[m]) O.ymax[m] = O.ymax[s];
        O.flags[m] |= (O.flags[s] & (~(SX_OBJ_MERGED | SX_OBJ_CROWDED)));
    }
}

// pixels of cleaned objects belong to their master in the allocation map
__global__ void k_alloc_victims(ObjBufs O, const unsigned *opix, int *alloc, int n, const int *n_dev) {
    int o = blockIdx.x;
    if (o >= sx_count(n, n_dev)) return;
    int m = O.fmaster[o];
    if (m < 0) return;
    int off = O.off[o], cnt = O.n[o];
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) alloc[opix[off + i]] = m;
}

// ---------------------------------------------------------------------------
// photometry and FLAGS of the survivors
// ---------------------------------------------------------------------------
struct EndRaw;

struct EndArgs {
    EndRaw *raw;    // per-object scratch between the photometry warps and k_end_finish
    const float *sub;
    const int *alloc;
    ObjBufs O;
    FrameScalars *sc;
    int w, h, n, mask_type;
    const int *n_dev;   // the object count on the device (n is then the capacity), or null
    double aperture, autoparam0, autoparam1, gain, zp, satur;
    int naper;                          // apertures (>= 1); the first is `aperture`
    double apertures[SEXGPU_MAXAPER];
    const float *wvar;  // calibrated variance map, or null
    KronBufs K;         // queued Kron boxes
    const sexgpu_nnw *nnw;  // CLASS_STAR network (device), or null
    double seeing, pixscale;
};

// src/cuda/cudaanalyse.cu:104-287 (computeaperflux, aperture k of diameter
// `diameter`).  The lanes of the warp evaluate 32 aperture pixels at a time
// (sub-pixel area, masked value); the three double sums then take the terms
// one by one in the raster order of the sequential loop, so the rounding is
// that loop's.  The first aperture fills the catalogue columns; with several,
// every one goes to O.aper.
__device__ void aper_warp(const EndArgs &A, int o, double mx, double my, int &flags, double diameter, int k) {
    const int lane = threadIdx.x & 31, w = A.w, h = A.h;
    const int corrflag = (A.mask_type == 2);
    const float backsig = A.sc->backsig;
    const double var = backsig * backsig;
    const float raper = diameter / 2.0;
    const float raper2 = raper * raper;
    const float rintlim = raper - 0.75;
    const float rintlim2 = (rintlim > 0.0) ? rintlim * rintlim : 0.0;
    const float rextlim2 = (raper + 0.75) * (raper + 0.75);
    const float scalex = 1.0 / SX_APER_OVERSAMP, scaley = scalex;
    const float scale2 = scalex * scaley;
    const float offsetx = 0.5 * (scalex - 1.0), offsety = 0.5 * (scaley - 1.0);
    int xmin = (int)(mx - raper + 0.499999);
    int xmax = (int)(mx + raper + 1.499999);
    int ymin = (int)(my - raper + 0.499999);
    int ymax = (int)(my + raper + 1.499999);
    if (xmin < 0) {
        xmin = 0;
        flags |= SX_OBJ_APERT_PB;
    }
    if (xmax > w) {
        xmax = w;
        flags |= SX_OBJ_APERT_PB;
    }
    if (ymin < 0) {
        ymin = 0;
        flags |= SX_OBJ_APERT_PB;
    }
    if (ymax > h) {
        ymax = h;
        flags |= SX_OBJ_APERT_PB;
    }
    double tv = 0.0, sigtv = 0.0, area = 0.0;
    const int bw = xmax - xmin, nn = bw * (ymax - ymin);
    for (int base = 0; base < nn; base += 32) {
        const int i = base + lane;
        bool in = false;
        float locarea = 0.0f;
        double pix = 0.0, pvar = var;
        if (i < nn) {
            const int yo = i / bw, x = xmin + (i - yo * bw), y = ymin + yo;
            float dx = x - mx, dy = y - my, r2;
            if ((r2 = dx * dx + dy * dy) < rextlim2) {
                in = true;
                if (r2 > rintlim2) {
                    dx += offsetx;
                    dy += offsety;
                    for (int sy = SX_APER_OVERSAMP; sy--; dy += scaley) {
                        float dx1 = dx, dy2 = dy * dy;
                        for (int sx = SX_APER_OVERSAMP; sx--; dx1 += scalex)
                            if (dx1 * dx1 + dy2 < raper2) locarea += scale2;
                    }
                } else
                    locarea = 1.0;
                pix = A.sub[(size_t)y * w + x];
                int t = A.alloc[(size_t)y * w + x], x2, y2;
                // with a weight map: the variance of the pixel actually used,
                // 0 for a pixel replaced by 0 (src/photom.c:128-145)
                if (A.wvar) pvar = A.wvar[(size_t)y * w + x];
                if ((t >= 0 && t != o) || pix <= -SX_BIG) {
                    if (corrflag && (x2 = (int)(2 * mx + 0.49999 - x)) >= 0 && x2 < w &&
                        (y2 = (int)(2 * my + 0.49999 - y)) >= 0 && y2 < h &&
                        ((t = A.alloc[(size_t)y2 * w + x2]) == o || t == -1) &&
                        A.sub[(size_t)y2 * w + x2] > -SX_BIG) {
                        pix = A.sub[(size_t)y2 * w + x2];
                        if (A.wvar) pvar = A.wvar[(size_t)y2 * w + x2];
                    } else {
                        pix = 0.0;
                        if (A.wvar) pvar = 0.0;
                    }
                }
            }
        }
        const double tsig = pvar * locarea, ttv = locarea * pix;
        for (unsigned m = __ballot_sync(0xffffffffu, in); m; m &= m - 1) {
            const int q = __ffs(m) - 1;
            area += __shfl_sync(0xffffffffu, locarea, q);
            sigtv += __shfl_sync(0xffffffffu, tsig, q);
            tv += __shfl_sync(0xffffffffu, ttv, q);
        }
    }
    if (lane != 0) return;
    if (A.O.dbkg) tv -= area * (double)A.O.dbkg[o];
    if (A.gain > 0.0 && tv > 0.0) sigtv += tv / A.gain;
    const float f = tv, fe = sqrt(sigtv), mg = tv > 0.0 ? -2.5 * log10(tv) + A.zp : 99.0,
                me = tv > 0.0 ? 1.086 * sqrt(sigtv) / tv : 99.0;
    if (k == 0) {
        A.O.flux_aper[o] = f;
        A.O.fluxerr_aper[o] = fe;
        A.O.mag_aper[o] = mg;
        A.O.magerr_aper[o] = me;
    }
    if (A.naper > 1) A.O.aper[(size_t)o * A.naper + k] = make_float4(f, fe, mg, me);
}

#define SX_RINT(x) (int)(floor(x + 0.5))

__device__ __forceinline__ XSum xs_warp_all2(XSum s) {
    s = xs_warp_reduce(s);
    unsigned long long lo = (unsigned long long)s.v, hi = (unsigned long long)(s.v >> 64);
    lo = __shfl_sync(0xffffffffu, lo, 0);
    hi = __shfl_sync(0xffffffffu, hi, 0);
    s.v = (__int128)(((unsigned __int128)hi << 64) | lo);
    s.e = __shfl_sync(0xffffffffu, s.e, 0);
    s.ovf = __shfl_sync(0xffffffffu, s.ovf, 0);
    return s;
}
__device__ __forceinline__ int wsum(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// AUTO / Kron photometry, src/cuda/cudaanalyse.cu:293-592.  Pass 1 sums
// r*pix and pix over the 6-sigma ellipse (kron radius), pass 2 the flux inside
// kron*ellipse.  Both sums are exact, so a box may be split freely: a warp
// takes the boxes of up to KronBufs::warp_max pixels; larger ones (a kron
// radius that grew over a faint, elongated object can span the frame) are
// queued and cut into KR_CHUNK-pixel work items for whole CTAs, whose
// partial sums a warp per object merges afterwards.
// ---------------------------------------------------------------------------
struct KronAcc {
    XSum s0, s1;  // pass 1: r*pix, pix;  pass 2: pix, variance
    int area, areab;
};

// what the photometry warps hand to k_end_finish (one thread per object)
struct EndRaw {
    KronAcc p2;     // pass-2 (AUTO) sums, when have2
    float kron;
    int flags, have2;
};

__device__ __forceinline__ void kacc_init(KronAcc &c) {
    xs_init(c.s0);
    xs_init(c.s1);
    c.area = c.areab = 0;
}

__device__ __forceinline__ void kacc_merge(KronAcc &c, const KronAcc &b) {
    xs_merge(c.s0, b.s0);
    xs_merge(c.s1, b.s1);
    c.area += b.area;
    c.areab += b.areab;
}

__device__ __forceinline__ void kacc_warp(KronAcc &c) {
    c.s0 = xs_warp_all2(c.s0);
    c.s1 = xs_warp_all2(c.s1);
    c.area = wsum(c.area);
    c.areab = wsum(c.areab);
}

__device__ __forceinline__ void kron_box(const EndArgs &A, double mx, double my, float dxlim, float dylim, KronGeo &g,
                                         int &flags) {
    if ((g.xmin = SX_RINT(mx - dxlim)) < 0) {
        g.xmin = 0;
        flags |= SX_OBJ_APERT_PB;
    }
    if ((g.xmax = SX_RINT(mx + dxlim) + 1) > A.w) {
        g.xmax = A.w;
        flags |= SX_OBJ_APERT_PB;
    }
    if ((g.ymin = SX_RINT(my - dylim)) < 0) {
        g.ymin = 0;
        flags |= SX_OBJ_APERT_PB;
    }
    if ((g.ymax = SX_RINT(my + dylim) + 1) > A.h) {
        g.ymax = A.h;
        flags |= SX_OBJ_APERT_PB;
    }
}

// pass-1 ellipse and box (cudaanalyse.cu:318-357)
__device__ __forceinline__ void kron_geo1(const EndArgs &A, int o, double mx, double my, KronGeo &g, int &flags) {
    const double autoaper0 = 0.0;
    const float a = A.O.a[o], b = A.O.b[o];
    float dxlim, dylim;
    if (SX_KRON_NSIG * sqrtf(a * b) > autoaper0 / 2.0) {
        g.cx2 = A.O.cxx[o];
        g.cy2 = A.O.cyy[o];
        g.cxy = A.O.cxy[o];
        dxlim = g.cx2 - g.cxy * g.cxy / (4.0 * g.cy2);
        dxlim = dxlim > 0.0 ? SX_KRON_NSIG / sqrtf(dxlim) : 0.0;
        dylim = g.cy2 - g.cxy * g.cxy / (4.0 * g.cx2);
        dylim = dylim > 0.0 ? SX_KRON_NSIG / sqrtf(dylim) : 0.0;
        g.klim2 = SX_KRON_NSIG * SX_KRON_NSIG;
    } else {
        g.cx2 = g.cy2 = 1.0;
        g.cxy = 0.0;
        dxlim = dylim = autoaper0 / 2.0;
        g.klim2 = dxlim * dxlim;
    }
    kron_box(A, mx, my, dxlim, dylim, g, flags);
}

// kron radius from pass 1 and the pass-2 ellipse and box (cudaanalyse.cu:
// 385-440); false when pass 1 found no pixel (no AUTO flux)
__device__ __forceinline__ bool kron_geo2(const EndArgs &A, int o, double mx, double my, const KronAcc &p, float &kron,
                                          KronGeo &g, int &flags) {
    const double autoaper1 = 0.0;
    const int areab = p.areab, area = p.area + p.areab;
    if (!area) return false;
    const double r1 = xs_double(p.s0), v1 = xs_double(p.s1);
    if (r1 > 0.0 && v1 > 0.0) {
        kron = A.autoparam0 * r1 / v1;
        if (kron < A.autoparam1) kron = A.autoparam1;
    } else
        kron = A.autoparam1;
    if ((float)areab / area > SX_CROWD_THRESHOLD) flags |= SX_OBJ_CROWDED;
    const float a = A.O.a[o], b = A.O.b[o];
    float dxlim, dylim;
    if (kron * sqrtf(a * b) > autoaper1 / 2.0) {
        g.cx2 = A.O.cxx[o];
        g.cy2 = A.O.cyy[o];
        g.cxy = A.O.cxy[o];
        dxlim = g.cx2 - g.cxy * g.cxy / (4.0 * g.cy2);
        dxlim = dxlim > 0.0 ? kron / sqrtf(dxlim) : 0.0;
        dylim = g.cy2 - g.cxy * g.cxy / (4.0 * g.cx2);
        dylim = dylim > 0.0 ? kron / sqrtf(dylim) : 0.0;
        g.klim2 = kron * kron;
    } else {
        g.cx2 = g.cy2 = 1.0;
        g.cxy = 0.0;
        dxlim = dylim = autoaper1 / 2.0;
        g.klim2 = dxlim * dxlim;
        kron = 0.0;
    }
    kron_box(A, mx, my, dxlim, dylim, g, flags);
    return true;
}

__device__ __forceinline__ int kron_npix(const KronGeo &g) { return (g.xmax - g.xmin) * (g.ymax - g.ymin); }

// box pixels i0, i0+step, ... below i1 (raster index inside the box)
template <int PASS>
__device__ __forceinline__ void kron_range(const EndArgs &A, int o, double mx, double my, const KronGeo &g, int i0,
                                           int i1, int step, KronAcc &c) {
    const int w = A.w, h = A.h, bw = g.xmax - g.xmin;
    const FastDiv bd = make_fastdiv_dev((unsigned)bw);
    const int corrflag = (A.mask_type == 2);
    for (int i = i0; i < i1; i += step) {
        const int yo = (int)fdiv((unsigned)i, bd), x = g.xmin + (i - yo * bw), y = g.ymin + yo;
        const float dx = x - mx, dy = y - my;
        if (PASS == 1) {
            float r2;
            if ((r2 = g.cx2 * dx * dx + g.cy2 * dy * dy + g.cxy * dx * dy) <= g.klim2) {
                const float pix = A.sub[(size_t)y * w + x];
                const int t = A.alloc[(size_t)y * w + x];
                if ((t == o || t == -1) & (pix > -SX_BIG)) {
                    c.area++;
                    xs_add(c.s0, sqrtf(r2) * pix);
                    xs_add(c.s1, pix);
                } else
                    c.areab++;
            }
        } else if ((g.cx2 * dx * dx + g.cy2 * dy * dy + g.cxy * dx * dy) <= g.klim2) {
            c.area++;
            float pix = A.sub[(size_t)y * w + x];
            int t = A.alloc[(size_t)y * w + x];
            float pvar = A.wvar ? A.wvar[(size_t)y * w + x] : 0.0f;
            if ((t >= 0 && t != o) || pix <= -SX_BIG) {
                c.areab++;
                int x2, y2;
                if (corrflag && (x2 = (int)(2 * mx + 0.49999 - x)) >= 0 && x2 < w &&
                    (y2 = (int)(2 * my + 0.49999 - y)) >= 0 && y2 < h &&
                    ((t = A.alloc[(size_t)y2 * w + x2]) == -1 || t == o) && A.sub[(size_t)y2 * w + x2] > -SX_BIG) {
                    pix = A.sub[(size_t)y2 * w + x2];
                    if (A.wvar) pvar = A.wvar[(size_t)y2 * w + x2];
                } else {
                    pix = 0.0;
                    pvar = 0.0f;
                }
            }
            xs_add(c.s0, pix);
            if (A.wvar) xs_add(c.s1, pvar);
        }
    }
}

// kron_range with the exact sums in double bins (see BinSum): the hints are
// the object's peak (and, for pass 1's r*pix, the ellipse's largest r).
// Returns false in every lane when any lane met a term outside the bins; the
// caller then sums with kron_range.  Pass 2 with a variance map is not binned.
template <int PASS>
__device__ __forceinline__ bool kron_range_bin(const EndArgs &A, int o, double mx, double my, const KronGeo &g,
                                               int i0, int i1, int step, KronAcc &out) {
    const int w = A.w, h = A.h, bw = g.xmax - g.xmin;
    const FastDiv bd = make_fastdiv_dev((unsigned)bw);
    const int corrflag = (A.mask_type == 2);
    const int top1 = bs_order(A.O.peak[o]), top0 = top1 + bs_order(sqrtf(g.klim2)) + 1;
    BinSum b0, b1;
    bs_init(b0);
    bs_init(b1);
    int area = 0, areab = 0;
    bool ok = true;
    for (int i = i0; i < i1; i += step) {
        const int yo = (int)fdiv((unsigned)i, bd), x = g.xmin + (i - yo * bw), y = g.ymin + yo;
        const float dx = x - mx, dy = y - my;
        if (PASS == 1) {
            float r2;
            if ((r2 = g.cx2 * dx * dx + g.cy2 * dy * dy + g.cxy * dx * dy) <= g.klim2) {
                const float pix = A.sub[(size_t)y * w + x];
                const int t = A.alloc[(size_t)y * w + x];
                if ((t == o || t == -1) & (pix > -SX_BIG)) {
                    area++;
                    ok &= bs_add(b0, sqrtf(r2) * pix, top0);
                    ok &= bs_add(b1, pix, top1);
                } else
                    areab++;
            }
        } else if ((g.cx2 * dx * dx + g.cy2 * dy * dy + g.cxy * dx * dy) <= g.klim2) {
            area++;
            float pix = A.sub[(size_t)y * w + x];
            int t = A.alloc[(size_t)y * w + x];
            if ((t >= 0 && t != o) || pix <= -SX_BIG) {
                areab++;
                int x2, y2;
                if (corrflag && (x2 = (int)(2 * mx + 0.49999 - x)) >= 0 && x2 < w &&
                    (y2 = (int)(2 * my + 0.49999 - y)) >= 0 && y2 < h &&
                    ((t = A.alloc[(size_t)y2 * w + x2]) == -1 || t == o) && A.sub[(size_t)y2 * w + x2] > -SX_BIG)
                    pix = A.sub[(size_t)y2 * w + x2];
                else
                    pix = 0.0;
            }
            ok &= bs_add(b0, pix, top1);
        }
    }
    if (!__all_sync(0xffffffffu, ok)) return false;
    out.s0 = bs_to_xsum(bs_warp_sum(b0));
    if (PASS == 1)
        out.s1 = bs_to_xsum(bs_warp_sum(b1));
    else
        xs_init(out.s1);
    out.area = wsum(area);
    out.areab = wsum(areab);
    return true;
}

// a warp's sums over box pixels i0, i0 + step, ... < i1 (every lane holds them)
template <int PASS>
__device__ __forceinline__ void kron_warp_sums(const EndArgs &A, int o, double mx, double my, const KronGeo &g,
                                               int i0, int i1, int step, KronAcc &c) {
    // at most BS_MAX_TERMS terms of the warp per bin
    const bool binned = (PASS == 1 || !A.wvar) && (long long)(i1 - (i0 & ~31)) <= (long long)BS_MAX_TERMS * step / 32;
    if (binned && kron_range_bin<PASS>(A, o, mx, my, g, i0, i1, step, c)) return;
    kacc_init(c);
    kron_range<PASS>(A, o, mx, my, g, i0, i1, step, c);
    kacc_warp(c);
}

// Queue object o's pass-`pass` box (warp-collective).  False when the queue is
// full; the warp then sums the box itself.
__device__ bool kron_defer(const EndArgs &A, int pass, int o, int flags, float kron, const KronGeo &g, int nn) {
    const int lane = threadIdx.x & 31;
    const int nch = (nn + KR_CHUNK - 1) / KR_CHUNK;
    int k = 0, c0 = 0;
    if (lane == 0) {
        k = atomicAdd(&A.sc->kitems[pass], 1);
        c0 = atomicAdd(&A.sc->kchunks[pass], nch);
    }
    k = __shfl_sync(0xffffffffu, k, 0);
    c0 = __shfl_sync(0xffffffffu, c0, 0);
    const bool ok = k < A.K.icap && c0 <= A.K.ccap - nch;
    // this warp's chunk range: item index, or -1 where the item did not fit
    const int cend = min(c0 + nch, A.K.ccap);
    for (int c = c0 + lane; c < cend; c += 32) A.K.chunk[pass][c] = ok ? k : -1;
    if (lane == 0 && k < A.K.icap) {
        KronItem it;
        it.o = o;
        it.flags = flags;
        it.c0 = c0;
        it.nch = ok ? nch : -1;
        it.kron = kron;
        it.g = g;
        A.K.item[pass][k] = it;
    }
    return ok;
}

// catalogue columns of a survivor (lane 0 writes); p2 = pass-2 sums if any
__device__ void end_finish(const EndArgs &A, int o, int flags, float kron, bool have2, const KronAcc &p2) {
    if ((threadIdx.x & 31) != 0) return;
    EndRaw R;
    R.p2 = p2;
    R.kron = kron;
    R.flags = flags;
    R.have2 = have2;
    A.raw[o] = R;
}

// catalogue columns of a survivor from its photometry sums: AUTO, ISOCOR and
// ISO fluxes, magnitudes and errors, FLAGS (one thread per object, so that
// this double-precision tail does not run on one lane of a warp)
__global__ void k_end_finish(EndArgs A) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= sx_count(A.n, A.n_dev) || A.O.fmaster[o] >= 0) return;
    const EndRaw R = A.raw[o];
    const KronAcc &p2 = R.p2;
    const bool have2 = R.have2 != 0;
    int flags = R.flags;
    float kron = R.kron;
    const float backsig = A.sc->backsig;
    const double var = backsig * backsig;
    double tv, sigtv;
    if (have2) {
        const int area = p2.area, areab = p2.areab;
        if ((float)areab > SX_CROWD_THRESHOLD * area) flags |= SX_OBJ_CROWDED;
        tv = xs_double(p2.s0);
        sigtv = A.wvar ? xs_double(p2.s1) : (double)area * var;
        if (A.O.dbkg) tv -= area * (double)A.O.dbkg[o];
        if (A.gain > 0.0 && tv > 0.0) sigtv += tv / A.gain;
        if (p2.s0.ovf | p2.s1.ovf) atomicOr(&A.sc->status, SX_ST_RANGE);
    } else
        tv = sigtv = 0.0;
    const float flux = A.O.flux[o], fluxerr = A.O.fluxerr[o], dthresh = A.O.dthr[o];
    const int fdnpix = A.O.fdnpix[o];
    float flux_auto = tv, fluxerr_auto = sqrt(sigtv);
    if (tv <= 0.0) kron = 0.0;
    A.O.kron[o] = kron;
    A.O.flux_auto[o] = flux_auto;
    A.O.fluxerr_auto[o] = fluxerr_auto;
    A.O.mag_auto[o] = flux_auto > 0.0 ? -2.5 * log10(flux_auto) + A.zp : 99.0;
    A.O.magerr_auto[o] = flux_auto > 0.0 ? 1.086 * fluxerr_auto / flux_auto : 99.0;
    // isocor, src/cuda/cudaanalyse.cu:62-98
    double ati = (flux > 0.0) ? (fdnpix * dthresh / flux) : 0.0;
    if (ati > 1.0)
        ati = 1.0;
    else if (ati < 0.0)
        ati = 0.0;
    A.O.flux_isocor[o] = flux / (1.0 - 0.196099 * ati - 0.751208 * ati * ati);
    if (flux > 0.0) {
        double dati, sg;
        sg = fluxerr / (flux * flux);
        dati = fdnpix ? ati * sqrt(sg + 1.0 / fdnpix) : 0.0;
        dati = 0.196099 * dati + 0.751208 * 2 * ati * dati;
        A.O.fluxerr_isocor[o] = sqrt(sg + dati * dati) * flux;
    } else
        A.O.fluxerr_isocor[o] = sqrt(fluxerr);
    float fluxerr_iso = sqrt(fluxerr);
    A.O.fluxerr_iso[o] = fluxerr_iso;
    A.O.mag_iso[o] = flux > 0.0 ? -2.5 * log10(flux) + A.zp : 99.0;
    A.O.magerr_iso[o] = flux > 0.0 ? 1.086 * fluxerr_iso / flux : 99.0;
    if (A.O.peak[o] + A.O.bkg[o] >= A.satur) flags |= SX_OBJ_SATUR;
    A.O.flags[o] = flags;
}

// after pass 1 (every lane holds its sums): pass 2 in this warp or queued
// defer_at: AUTO boxes of more pixels than this are queued for whole blocks
__device__ void kron_after1(const EndArgs &A, int o, double mx, double my, int flags, const KronAcc &p1,
                            int defer_at) {
    if ((p1.s0.ovf | p1.s1.ovf) && (threadIdx.x & 31) == 0) atomicOr(&A.sc->status, SX_ST_RANGE);
    float kron = 0.0f;
    KronGeo g;
    KronAcc p2;
    kacc_init(p2);
    if (!kron_geo2(A, o, mx, my, p1, kron, g, flags)) {
        end_finish(A, o, flags, kron, false, p2);
        return;
    }
    const int nn = kron_npix(g);
    if (nn > defer_at && kron_defer(A, 1, o, flags, kron, g, nn)) return;
    kron_warp_sums<2>(A, o, mx, my, g, threadIdx.x & 31, nn, 32, p2);
    end_finish(A, o, flags, kron, true, p2);
}

// one warp per surviving object (eight CTAs of four warps per SM)
__global__ void __launch_bounds__(128, 8) k_endobject(EndArgs A) {
    const int lane = threadIdx.x & 31;
    const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (o >= sx_count(A.n, A.n_dev)) return;
    if (A.O.fmaster[o] >= 0) return;
    int flags = A.O.flags[o];
    const double mx = A.O.mx[o], my = A.O.my[o];
    for (int k = 0; k < A.naper; k++) aper_warp(A, o, mx, my, flags, A.apertures[k], k);
    KronGeo g;
    kron_geo1(A, o, mx, my, g, flags);
    const int nn = kron_npix(g);
    if (nn > A.K.warp_max && kron_defer(A, 0, o, flags, 0.0f, g, nn)) return;
    KronAcc p1;
    kron_warp_sums<1>(A, o, mx, my, g, lane, nn, 32, p1);
    kron_after1(A, o, mx, my, flags, p1, A.K.warp_max);
}

// queued boxes: one CTA per KR_CHUNK-pixel work item, partial sums per item
template <int PASS>
__global__ void __launch_bounds__(KR_THREADS) k_kron_chunks(EndArgs A) {
    __shared__ KronAcc red[KR_THREADS / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nc = min(A.sc->kchunks[PASS - 1], A.K.ccap);
    for (int c = blockIdx.x; c < nc; c += gridDim.x) {
        const int k = A.K.chunk[PASS - 1][c];
        if (k < 0) continue;
        const KronItem it = A.K.item[PASS - 1][k];
        const int i0 = (c - it.c0) * KR_CHUNK, i1 = min(kron_npix(it.g), i0 + KR_CHUNK);
        KronAcc acc;
        kron_warp_sums<PASS>(A, it.o, A.O.mx[it.o], A.O.my[it.o], it.g, i0 + threadIdx.x, i1, KR_THREADS, acc);
        if (lane == 0) red[wid] = acc;
        __syncthreads();
        if (wid == 0) {
            KronAcc r;
            kacc_init(r);
            if (lane < KR_THREADS / 32) r = red[lane];
            kacc_warp(r);
            if (lane == 0) A.K.part[PASS - 1][c] = r;
        }
        __syncthreads();
    }
}

// queued boxes: one warp per object merges its items' sums and continues;
// the objects here have large Kron boxes, and their AUTO boxes of more than
// KR_MERGE_MAX pixels go to the block queue too, so that this tail kernel
// does not end on one warp summing thousands of pixels
constexpr int KR_MERGE_MAX = 1024;

template <int PASS>
__global__ void k_kron_merge(EndArgs A) {
    const int lane = threadIdx.x & 31;
    const int n = min(A.sc->kitems[PASS - 1], A.K.icap);
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < n; k += nw) {
        const KronItem it = A.K.item[PASS - 1][k];
        if (it.nch < 0) continue;
        KronAcc acc;
        kacc_init(acc);
        for (int j = lane; j < it.nch; j += 32) kacc_merge(acc, A.K.part[PASS - 1][it.c0 + j]);
        kacc_warp(acc);
        if (PASS == 1)
            kron_after1(A, it.o, A.O.mx[it.o], A.O.my[it.o], it.flags, acc, min(A.K.warp_max, KR_MERGE_MAX));
        else
            end_finish(A, it.o, it.flags, it.kron, true, acc);
    }
}

// CLASS_STAR, src/cuda/cudaanalyse.cu:2901-2920 with the network response of
// :599-632 (src/neurro.c neurresp): inputs are log10 of the eight isophotal
// areas in seeing units and of FLUX_MAX over the threshold, plus log10 of the
// seeing; every layer applies the logistic function; double arithmetic.
__global__ void k_class_star(ObjBufs O, int n, const int *n_dev, const sexgpu_nnw *__restrict__ net, double fwhm,
                             double pixscale) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= sx_count(n, n_dev) || O.fmaster[o] >= 0) return;
    double fac2 = fwhm / pixscale;
    fac2 *= fac2;
    const float thresh = O.athr[o], peak = O.peak[o];
    double in[SEXGPU_NNW_NEURONS], nx[SEXGPU_NNW_NEURONS];
    const int *iso = O.iso + (size_t)o * SX_NISO_;
    int j = 0;
    in[j] = log10(iso[0] ? iso[0] / fac2 : 0.01);
    in[++j] = thresh > 0.0 ? log10(peak > 0.0 ? peak / thresh : 0.1) : -1.0;
    for (int i = 1; i < SX_NISO_; i++) in[++j] = log10(iso[i] ? iso[i] / fac2 : 0.01);
    in[++j] = log10(fwhm);
    const int last = net->nlayers - 1;
    for (int i = 0; i < net->nn[0]; i++) in[i] = in[i] * net->inscale[i] + net->inbias[i];
    for (int l = 0; l < last; l++) {
        for (int k = 0; k < net->nn[l + 1]; k++) {
            double sum = net->b[l][k];
            for (int i = 0; i < net->nn[l]; i++) sum += net->w[l][i][k] * in[i];
            nx[k] = 1.0 / (1.0 + exp(-sum));
        }
        for (int k = 0; k < net->nn[l + 1]; k++) in[k] = nx[k];
    }
    O.sprob[o] = (float)((in[0] - net->outbias[0]) / net->outscale[0]);
}

void launch_endobject(const EndArgs &E, int nobj, cudaStream_t st, int &launches) {
    if (nobj <= 0) return;
    k_endobject<<<(unsigned)((nobj + 3) / 4), 128, 0, st>>>(E);
    k_kron_chunks<1><<<KR_GRID, KR_THREADS, 0, st>>>(E);
    k_kron_merge<1><<<KR_GRID / 2, 128, 0, st>>>(E);
    k_kron_chunks<2><<<KR_GRID, KR_THREADS, 0, st>>>(E);
    k_kron_merge<2><<<KR_GRID / 2, 128, 0, st>>>(E);
    k_end_finish<<<(unsigned)((nobj + 127) / 128), 128, 0, st>>>(E);
    launches += 6;
    if (E.nnw) {
        k_class_star<<<(unsigned)((nobj + 127) / 128), 128, 0, st>>>(E.O, nobj, E.n_dev, E.nnw, E.seeing,
                                                                      E.pixscale);
        launches += 1;
    }
}

// ---------------------------------------------------------------------------
// catalogue order and output
// ---------------------------------------------------------------------------
// survivors compacted in index order (scan of the survivor flags)
__global__ void k_surv_flags(ObjBufs O, int n, const int *n_dev, int *flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < sx_count(n, n_dev)) flag[i] = O.fmaster[i] < 0 ? 1 : 0;
}

__global__ void k_surv_compact(ObjBufs O, const int *rymax, const int *rlastx, const int *pos, int n,
                               const int *n_dev, int w, int numbering, unsigned *keys, unsigned *vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= sx_count(n, n_dev) || O.fmaster[i] >= 0) return;
    int r = O.root[i], j = pos[i];
    keys[j] = numbering == 0 ? (unsigned)rymax[r] * (unsigned)w + (unsigned)rlastx[r] : 0u;
    vals[j] = (unsigned)i;
}

__global__ void k_number(ObjBufs O, const unsigned *vals, int ns, const int *ns_dev) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < sx_count(ns, ns_dev)) O.number[vals[k]] = k + 1;
}

__global__ void k_write_rows(ObjBufs O, const unsigned *vals, int ns, const int *ns_dev, sexgpu_object *rows) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= sx_count(ns, ns_dev)) return;
    int o = (int)vals[k];
    // built in a union with 16-byte words so that the row, padding bytes
    // included, is stored as whole words (rows are byte-for-byte reproducible)
    union {
        sexgpu_object o;
        uint4 v[sizeof(sexgpu_object) / 16];
    } u;
    static_assert(sizeof(sexgpu_object) % 16 == 0, "row size");
    for (int i = 0; i < (int)(sizeof(sexgpu_object) / 16); i++) u.v[i] = make_uint4(0, 0, 0, 0);
    sexgpu_object &q = u.o;
    q.number = k + 1;
    q.root = O.root[o];
    q.level = O.level[o];
    q.fdnpix = O.fdnpix[o];
    q.dnpix = O.dnpix[o];
    q.npix = O.npix[o];
    q.xmin = O.xmin[o];
    q.xmax = O.xmax[o];
    q.ymin = O.ymin[o];
    q.ymax = O.ymax[o];
    q.peakx = O.peakx[o];
    q.peaky = O.peaky[o];
    q.flags = O.flags[o];
    for (int i = 0; i < SX_NISO_; i++) q.iso[i] = O.iso[(size_t)o * SX_NISO_ + i];
    q.fdflux = O.fdflux[o];
    q.dflux = O.dflux[o];
    q.flux = O.flux[o];
    q.fluxerr = O.fluxerr[o];
    q.fdpeak = O.fdpeak[o];
    q.dpeak = O.dpeak[o];
    q.peak = O.peak[o];
    q.mx = O.mx[o];
    q.my = O.my[o];
    q.mx2 = O.mx2[o];
    q.my2 = O.my2[o];
    q.mxy = O.mxy[o];
    q.a = O.a[o];
    q.b = O.b[o];
    q.theta = O.theta[o];
    q.abcor = O.abcor[o];
    q.cxx = O.cxx[o];
    q.cyy = O.cyy[o];
    q.cxy = O.cxy[o];
    q.class_star = O.sprob ? O.sprob[o] : 0.0f;
    q.poserr_mx2 = O.pmx2[o];
    q.poserr_my2 = O.pmy2[o];
    q.poserr_mxy = O.pmxy[o];
    q.bkg = O.bkg[o];
    q.thresh = O.dbkg ? O.athr[o] - O.dbkg[o] : O.athr[o];
    q.dthresh = O.dthr[o];
    q.mthresh = O.mthresh[o];
    q.fwhm = O.fwhm[o];
    q.flux_iso = O.flux[o];
    q.fluxerr_iso = O.fluxerr_iso[o];
    q.mag_iso = O.mag_iso[o];
    q.magerr_iso = O.magerr_iso[o];
    q.flux_isocor = O.flux_isocor[o];
    q.fluxerr_isocor = O.fluxerr_isocor[o];
    q.flux_aper = O.flux_aper[o];
    q.fluxerr_aper = O.fluxerr_aper[o];
    q.mag_aper = O.mag_aper[o];
    q.magerr_aper = O.magerr_aper[o];
    q.kronfactor = O.kron[o];
    q.flux_auto = O.flux_auto[o];
    q.fluxerr_auto = O.fluxerr_auto[o];
    q.mag_auto = O.mag_auto[o];
    q.magerr_auto = O.magerr_auto[o];
    q.elong = q.a / q.b;
    q.ellip = 1 - q.b / q.a;
    q.polar = (q.a * q.a - q.b * q.b) / (q.a * q.a + q.b * q.b);
    // whole words: an assignment may store the members only and leave the
    // padding of the destination row as it was
    uint4 *dst = reinterpret_cast<uint4 *>(rows + k);
    for (int i = 0; i < (int)(sizeof(sexgpu_object) / 16); i++) dst[i] = u.v[i];
}

// every aperture of the catalogue rows, in catalogue order (naper per row)
__global__ void k_write_apers(ObjBufs O, const unsigned *order, int ns, int naper, float4 *out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= ns) return;
    const int o = (int)order[r];
    for (int k = 0; k < naper; k++)
        out[(size_t)r * naper + k] = naper > 1 ? O.aper[(size_t)o * naper + k]
                                               : make_float4(O.flux_aper[o], O.fluxerr_aper[o], O.mag_aper[o],
                                                             O.magerr_aper[o]);
}

// segmentation map: NUMBER of the owning object, 0 elsewhere
__global__ void k_segmap(const int *alloc, const int *number, int *seg, long long npix) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    int a = alloc[p];
    seg[p] = (a >= 0 && a != SX_ALLOC_OTHER) ? number[a] : 0;
}

}  // namespace sx
