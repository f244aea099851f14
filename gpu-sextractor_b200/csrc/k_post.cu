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

__global__ void k_clean_count(ObjBufs O, int n, int *cellcnt, int gx, int gy) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    O.master[i] = 0x7fffffff;
    atomicAdd(&cellcnt[clean_cell(O.mx[i], O.my[i], gx, gy)], 1);
}

__global__ void k_clean_pack(ObjBufs O, int n, double beta, const int *cellstart, int *cellcur, CleanObj *packed,
                             int gx, int gy) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
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
// of larger a (lower index on ties), which searches 20*a around itself; one
// warp per object, lanes over the cells of the search box
__global__ void k_clean_pairs(const CleanObj *__restrict__ packed, int n, double beta,
                              const int *__restrict__ cellstart, int *master, int gx, int gy) {
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (k >= n) return;
    const CleanObj me = packed[k];
    const double rad = 20.0 * me.a * 1.001 + 2.0;
    int x0 = max((int)floor((me.mx - rad) / CL_CELL), 0), x1 = min((int)floor((me.mx + rad) / CL_CELL), gx - 1);
    int y0 = max((int)floor((me.my - rad) / CL_CELL), 0), y1 = min((int)floor((me.my + rad) / CL_CELL), gy - 1);
    int bw = x1 - x0 + 1, nc = bw * (y1 - y0 + 1);
    for (int c = lane; c < nc; c += 32) {
        int cell = (y0 + c / bw) * gx + x0 + c % bw;
        for (int t = cellstart[cell]; t < cellstart[cell + 1]; t++) {
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
__global__ void k_clean_chain(ObjBufs O, int n, unsigned *vkey, unsigned *vval, int *nvict) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int m = O.master[i];
    if (m == 0x7fffffff) {
        O.fmaster[i] = -1;
        return;
    }
    for (int it = 0; it < n && O.master[m] != 0x7fffffff; it++) m = O.master[m];
    O.fmaster[i] = m;
    int k = atomicAdd(nvict, 1);
    vkey[k] = (unsigned)m;
    vval[k] = (unsigned)i;
}

// victims sorted by (master, index): each segment head merges its segment
__global__ void k_clean_merge(ObjBufs O, const unsigned *vkey, const unsigned *vval, int nv) {
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
__global__ void k_alloc_victims(ObjBufs O, const unsigned *opix, int *alloc, int n) {
    int o = blockIdx.x;
    if (o >= n) return;
    int m = O.fmaster[o];
    if (m < 0) return;
    int off = O.off[o], cnt = O.n[o];
    for (int i = threadIdx.x; i < cnt; i += blockDim.x) alloc[opix[off + i]] = m;
}

// ---------------------------------------------------------------------------
// photometry and FLAGS of the survivors
// ---------------------------------------------------------------------------
struct EndArgs {
    const float *sub;
    const int *alloc;
    ObjBufs O;
    FrameScalars *sc;
    int w, h, n, mask_type;
    double aperture, autoparam0, autoparam1, gain, zp, satur;
    const float *wvar;  // calibrated variance map, or null
};

// src/cuda/cudaanalyse.cu:104-287 (computeaperflux, one aperture).  The
// lanes of the warp evaluate 32 aperture pixels at a time (sub-pixel area,
// masked value); the three double sums then take the terms one by one in the
// raster order of the sequential loop, so the rounding is that loop's.
__device__ void aper_warp(const EndArgs &A, int o, double mx, double my, int &flags) {
    const int lane = threadIdx.x & 31, w = A.w, h = A.h;
    const int corrflag = (A.mask_type == 2);
    const float backsig = A.sc->backsig;
    const double var = backsig * backsig;
    const float raper = A.aperture / 2.0;
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
    tv -= area * 0.0;
    if (A.gain > 0.0 && tv > 0.0) sigtv += tv / A.gain;
    A.O.flux_aper[o] = tv;
    A.O.fluxerr_aper[o] = sqrt(sigtv);
    A.O.mag_aper[o] = tv > 0.0 ? -2.5 * log10(tv) + A.zp : 99.0;
    A.O.magerr_aper[o] = tv > 0.0 ? 1.086 * sqrt(sigtv) / tv : 99.0;
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

// one warp per surviving object
__global__ void k_endobject(EndArgs A) {
    const int lane = threadIdx.x & 31;
    const int o = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (o >= A.n) return;
    if (A.O.fmaster[o] >= 0) return;
    const int w = A.w, h = A.h;
    int flags = A.O.flags[o];
    float a = A.O.a[o], b = A.O.b[o];
    double mx = A.O.mx[o], my = A.O.my[o];
    float flux = A.O.flux[o], fluxerr = A.O.fluxerr[o], dthresh = A.O.dthr[o], backsig = A.sc->backsig;
    int fdnpix = A.O.fdnpix[o];
    aper_warp(A, o, mx, my, flags);
    // AUTO / Kron, src/cuda/cudaanalyse.cu:293-592
    double var = backsig * backsig;
    int corrflag = (A.mask_type == 2);
    float dx, dy, cx2, cy2, cxy, r2, klim2, dxlim, dylim, pix, kron = 0.0f;
    int xmin, xmax, ymin, ymax, area, areab;
    const double autoaper0 = 0.0, autoaper1 = 0.0;
    float cxx = A.O.cxx[o], cyy = A.O.cyy[o], cxyo = A.O.cxy[o];
    if (SX_KRON_NSIG * sqrtf(a * b) > autoaper0 / 2.0) {
        cx2 = cxx;
        cy2 = cyy;
        cxy = cxyo;
        dxlim = cx2 - cxy * cxy / (4.0 * cy2);
        dxlim = dxlim > 0.0 ? SX_KRON_NSIG / sqrtf(dxlim) : 0.0;
        dylim = cy2 - cxy * cxy / (4.0 * cx2);
        dylim = dylim > 0.0 ? SX_KRON_NSIG / sqrtf(dylim) : 0.0;
        klim2 = SX_KRON_NSIG * SX_KRON_NSIG;
    } else {
        cx2 = cy2 = 1.0;
        cxy = 0.0;
        dxlim = dylim = autoaper0 / 2.0;
        klim2 = dxlim * dxlim;
    }
    if ((xmin = SX_RINT(mx - dxlim)) < 0) {
        xmin = 0;
        flags |= SX_OBJ_APERT_PB;
    }
    if ((xmax = SX_RINT(mx + dxlim) + 1) > w) {
        xmax = w;
        flags |= SX_OBJ_APERT_PB;
    }
    if ((ymin = SX_RINT(my - dylim)) < 0) {
        ymin = 0;
        flags |= SX_OBJ_APERT_PB;
    }
    if ((ymax = SX_RINT(my + dylim) + 1) > h) {
        ymax = h;
        flags |= SX_OBJ_APERT_PB;
    }
    XSum sr1, sv1;
    xs_init(sr1);
    xs_init(sv1);
    area = areab = 0;
    {
        int bw = xmax - xmin, nn = bw * (ymax - ymin);
        const FastDiv bd = make_fastdiv_dev((unsigned)bw);
        for (int i = lane; i < nn; i += 32) {
            int yo = (int)fdiv((unsigned)i, bd), x = xmin + (i - yo * bw), y = ymin + yo;
            dx = x - mx;
            dy = y - my;
            if ((r2 = cx2 * dx * dx + cy2 * dy * dy + cxy * dx * dy) <= klim2) {
                pix = A.sub[(size_t)y * w + x];
                int t = A.alloc[(size_t)y * w + x];
                if ((t == o || t == -1) & (pix > -SX_BIG)) {
                    area++;
                    xs_add(sr1, sqrtf(r2) * pix);
                    xs_add(sv1, pix);
                } else
                    areab++;
            }
        }
    }
    sr1 = xs_warp_all2(sr1);
    sv1 = xs_warp_all2(sv1);
    area = wsum(area);
    areab = wsum(areab);
    area += areab;
    double tv, sigtv;
    double r1 = xs_double(sr1), v1 = xs_double(sv1);
    if (area) {
        if (r1 > 0.0 && v1 > 0.0) {
            kron = A.autoparam0 * r1 / v1;
            if (kron < A.autoparam1) kron = A.autoparam1;
        } else
            kron = A.autoparam1;
        if ((float)areab / area > SX_CROWD_THRESHOLD) flags |= SX_OBJ_CROWDED;
        if (kron * sqrtf(a * b) > autoaper1 / 2.0) {
            cx2 = cxx;
            cy2 = cyy;
            cxy = cxyo;
            dxlim = cx2 - cxy * cxy / (4.0 * cy2);
            dxlim = dxlim > 0.0 ? kron / sqrtf(dxlim) : 0.0;
            dylim = cy2 - cxy * cxy / (4.0 * cx2);
            dylim = dylim > 0.0 ? kron / sqrtf(dylim) : 0.0;
            klim2 = kron * kron;
        } else {
            cx2 = cy2 = 1.0;
            cxy = 0.0;
            dxlim = dylim = autoaper1 / 2.0;
            klim2 = dxlim * dxlim;
            kron = 0.0;
        }
        if ((xmin = SX_RINT(mx - dxlim)) < 0) {
            xmin = 0;
            flags |= SX_OBJ_APERT_PB;
        }
        if ((xmax = SX_RINT(mx + dxlim) + 1) > w) {
            xmax = w;
            flags |= SX_OBJ_APERT_PB;
        }
        if ((ymin = SX_RINT(my - dylim)) < 0) {
            ymin = 0;
            flags |= SX_OBJ_APERT_PB;
        }
        if ((ymax = SX_RINT(my + dylim) + 1) > h) {
            ymax = h;
            flags |= SX_OBJ_APERT_PB;
        }
        area = areab = 0;
        XSum stv, svar;
        xs_init(stv);
        xs_init(svar);
        int bw = xmax - xmin, nn = bw * (ymax - ymin);
        const FastDiv bd = make_fastdiv_dev((unsigned)bw);
        for (int i = lane; i < nn; i += 32) {
            int yo = (int)fdiv((unsigned)i, bd), x = xmin + (i - yo * bw), y = ymin + yo;
            dx = x - mx;
            dy = y - my;
            if ((cx2 * dx * dx + cy2 * dy * dy + cxy * dx * dy) <= klim2) {
                area++;
                pix = A.sub[(size_t)y * w + x];
                int t = A.alloc[(size_t)y * w + x];
                float pvar = A.wvar ? A.wvar[(size_t)y * w + x] : 0.0f;
                if ((t >= 0 && t != o) || pix <= -SX_BIG) {
                    areab++;
                    int x2, y2;
                    if (corrflag && (x2 = (int)(2 * mx + 0.49999 - x)) >= 0 && x2 < w &&
                        (y2 = (int)(2 * my + 0.49999 - y)) >= 0 && y2 < h &&
                        ((t = A.alloc[(size_t)y2 * w + x2]) == -1 || t == o) &&
                        A.sub[(size_t)y2 * w + x2] > -SX_BIG) {
                        pix = A.sub[(size_t)y2 * w + x2];
                        if (A.wvar) pvar = A.wvar[(size_t)y2 * w + x2];
                    } else {
                        pix = 0.0;
                        pvar = 0.0f;
                    }
                }
                xs_add(stv, pix);
                if (A.wvar) xs_add(svar, pvar);
            }
        }
        stv = xs_warp_all2(stv);
        if (A.wvar) svar = xs_warp_all2(svar);
        area = wsum(area);
        areab = wsum(areab);
        if ((float)areab > SX_CROWD_THRESHOLD * area) flags |= SX_OBJ_CROWDED;
        tv = xs_double(stv);
        sigtv = A.wvar ? xs_double(svar) : (double)area * var;
        tv -= area * (double)0.0f;
        if (A.gain > 0.0 && tv > 0.0) sigtv += tv / A.gain;
        if ((stv.ovf | svar.ovf) && lane == 0) atomicOr(&A.sc->status, SX_ST_RANGE);
    } else
        tv = sigtv = 0.0;
    if ((sr1.ovf | sv1.ovf) && lane == 0) atomicOr(&A.sc->status, SX_ST_RANGE);
    if (lane != 0) return;
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

// ---------------------------------------------------------------------------
// catalogue order and output
// ---------------------------------------------------------------------------
// survivors compacted in index order (scan of the survivor flags)
__global__ void k_surv_flags(ObjBufs O, int n, int *flag) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) flag[i] = O.fmaster[i] < 0 ? 1 : 0;
}

__global__ void k_surv_compact(ObjBufs O, const int *rymax, const int *rlastx, const int *pos, int n, int w,
                               int numbering, unsigned *keys, unsigned *vals) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || O.fmaster[i] >= 0) return;
    int r = O.root[i], j = pos[i];
    keys[j] = numbering == 0 ? (unsigned)rymax[r] * (unsigned)w + (unsigned)rlastx[r] : 0u;
    vals[j] = (unsigned)i;
}

__global__ void k_number(ObjBufs O, const unsigned *vals, int ns) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < ns) O.number[vals[k]] = k + 1;
}

__global__ void k_write_rows(ObjBufs O, const unsigned *vals, int ns, float dthresh, float thresh,
                             sexgpu_object *rows) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ns) return;
    int o = (int)vals[k];
    sexgpu_object q;
    memset(&q, 0, sizeof(q));  // padding bytes too: rows are byte-for-byte reproducible
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
    q.poserr_mx2 = O.pmx2[o];
    q.poserr_my2 = O.pmy2[o];
    q.poserr_mxy = O.pmxy[o];
    q.bkg = O.bkg[o];
    q.thresh = O.athr[o];
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
    rows[k] = q;
}

// segmentation map: NUMBER of the owning object, 0 elsewhere
__global__ void k_segmap(const int *alloc, const int *number, int *seg, long long npix) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npix) return;
    int a = alloc[p];
    seg[p] = (a >= 0 && a != SX_ALLOC_OTHER) ? number[a] : 0;
}

}  // namespace sx
