// k_analyse.cu -- per-object analysis after deblending: the robust
// preanalysis of deblended objects over their final pixels
// (src/cuda/cudaanalyse.cu:1906-2124) and examineiso (:2176-2581).
//
// One warp per object walks the object's pixel list (contiguous, raster
// order), in two kernels: the robust preanalysis, whose moments examineiso
// reads, then examineiso itself.  Sums that feed decisions or integer outputs are exact (XSum);
// the double sums of the position errors and of the FWHM fit are reduced in
// a fixed lane order.
#include "common.cuh"
#include "kernels.cuh"

namespace sx {

constexpr int AN_WARPS = 8;
// four resident CTAs per SM (at most 64 registers, a few spilled): these
// kernels wait on pixel-list loads, and residency hides that better than
// registers saved (analyse stage 1.37 ms at 4 CTAs/SM, 1.45 at 3 with fewer
// spills, 1.65 at 2 with none; one 4096^2 frame)
constexpr int AN_MINB = 4;

__device__ __forceinline__ unsigned warp_max_u(unsigned v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_min_i(int v) {
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_ull(unsigned long long v) {
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// fixed-order (butterfly) double sum; identical in every lane
__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ XSum xs_warp_all(XSum s) { return xs_warp_sum(s); }

// k-th smallest (0-based) of the cd values of n pixels, as float bits; the
// values are positive (object pixels lie above the detection threshold), so
// their bit patterns sort like the values.  Four 8-bit radix passes; in each
// pass the digit that holds rank k is found by a warp scan over 256 bins
// (lane l owns bins 8l..8l+7).
__device__ unsigned warp_select(const unsigned *opix, int n, const float *cd, int k, unsigned *hist) {
    const int lane = threadIdx.x & 31;
    unsigned prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = lane; i < 256; i += 32) hist[i] = 0;
        __syncwarp();
        for (int i = lane; i < n; i += 32) {
            unsigned key = __float_as_uint(__ldg(cd + __ldg(opix + i)));
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255], 1u);
        }
        __syncwarp();
        const uint4 h0 = reinterpret_cast<const uint4 *>(hist)[lane * 2];
        const uint4 h1 = reinterpret_cast<const uint4 *>(hist)[lane * 2 + 1];
        const unsigned c[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
        unsigned tot = c[0] + c[1] + c[2] + c[3] + c[4] + c[5] + c[6] + c[7];
        unsigned incl = tot;
        for (int o = 1; o < 32; o <<= 1) {
            unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        unsigned excl = incl - tot;
        unsigned sel = __ballot_sync(0xffffffffu, incl > (unsigned)k);
        int owner = __ffs(sel) - 1;  // k < n, so some lane holds rank k
        unsigned digit = 0, below = excl;
        if (lane == owner) {
            int j = 0;
#pragma unroll
            for (int t = 0; t < 7; t++)
                if (j == t && below + c[t] <= (unsigned)k) {
                    below += c[t];
                    j = t + 1;
                }
            digit = lane * 8 + j;
        }
        digit = __shfl_sync(0xffffffffu, digit, owner);
        below = __shfl_sync(0xffffffffu, below, owner);
        prefix |= digit << shift;
        mask |= 255u << shift;
        k -= (int)below;
        __syncwarp();
    }
    return prefix;
}

// what the pixel pass of the robust preanalysis hands to its finishing
// kernel (one thread per object)
struct RobustRaw {
    double mx, my, mx2, my2, mxy;
    float rv, peak, cpeak;
    int dnpix, area2, xmin, xmax, ymin, ymax, flags;
};

// what the pixel pass of examineiso hands to its finishing kernel
struct ExamRaw {
    XSum stv, svar;
    double esum, emx2, emy2, emxy, s, sx, sy, sxx, sxy;
    float opeak, thresh0, mthresh;
    int peakpix, area;
};

struct AnaArgs {
    RobustRaw *raw;     // per-object scratch between the two robust kernels
    ExamRaw *xraw;      // per-object scratch between the two examineiso kernels
    const float *cd, *sub, *back;
    const unsigned *opix;
    ObjBufs O;
    FrameScalars *sc;
    int w, h, nbx, nby, bw, bh, nobj, minarea, clean_flag;
    const int *nobj_dev;  // the object count on the device (nobj is then the capacity), or null
    FastDiv wdiv;
    double gain, satur;
    const float *wvar;  // calibrated variance map, or null
    int wthr;           // analysis threshold follows the local rms
    double afac;        // ANALYSIS_THRESH
    int bp_thick;       // BACKPHOTO_THICK (used when O.dbkg is set)
};

// Robust preanalysis of a deblended object over its final pixels
// (src/cuda/cudaanalyse.cu:1906-2124); objects of level 0 kept the values of
// the first preanalysis.  One warp per object sums over the pixels; the
// moments, ellipse and area correction are finished by k_robust_finish, one
// thread per object, so that the double-precision tail does not run on one
// lane of a warp.
__global__ void __launch_bounds__(AN_WARPS * 32, AN_MINB) k_analyse_robust(AnaArgs A) {
    const int lane = threadIdx.x & 31;
    const int o = blockIdx.x * AN_WARPS + (threadIdx.x >> 5);
    if (o >= sx_count(A.nobj, A.nobj_dev) || A.O.level[o] == 0) return;
    const int n = A.O.n[o], off = A.O.off[o], w = A.w, h = A.h;
    const unsigned *pix = A.opix + off;
    const float dthresh = A.O.dthr[o];
    int flags = A.O.flags[o];

    // exact sums in double bins (hint: the object's filtered peak), or with
    // XSum when a term falls outside them or the object is too large
    const bool binned = n <= BS_MAX_TERMS;
    BinSum brv;
    bs_init(brv);
    bool ok = binned;
    const int top_c = bs_order(A.O.fdpeak[o]);
    unsigned pk = 0u, cpk = 0u;
    int xmin = 0x7fffffff, xmax = -1, ymin = 0x7fffffff, ymax = -1;
    for (int i = lane; i < n; i += 32) {
        unsigned p = __ldg(pix + i);
        int y = (int)fdiv(p, A.wdiv), x = (int)p - y * w;
        pk = max(pk, f2ord(__ldg(A.sub + p)));
        float c = __ldg(A.cd + p);
        cpk = max(cpk, f2ord(c));
        if (binned) ok &= bs_add(brv, c, top_c);
        xmin = min(xmin, x);
        xmax = max(xmax, x);
        ymin = min(ymin, y);
        ymax = max(ymax, y);
    }
    XSum srv;
    if (__all_sync(0xffffffffu, ok)) {
        srv = bs_to_xsum(bs_warp_sum(brv));
    } else {
        xs_init(srv);
        for (int i = lane; i < n; i += 32) xs_add(srv, __ldg(A.cd + __ldg(pix + i)));
        srv = xs_warp_sum(srv);
    }
    float peak = ord2f(warp_max_u(pk)), cpeak = ord2f(warp_max_u(cpk));
    xmin = warp_min_i(xmin);
    xmax = warp_max_i(xmax);
    ymin = warp_min_i(ymin);
    ymax = warp_max_i(ymax);
    if (xmin == 0 || xmax == w - 1 || ymin == 0 || ymax == h - 1) flags |= SX_OBJ_TRUNC;
    float rv = xs_float(srv);
    double dth = dthresh, dthresh2 = (dth + peak) / 2.0;
    // second pass: the moments' terms are below cpeak times the box sides
    const int bx = 32 - __clz(xmax - xmin), by = 32 - __clz(ymax - ymin), tc = bs_order(cpeak) + 1;
    BinSum bmx, bmy, bmx2, bmy2, bmxy, btv;
    bs_init(bmx);
    bs_init(bmy);
    bs_init(bmx2);
    bs_init(bmy2);
    bs_init(bmxy);
    bs_init(btv);
    ok = binned;
    const int tv_top = bs_order(peak);
    int dnpix = 0, area2 = 0;
    for (int i = lane; i < n; i += 32) {
        unsigned p = __ldg(pix + i);
        int yy = (int)fdiv(p, A.wdiv), x = (int)p - yy * w - xmin, y = yy - ymin;
        float cval = __ldg(A.cd + p), val = __ldg(A.sub + p);
        dnpix += val > dth;
        area2 += val > dthresh2;
        if (binned) {
            ok &= bs_add(btv, val, tv_top);
            ok &= bs_add(bmx, cval * x, tc + bx);
            ok &= bs_add(bmy, cval * y, tc + by);
            ok &= bs_add(bmx2, cval * x * x, tc + 2 * bx);
            ok &= bs_add(bmy2, cval * y * y, tc + 2 * by);
            ok &= bs_add(bmxy, cval * x * y, tc + bx + by);
        }
    }
    dnpix = warp_sum_i(dnpix);
    area2 = warp_sum_i(area2);
    XSum stv, smx, smy, smx2, smy2, smxy;
    if (__all_sync(0xffffffffu, ok)) {
        stv = bs_to_xsum(bs_warp_sum(btv));
        smx = bs_to_xsum(bs_warp_sum(bmx));
        smy = bs_to_xsum(bs_warp_sum(bmy));
        smx2 = bs_to_xsum(bs_warp_sum(bmx2));
        smy2 = bs_to_xsum(bs_warp_sum(bmy2));
        smxy = bs_to_xsum(bs_warp_sum(bmxy));
    } else {
        Moments6 m;
        moments_xsum(A.cd, A.sub, pix, nullptr, 0, n, A.wdiv, w, xmin, ymin, &m);
        stv = m.tv;
        smx = m.mx;
        smy = m.my;
        smx2 = m.mx2;
        smy2 = m.my2;
        smxy = m.mxy;
    }
    if (lane != 0) return;
    if (srv.ovf | stv.ovf | smx.ovf | smy.ovf | smx2.ovf | smy2.ovf | smxy.ovf) atomicOr(&A.sc->status, SX_ST_RANGE);
    RobustRaw R;
    R.mx = xs_double(smx);
    R.my = xs_double(smy);
    R.mx2 = xs_double(smx2);
    R.my2 = xs_double(smy2);
    R.mxy = xs_double(smxy);
    R.rv = rv;
    R.peak = peak;
    R.cpeak = cpeak;
    R.dnpix = dnpix;
    R.area2 = area2;
    R.xmin = xmin;
    R.xmax = xmax;
    R.ymin = ymin;
    R.ymax = ymax;
    R.flags = flags;
    A.raw[o] = R;
    A.O.dflux[o] = xs_float(stv);
}

__global__ void k_robust_finish(AnaArgs A) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= sx_count(A.nobj, A.nobj_dev) || A.O.level[o] == 0) return;
    const RobustRaw R = A.raw[o];
    const int xmin = R.xmin, ymin = R.ymin, flags = R.flags, dnpix = R.dnpix, area2 = R.area2;
    const float rv = R.rv, peak = R.peak, cpeak = R.cpeak;
    const double dth = A.O.dthr[o], dthresh2 = (dth + peak) / 2.0;
    double mxo = A.O.mx[o], myo = A.O.my[o];
    double rvd = rv, mx = R.mx, my = R.my;
    double mx2 = R.mx2, my2 = R.my2, mxy = R.mxy;
    double xm = mx / rvd, ym = my / rvd, xm2, ym2, xym;
    if (flags & SX_OBJ_MERGED) {
        double xn = mxo - xmin, yn = myo - ymin;
        xm2 = mx2 / rvd + xn * xn - 2 * xm * xn;
        ym2 = my2 / rvd + yn * yn - 2 * ym * yn;
        xym = mxy / rvd + xn * yn - xm * yn - xn * ym;
        xm = xn;
        ym = yn;
    } else {
        xm2 = mx2 / rvd - xm * xm;
        ym2 = my2 / rvd - ym * ym;
        xym = mxy / rvd - xm * ym;
    }
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
    float a = (float)sqrt(pmx2), b = (float)sqrt(pmy2);
    float abcor;
    darea = (double)area2 - dnpix;
    t1t2 = dth / dthresh2;
    if (t1t2 > 0.0) {
        abcor = (darea < 0.0 ? darea : -1.0) / (2 * SX_PI * log(t1t2 < 1.0 ? t1t2 : 0.99) * a * b);
        if (abcor > 1.0) abcor = 1.0;
    } else
        abcor = 1.0;
    A.O.flags[o] = flags;
    A.O.singu[o] = singu;
    A.O.xmin[o] = xmin;
    A.O.xmax[o] = R.xmax;
    A.O.ymin[o] = ymin;
    A.O.ymax[o] = R.ymax;
    A.O.fdflux[o] = rv;
    A.O.fdpeak[o] = cpeak;
    A.O.dpeak[o] = peak;
    A.O.dnpix[o] = dnpix;
    A.O.mx[o] = xm + xmin;
    A.O.my[o] = ym + ymin;
    A.O.mx2[o] = xm2;
    A.O.my2[o] = ym2;
    A.O.mxy[o] = xym;
    A.O.a[o] = a;
    A.O.b[o] = b;
    A.O.theta[o] = theta * 180.0 / SX_PI;
    A.O.cxx[o] = (float)(ym2 / temp2);
    A.O.cyy[o] = (float)(xm2 / temp2);
    A.O.cxy[o] = (float)(-2 * xym / temp2);
    A.O.abcor[o] = abcor;
}

// examineiso (src/cuda/cudaanalyse.cu:2176-2581) and the CLEAN threshold
// mthresh of every object.
__global__ void __launch_bounds__(AN_WARPS * 32, AN_MINB) k_examineiso(AnaArgs A) {
    __shared__ __align__(16) unsigned hist[AN_WARPS][256];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int o = blockIdx.x * AN_WARPS + wid;
    if (o >= sx_count(A.nobj, A.nobj_dev)) return;
    const int n = A.O.n[o], off = A.O.off[o], w = A.w;
    const unsigned *pix = A.opix + off;
    const float dthresh = A.O.dthr[o], thresh = A.O.athr[o], gthresh = A.sc->thresh, backsig = A.sc->backsig;
    const double mxo = A.O.mx[o], myo = A.O.my[o];
    double dbacknoise2 = backsig * backsig;
    unsigned pk = 0u;
    unsigned long long best = 0ull;
    int area = 0;
    XSum stv, svar;
    xs_init(stv);
    xs_init(svar);
    // the flux in double bins (hint: the object's peak), else with XSum
    const bool binned = n <= BS_MAX_TERMS;
    bool ok = binned;
    BinSum btv;
    bs_init(btv);
    const int tv_top = bs_order(A.O.dpeak[o]);
    double esum = 0, emx2 = 0, emy2 = 0, emxy = 0;
    for (int i = lane; i < n; i += 32) {
        unsigned p = __ldg(pix + i);
        int iy = (int)fdiv(p, A.wdiv), ix = (int)p - iy * w;
        float pv = __ldg(A.sub + p), cdpix = __ldg(A.cd + p);
        pk = max(pk, f2ord(pv));
        // first maximum of cd in raster order: max cd, then smallest index
        unsigned long long key = ((unsigned long long)f2ord(cdpix) << 32) | (unsigned)(0xffffffffu - p);
        best = max(best, key);
        // with a weight map: the pixel's own analysis threshold and variance
        const float pvar = A.wvar ? __ldg(A.wvar + p) : 0.0f;
        area += pv > sx_pix_thr(A.wthr, A.afac, pvar, gthresh);
        if (binned)
            ok &= bs_add(btv, pv, tv_top);
        if (A.wvar) xs_add(svar, pvar);
        double err = A.wvar ? (double)pvar : dbacknoise2;
        if (A.gain > 0.0 && cdpix > 0.0) err += cdpix / A.gain;
        double x = ix - mxo, y = iy - myo;
        esum += err;
        emx2 += err * x * x;
        emy2 += err * y * y;
        emxy += err * x * y;
    }
    float peak = ord2f(warp_max_u(pk));
    best = warp_max_ull(best);
    area = warp_sum_i(area);
    if (__all_sync(0xffffffffu, ok)) {
        stv = bs_to_xsum(bs_warp_sum(btv));
    } else {
        for (int i = lane; i < n; i += 32) xs_add(stv, __ldg(A.sub + __ldg(pix + i)));
        stv = xs_warp_sum(stv);
    }
    if (A.wvar) svar = xs_warp_sum(svar);
    esum = warp_sum_d(esum);
    emx2 = warp_sum_d(emx2);
    emy2 = warp_sum_d(emy2);
    emxy = warp_sum_d(emxy);
    float mthresh = 0.0f;
    if (A.clean_flag && n >= A.minarea) {
        unsigned kbits = warp_select(pix, n, A.cd, n - A.minarea, hist[wid]);
        mthresh = __uint_as_float(kbits) - dthresh;
    }
    // LOCAL photometry background (src/back.c:568 localback): the annulus mode,
    // subtracted from the flux, threshold, peak and FWHM fit (analyse.c
    // examineiso; the reference's GPU path keeps GLOBAL, dbkg = 0)
    const float dbkg = A.O.dbkg ? A.O.dbkg[o] : 0.0f;
    // isophotal thresholds: lane k < 8 evaluates threshold k, every lane reads all
    float othresh = thresh - dbkg;
    float opeak = peak - dbkg;
    float tk = 0.0f;
    if (opeak > 0.0 && othresh > 0.0 && lane < SX_NISO_)
        tk = othresh * pow((double)opeak / othresh, (double)lane / SX_NISO_);
    float threshs[SX_NISO_];
#pragma unroll
    for (int k = 0; k < SX_NISO_; k++) threshs[k] = __shfl_sync(0xffffffffu, tk, k);
    int iso[SX_NISO_];
#pragma unroll
    for (int k = 0; k < SX_NISO_; k++) iso[k] = 0;
    float thresh0 = opeak / 5.0;
    if (thresh0 < othresh) thresh0 = othresh;
    double s = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
    double sat = (double)(A.satur - (double)dbkg);
    for (int i = lane; i < n; i += 32) {
        unsigned p = __ldg(pix + i);
        float v = __ldg(A.sub + p);
        bool go = true;
#pragma unroll
        for (int k = 0; k < SX_NISO_; k++) {
            go = go && v > threshs[k];
            iso[k] += go;
        }
        double pv = v - (double)dbkg;
        if (thresh0 > 0.0 && pv > thresh0 && pv < sat) {
            int iy = (int)fdiv(p, A.wdiv), ix = (int)p - iy * w;
            double dx = ix - mxo, dy = iy - myo;
            double lpix = log(pv);
            double inverr2 = pv * pv;
            s += inverr2;
            double d2 = dx * dx + dy * dy;
            sx += d2 * inverr2;
            sxx += d2 * d2 * inverr2;
            sy += lpix * inverr2;
            sxy += lpix * d2 * inverr2;
        }
    }
#pragma unroll
    for (int k = 0; k < SX_NISO_; k++) iso[k] = warp_sum_i(iso[k]);
    s = warp_sum_d(s);
    sx = warp_sum_d(sx);
    sy = warp_sum_d(sy);
    sxx = warp_sum_d(sxx);
    sxy = warp_sum_d(sxy);
    if (lane != 0) return;
    ExamRaw X;
    X.stv = stv;
    X.svar = svar;
    X.esum = esum;
    X.emx2 = emx2;
    X.emy2 = emy2;
    X.emxy = emxy;
    X.s = s;
    X.sx = sx;
    X.sy = sy;
    X.sxx = sxx;
    X.sxy = sxy;
    X.opeak = opeak;
    X.thresh0 = thresh0;
    X.mthresh = mthresh;
    X.peakpix = (int)(0xffffffffu - (unsigned)(best & 0xffffffffu));
    X.area = area;
    A.xraw[o] = X;
#pragma unroll
    for (int k = 0; k < SX_NISO_; k++) A.O.iso[(size_t)o * SX_NISO_ + k] = iso[k];
}

// examineiso, per object: position errors, fluxes, FWHM fit, background
// (one thread per object, so that this double-precision tail does not run on
// one lane of a warp)
__global__ void k_examine_finish(AnaArgs A) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= sx_count(A.nobj, A.nobj_dev)) return;
    const ExamRaw X = A.xraw[o];
    const XSum stv = X.stv, svar = X.svar;
    double esum = X.esum, emx2 = X.emx2, emy2 = X.emy2, emxy = X.emxy;
    const double s = X.s, sx = X.sx, sy = X.sy, sxx = X.sxx, sxy = X.sxy;
    const float opeak = X.opeak, thresh0 = X.thresh0, mthresh = X.mthresh;
    const int peakpix = X.peakpix, area = X.area, n = A.O.n[o], w = A.w;
    const double mxo = A.O.mx[o], myo = A.O.my[o];
    const float backsig = A.sc->backsig;
    const double var = backsig * backsig;
    const float dbkg = A.O.dbkg ? A.O.dbkg[o] : 0.0f;
    const int singu = A.O.singu[o];
    const float fdflux = A.O.fdflux[o], a = A.O.a[o], b = A.O.b[o];
    float bkg = back_at(A.back, A.nbx, A.nby, A.bw, A.bh, (int)(mxo + 0.5), (int)(myo + 0.5));
    {
        double flux2 = fdflux * fdflux;
        emx2 /= flux2;
        emy2 /= flux2;
        emxy /= flux2;
        esum *= 0.08333 / flux2;
        if (singu && (emx2 * emy2 - emxy * emxy) < esum * esum) {
            emx2 += esum;
            emy2 += esum;
        }
    }
    double tvd = xs_double(stv);
    if (A.O.dbkg) tvd -= (double)((float)n * dbkg);   // int * float: a float product
    double sigtv = A.wvar ? xs_double(svar) : (double)n * var;
    if (A.gain > 0.0 && tvd > 0.0) sigtv += tvd / A.gain;
    float fwhm = 0.0f;
    if (thresh0 > 0.0) {
        double d = s * sxx - sx * sx;
        if (fabs(d) > 0.0) {
            double bb = -(s * sxy - sx * sy) / d, bmax;
            if (bb < (bmax = 1 / (13 * a * b))) bb = bmax;
            fwhm = (float)(1.6651 / sqrt(bb));
            if (fwhm > 0.0) fwhm -= 1 / (4 * fwhm);
        }
    }
    int py = (int)fdiv((unsigned)peakpix, A.wdiv);
    // the mode is added only where it was measured (src/back.c:659)
    A.O.bkg[o] = A.O.dbkg && A.O.lstat[o].nlevels >= 0 ? bkg + dbkg : bkg;
    A.O.peak[o] = opeak;
    A.O.peakx[o] = peakpix - py * w + 1;
    A.O.peaky[o] = py + 1;
    A.O.npix[o] = area;
    A.O.flux[o] = tvd;
    A.O.fluxerr[o] = sigtv;
    A.O.mthresh[o] = mthresh;
    A.O.pmx2[o] = emx2;
    A.O.pmy2[o] = emy2;
    A.O.pmxy[o] = emxy;
    A.O.fwhm[o] = fwhm;
    A.O.fdnpix[o] = n;
    if (stv.ovf | svar.ovf) atomicOr(&A.sc->status, SX_ST_RANGE);
}

// Object pixel lists: the objects of one raw object are consecutive and
// share out exactly its pixels, so ordering all pixels by object (raster
// order inside each object) is a stable partition of every raw object's
// pixel range by object.  One warp per raw object walks its pixels in order,
// 32 at a time; lanes holding the same object take consecutive slots from
// that object's cursor in shared memory.  A raw object that is one object is
// copied; raw objects of more than OP_KMAX objects are left to
// k_obj_partition_big (their cursors in dynamic shared memory).
constexpr int OP_WARPS = 8;
constexpr int OP_KMAX = 256;
constexpr int OP_BIG_KMAX = 12288;  // cursors of k_obj_partition_big in shared memory (48 KB)
constexpr int OP_BIG_GRID = 148;

// one warp: the raw object's pixels in order, 32 at a time, each lane's
// pixel to the next slot of its object (cursors c[0..K), any memory space)
__device__ __forceinline__ void obj_partition_walk(const unsigned *__restrict__ rpix,
                                                   const unsigned *__restrict__ objkey, int off, int P, int K, int ob,
                                                   const int *__restrict__ ooff, unsigned *__restrict__ opix, int *c) {
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < K; k += 32) c[k] = ooff[ob + k];
    __syncwarp();
    // OP_AHEAD chunks of 32 pixels per step: their loads are issued together,
    // then the chunks take their slots in order
    constexpr int OP_AHEAD = 4;
    for (int i0 = 0; i0 < P; i0 += 32 * OP_AHEAD) {
        int key[OP_AHEAD];
        unsigned px[OP_AHEAD];
#pragma unroll
        for (int a = 0; a < OP_AHEAD; a++) {
            const int i = i0 + a * 32 + lane;
            key[a] = i < P ? (int)objkey[off + i] - ob : -1;
            px[a] = i < P ? rpix[off + i] : 0u;
        }
#pragma unroll
        for (int a = 0; a < OP_AHEAD; a++) {
            const unsigned grp = __match_any_sync(0xffffffffu, key[a]);
            const int leader = __ffs(grp) - 1;
            const int rank = __popc(grp & ((1u << lane) - 1u));
            int base = 0;
            if (key[a] >= 0 && lane == leader) {
                base = c[key[a]];
                c[key[a]] = base + __popc(grp);
            }
            base = __shfl_sync(0xffffffffu, base, leader);
            if (key[a] >= 0) opix[base + rank] = px[a];
            __syncwarp();
        }
    }
}

__global__ void __launch_bounds__(OP_WARPS * 32) k_obj_partition(const unsigned *__restrict__ rpix,
                                                                 const unsigned *__restrict__ objkey,
                                                                 const int *__restrict__ roff,
                                                                 const int *__restrict__ rsize,
                                                                 const int *__restrict__ rnkept,
                                                                 const int *__restrict__ objbase,
                                                                 const int *__restrict__ ooff, int nroots,
                                                                 const int *nroots_dev, unsigned *__restrict__ opix,
                                                                 int *nbig, int *biglist) {
    __shared__ int cur[OP_WARPS][OP_KMAX];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int r = blockIdx.x * OP_WARPS + wid;
    if (r >= sx_count(nroots, nroots_dev)) return;
    const int off = roff[r], P = rsize[r], K = rnkept[r], ob = objbase[r];
    if (K <= 1) {
#pragma unroll 4
        for (int i = lane; i < P; i += 32) opix[off + i] = rpix[off + i];
        return;
    }
    if (K > OP_KMAX) {  // left to k_obj_partition_big
        if (lane == 0) biglist[atomicAdd(nbig, 1)] = r;
        return;
    }
    obj_partition_walk(rpix, objkey, off, P, K, ob, ooff, opix, cur[wid]);
}

// raw objects of more than OP_KMAX objects (the list k_obj_partition made, in
// any order: each writes its own range): one warp each, cursors in dynamic
// shared memory up to OP_BIG_KMAX objects, else in gcur (global)
__global__ void __launch_bounds__(32) k_obj_partition_big(const unsigned *__restrict__ rpix,
                                                          const unsigned *__restrict__ objkey,
                                                          const int *__restrict__ roff, const int *__restrict__ rsize,
                                                          const int *__restrict__ rnkept,
                                                          const int *__restrict__ objbase,
                                                          const int *__restrict__ ooff, const int *nbig,
                                                          const int *__restrict__ biglist,
                                                          unsigned *__restrict__ opix, int *gcur) {
    extern __shared__ int bigcur[];
    const int nb = *nbig;
    for (int i = blockIdx.x; i < nb; i += gridDim.x) {
        const int r = biglist[i], K = rnkept[r];
        const int ob = objbase[r];
        obj_partition_walk(rpix, objkey, roff[r], rsize[r], K, ob, ooff, opix,
                           K <= OP_BIG_KMAX ? bigcur : gcur + ob);
        __syncwarp();
    }
}

// gcur: scratch of one int per object; nbig (zero on entry) and biglist
// (nroots ints): the raw objects k_obj_partition leaves to the big kernel.
// nroots_dev (device, or null): the number of roots when only the device
// knows it; nroots is then the capacity.
void launch_obj_partition(const unsigned *rpix, const unsigned *objkey, const RootBufs &R, const int *ooff,
                          int nroots, const int *nroots_dev, unsigned *opix, int *gcur, int *nbig, int *biglist,
                          cudaStream_t st) {
    if (nroots <= 0) return;
    k_obj_partition<<<(unsigned)((nroots + OP_WARPS - 1) / OP_WARPS), OP_WARPS * 32, 0, st>>>(
        rpix, objkey, R.off, R.size, R.nkept, R.objbase, ooff, nroots, nroots_dev, opix, nbig, biglist);
    k_obj_partition_big<<<(unsigned)std::min(nroots, OP_BIG_GRID), 32, OP_BIG_KMAX * sizeof(int), st>>>(
        rpix, objkey, R.off, R.size, R.nkept, R.objbase, ooff, nbig, biglist, opix, gcur);
}

void launch_analyse(const AnaArgs &A, cudaStream_t st) {
    if (A.nobj <= 0) return;
    const unsigned grid = (A.nobj + AN_WARPS - 1) / AN_WARPS;
    k_analyse_robust<<<grid, AN_WARPS * 32, 0, st>>>(A);
    k_robust_finish<<<(unsigned)((A.nobj + 127) / 128), 128, 0, st>>>(A);
    if (A.O.dbkg) {
        k_local_stat<<<(unsigned)((A.nobj + 127) / 128), 128, 0, st>>>(A.sub, A.w, A.h, A.bp_thick, A.O.xmin,
                                                                         A.O.xmax, A.O.ymin, A.O.ymax, A.nobj,
                                                                         A.nobj_dev, A.O.lstat);
        k_local_guess<<<(unsigned)A.nobj, GUESS_THREADS, 0, st>>>(A.sub, A.w, A.h, A.bp_thick, A.O.xmin, A.O.xmax,
                                                                   A.O.ymin, A.O.ymax, A.nobj, A.nobj_dev, A.O.lstat,
                                                                   A.O.dbkg);
    }
    k_examineiso<<<grid, AN_WARPS * 32, 0, st>>>(A);
    k_examine_finish<<<(unsigned)((A.nobj + 127) / 128), 128, 0, st>>>(A);
}

}  // namespace sx
