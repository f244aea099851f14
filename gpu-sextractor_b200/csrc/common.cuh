// common.cuh -- shared device helpers for libsexgpu (sm_100a).
//
// Compiled with -fmad=false: every floating-point expression below evaluates
// with separately rounded IEEE operations in the order written, the same
// arithmetic the reference's host C code performs.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define SX_BIG 1e+30
// blank (NaN) input pixels read as -BIG, like the FITS reader's blank value
__device__ __forceinline__ float sx_unblank(float v) { return v != v ? -1e+30f : v; }
#define SX_PI 3.1415926535898
#define SX_EPS (1e-4)
#define SX_BACK_MINGOODFRAC 0.5
#define SX_QUANTIF_NSIGMA 5
#define SX_QUANTIF_NMAXLEVELS 4096
#define SX_QUANTIF_AMIN 4
#define SX_MAXDEBAREA 3
#define SX_CLEAN_ZONE 10.0
#define SX_APER_OVERSAMP 5
#define SX_KRON_NSIG (3 * 2.0)
#define SX_CROWD_THRESHOLD 0.1
#define SX_MAXCONV 31
#define SX_NISO_ 8

// object flags, src/cuda/cudatypes.h:30-37
#define SX_OBJ_CROWDED 0x0001
#define SX_OBJ_MERGED 0x0002
#define SX_OBJ_SATUR 0x0004
#define SX_OBJ_TRUNC 0x0008
#define SX_OBJ_APERT_PB 0x0010

// device status word bits
#define SX_ST_RANGE 1
#define SX_ST_LOOP 2
#define SX_ST_CAPACITY 4  // a count beyond the capacity a captured pipeline was sized for
#define SX_ST_LOAD 8     // a tile load of the subtract/filter pipeline did not complete in time
#define SX_ST_THRESH 16   // zero or negative detection or analysis threshold
#define SX_ST_STOP (SX_ST_RANGE | SX_ST_LOOP | SX_ST_CAPACITY | SX_ST_LOAD | SX_ST_THRESH)

// A count known on the device only: *n_dev, at most the capacity n the launch
// was sized for; n itself when n_dev is null (the count known on the host).
__device__ __forceinline__ int sx_count(int n, const int *n_dev) { return n_dev ? min(n, max(*n_dev, 0)) : n; }

#define SX_ALLOC_OTHER 0x7fffffff

// ---------------------------------------------------------------------------
// Exact, order-free sums of float terms.
//
// The value v * 2^(e-23) is exact; e is the smallest binary exponent of the
// non-zero terms seen so far.  Adding a smaller-exponent term shifts v left
// (exactly).  Any order of adds and merges gives the same exact value, which
// is rounded once when read; denormal terms count as zero; a sum whose
// dynamic range would exceed 125 bits raises ovf.
// ---------------------------------------------------------------------------
#define XS_EMPTY 1000

struct XSum {
    __int128 v;
    int e;
    int ovf;
};

__device__ __forceinline__ void xs_init(XSum &s) {
    s.v = 0;
    s.e = XS_EMPTY;
    s.ovf = 0;
}

__device__ __forceinline__ int xs_bits(__int128 v) {
    unsigned __int128 m = v < 0 ? (unsigned __int128)(-v) : (unsigned __int128)v;
    unsigned long long hi = (unsigned long long)(m >> 64), lo = (unsigned long long)m;
    if (hi) return 128 - __clzll(hi);
    if (lo) return 64 - __clzll(lo);
    return 0;
}

__device__ __forceinline__ void xs_rescale(XSum &s, int e) {
    if (e >= s.e) return;
    if (s.v != 0) {
        int sh = s.e - e;
        if (sh > 125 || xs_bits(s.v) + sh > 125) {
            s.ovf = 1;
            s.v = 0;
        } else {
            s.v = (__int128)((unsigned __int128)s.v << sh);
        }
    }
    s.e = e;
}

__device__ __forceinline__ void xs_add(XSum &s, float f) {
    unsigned int u = __float_as_uint(f);
    int ef = (int)((u >> 23) & 0xff);
    if (ef == 0) return;
    ef -= 127;
    if (ef < s.e) xs_rescale(s, ef);
    int sh = ef - s.e;
    if (sh > 100) {
        s.ovf = 1;
        return;
    }
    unsigned int m = (u & 0x7fffffu) | 0x800000u;
    __int128 t = (__int128)((unsigned __int128)m << sh);
    if (u >> 31)
        s.v -= t;
    else
        s.v += t;
}

__device__ __forceinline__ void xs_merge(XSum &s, XSum b) {
    if (b.ovf) s.ovf = 1;
    if (b.e == XS_EMPTY) return;
    if (s.e == XS_EMPTY) {
        s.v = b.v;
        s.e = b.e;
        return;
    }
    if (b.e < s.e)
        xs_rescale(s, b.e);
    else if (s.e < b.e)
        xs_rescale(b, s.e);
    if (b.ovf) s.ovf = 1;
    s.v += b.v;
}

// exact value -> nearest double (ties to even)
__device__ __forceinline__ double xs_double(const XSum &s) {
    if (s.v == 0 || s.e == XS_EMPTY) return 0.0;
    bool neg = s.v < 0;
    unsigned __int128 mag = neg ? (unsigned __int128)(-s.v) : (unsigned __int128)s.v;
    unsigned long long hi = (unsigned long long)(mag >> 64), lo = (unsigned long long)mag;
    double d;
    int sc;
    if (!hi) {
        d = __ull2double_rn(lo);
        sc = 0;
    } else {
        int k = 127 - __clzll(hi);  // msb position
        int drop = k - 63;
        unsigned long long top = (unsigned long long)(mag >> drop);
        unsigned __int128 rem = mag & ((((unsigned __int128)1) << drop) - 1);
        if (rem) top |= 1ull;
        d = __ull2double_rn(top);
        sc = drop;
    }
    d = scalbn(d, sc + s.e - 23);
    return neg ? -d : d;
}

__device__ __forceinline__ float xs_float(const XSum &s) { return (float)xs_double(s); }

__device__ __forceinline__ XSum xs_shfl_down(const XSum &s, int off) {
    XSum r;
    unsigned long long lo = (unsigned long long)s.v, hi = (unsigned long long)(s.v >> 64);
    lo = __shfl_down_sync(0xffffffffu, lo, off);
    hi = __shfl_down_sync(0xffffffffu, hi, off);
    r.v = (__int128)(((unsigned __int128)hi << 64) | lo);
    r.e = __shfl_down_sync(0xffffffffu, s.e, off);
    r.ovf = __shfl_down_sync(0xffffffffu, s.ovf, off);
    return r;
}

// full-warp reduction by a merge tree; the result is valid in lane 0
__device__ __noinline__ XSum xs_warp_reduce_tree(XSum s) {
    for (int off = 16; off > 0; off >>= 1) xs_merge(s, xs_shfl_down(s, off));
    return s;
}

// Full-warp exact sum, valid in every lane.  Every lane's value is brought to
// the warp's smallest exponent; when each then fits in 122 bits the 32 of them
// add in an int128 without overflow (a butterfly of plain integer adds).
// Otherwise the merge tree above decides, with its range check.  The exact
// value, and so every rounding of it, is the same either way.
__device__ __forceinline__ XSum xs_warp_sum(XSum s) {
    int emin = s.e;
    for (int o = 16; o > 0; o >>= 1) emin = min(emin, __shfl_xor_sync(0xffffffffu, emin, o));
    int ovf = __any_sync(0xffffffffu, s.ovf);
    XSum r;
    r.e = emin;
    r.ovf = ovf;
    r.v = 0;
    if (emin == XS_EMPTY) return r;
    bool fits = true;
    __int128 v = 0;
    if (s.e != XS_EMPTY && s.v != 0) {
        int sh = s.e - emin;
        if (sh > 122 || xs_bits(s.v) + sh > 122)
            fits = false;
        else
            v = (__int128)((unsigned __int128)s.v << sh);
    }
    if (__all_sync(0xffffffffu, fits)) {
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long lo = (unsigned long long)v, hi = (unsigned long long)(v >> 64);
            lo = __shfl_xor_sync(0xffffffffu, lo, o);
            hi = __shfl_xor_sync(0xffffffffu, hi, o);
            v += (__int128)(((unsigned __int128)hi << 64) | lo);
        }
        r.v = v;
        return r;
    }
    s = xs_warp_reduce_tree(s);
    unsigned long long lo = (unsigned long long)s.v, hi = (unsigned long long)(s.v >> 64);
    lo = __shfl_sync(0xffffffffu, lo, 0);
    hi = __shfl_sync(0xffffffffu, hi, 0);
    r.v = (__int128)(((unsigned __int128)hi << 64) | lo);
    r.e = __shfl_sync(0xffffffffu, s.e, 0);
    r.ovf = __shfl_sync(0xffffffffu, s.ovf, 0);
    return r;
}

// the same, for callers that read the result in lane 0 only
__device__ __forceinline__ XSum xs_warp_reduce(XSum s) { return xs_warp_sum(s); }

// ---------------------------------------------------------------------------
// Exact sums of float terms, binned form: three double bins of 16 binary
// orders each, the top one ending at the order `top` (a hint, for instance
// the order of the largest term expected).  A term of order e = exponent
// field - 127 goes to bin k = (top - e) >> 4 when 0 <= k <= 2: it is a
// multiple of 2^(top-16k-38) below 2^(top-16k+1), so up to 2^14 such terms
// (of one bin, over every lane that adds them up) sum below 2^53 units of
// 2^(top-16k-38), and every double addition in the bin is exact.  A nonzero
// term outside the bins is not added and makes bs_add return false; the
// caller then takes the sum again with XSum.  Zero and subnormal terms add
// nothing, as in xs_add, so a valid binned sum moved into an XSum has exactly
// the value the XSum of the same terms has.  The hint only decides which
// terms fit: a wrong one costs a second pass, never a different result.
// ---------------------------------------------------------------------------
constexpr int BS_MAX_TERMS = 1 << 14;  // terms per sum (all lanes together)

struct BinSum {
    double b0, b1, b2;
};

__device__ __forceinline__ void bs_init(BinSum &s) { s.b0 = s.b1 = s.b2 = 0.0; }

__device__ __forceinline__ bool bs_add(BinSum &s, float f, int top) {
    const unsigned u = __float_as_uint(f);
    const int ef = (int)((u >> 23) & 0xff);
    if (ef == 0) return true;
    const int k = (top + 127 - ef) >> 4;
    const double d = (double)f;
    s.b0 += k == 0 ? d : 0.0;
    s.b1 += k == 1 ? d : 0.0;
    s.b2 += k == 2 ? d : 0.0;
    return (unsigned)k < 3u;
}

// order of a float for the hint: exponent field - 127 (-127 for 0)
__device__ __forceinline__ int bs_order(float f) { return (int)((__float_as_uint(f) >> 23) & 0xff) - 127; }

// full-warp sum of the bins (exact: each bin's terms over the warp number
// at most BS_MAX_TERMS); valid in every lane
__device__ __forceinline__ BinSum bs_warp_sum(BinSum s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s.b0 += __shfl_xor_sync(0xffffffffu, s.b0, o);
        s.b1 += __shfl_xor_sync(0xffffffffu, s.b1, o);
        s.b2 += __shfl_xor_sync(0xffffffffu, s.b2, o);
    }
    return s;
}

// s += d exactly, for a double d that is a multiple of a power of two no
// smaller than 2^-1074 (every bin sum is)
__device__ __forceinline__ void xs_add_double(XSum &s, double d) {
    if (d == 0.0) return;
    const unsigned long long u = (unsigned long long)__double_as_longlong(d);
    const int ed = (int)((u >> 52) & 0x7ff);
    unsigned long long m = u & 0xfffffffffffffull;
    if (ed) m |= 1ull << 52;
    const int tz = __ffsll((long long)m) - 1;
    m >>= tz;
    // d = m * 2^(te - 23) in the units of xs_add
    const int te = (ed ? ed : 1) - 1075 + tz + 23;
    if (te < s.e) xs_rescale(s, te);
    const int sh = te - s.e;
    if (sh + (64 - __clzll(m)) > 125) {
        s.ovf = 1;
        return;
    }
    const __int128 t = (__int128)((unsigned __int128)m << sh);
    if (u >> 63)
        s.v -= t;
    else
        s.v += t;
}

// (out of line: called once per sum and object, it keeps one copy of the
// conversion in the instruction cache instead of one per sum)
__device__ __noinline__ XSum bs_to_xsum(const BinSum &b) {
    XSum x;
    xs_init(x);
    xs_add_double(x, b.b2);
    xs_add_double(x, b.b1);
    xs_add_double(x, b.b0);
    return x;
}

// ---------------------------------------------------------------------------
// Fixed-scale exact accumulators usable with atomics: value =
// sum_k (int64)w[k] * 2^(32k) in units of 2^(e0-23).  A float term of
// exponent e >= e0 is split into 32-bit limbs; each limb word stays exact for
// up to 2^31 terms.
// ---------------------------------------------------------------------------
struct Limbs4 {
    unsigned long long w[4];
};

__device__ __forceinline__ void limbs_term(float f, int e0, unsigned int lim[4], bool &neg, int &bad) {
    unsigned int u = __float_as_uint(f);
    int ef = (int)((u >> 23) & 0xff);
    lim[0] = lim[1] = lim[2] = lim[3] = 0;
    neg = (u >> 31) != 0;
    if (ef == 0) return;
    int sh = ef - 127 - e0;
    if (sh < 0 || sh > 100) {
        bad = 1;
        return;
    }
    unsigned __int128 t = ((unsigned __int128)((u & 0x7fffffu) | 0x800000u)) << sh;
    lim[0] = (unsigned int)t;
    lim[1] = (unsigned int)(t >> 32);
    lim[2] = (unsigned int)(t >> 64);
    lim[3] = (unsigned int)(t >> 96);
}

__device__ __forceinline__ void limbs_atomic_add_term(unsigned long long *acc, float f, int e0, int *status) {
    unsigned int lim[4];
    bool neg;
    int bad = 0;
    limbs_term(f, e0, lim, neg, bad);
    if (bad) {
        atomicOr(status, SX_ST_RANGE);
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; k++)
        if (lim[k]) atomicAdd(acc + k, neg ? (unsigned long long)(-(long long)lim[k]) : (unsigned long long)lim[k]);
}

__device__ __forceinline__ XSum limbs_to_xsum(const unsigned long long *w, int e0) {
    XSum s;
    __int128 v = 0;
#pragma unroll
    for (int k = 3; k >= 0; k--) v = (v << 32) + (__int128)(long long)w[k];
    s.v = v;
    s.e = e0;
    s.ovf = 0;
    return s;
}

// orderable integer image of a float (monotone for all finite floats)
__device__ __forceinline__ unsigned int f2ord(float f) {
    unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned int o) {
    unsigned int u = (o & 0x80000000u) ? (o & 0x7fffffffu) : ~o;
    return __uint_as_float(u);
}

// Division of a pixel index by the frame width without the integer divide:
// q = floor(p * m / 2^64) with m = ceil(2^64 / d) is exact whenever
// p * d < 2^64, which holds for any 32-bit p and d.  d == 1 is m == 0.
struct FastDiv {
    unsigned long long m;
    unsigned d;
};
inline FastDiv make_fastdiv(unsigned d) {
    FastDiv f;
    f.d = d;
    f.m = d > 1 ? (~0ull) / d + 1 : 0ull;
    return f;
}
__device__ __forceinline__ FastDiv make_fastdiv_dev(unsigned d) {
    FastDiv f;
    f.d = d;
    f.m = d > 1 ? (~0ull) / d + 1 : 0ull;
    return f;
}
__device__ __forceinline__ unsigned fdiv(unsigned p, const FastDiv &f) {
    return f.m ? (unsigned)__umul64hi((unsigned long long)p, f.m) : p;
}

// The six exact moment sums of a preanalysis with XSum (warp-collective):
// sub values and cd x^a y^b terms over pixels pix[i] (or pix[list[base + i]]),
// x, y relative to (x0, y0).  Not inlined: the rare path when binned sums do
// not hold the terms, kept out of the callers' registers.
struct Moments6 {
    XSum tv, mx, my, mx2, my2, mxy;
};

__device__ __noinline__ void moments_xsum(const float *cd, const float *sub, const unsigned *pix,
                                          const unsigned short *list, int base, int n, FastDiv wdiv, int w, int x0,
                                          int y0, Moments6 *out) {
    Moments6 m;
    xs_init(m.tv);
    xs_init(m.mx);
    xs_init(m.my);
    xs_init(m.mx2);
    xs_init(m.my2);
    xs_init(m.mxy);
    for (int i = threadIdx.x & 31; i < n; i += 32) {
        const unsigned p = pix[list ? list[base + i] : i];
        const int yy = (int)fdiv(p, wdiv), x = (int)p - yy * w - x0, y = yy - y0;
        const float cval = cd[p], val = sub[p];
        xs_add(m.mx, cval * x);
        xs_add(m.my, cval * y);
        xs_add(m.mx2, cval * x * x);
        xs_add(m.my2, cval * y * y);
        xs_add(m.mxy, cval * x * y);
        xs_add(m.tv, val);
    }
    m.tv = xs_warp_sum(m.tv);
    m.mx = xs_warp_sum(m.mx);
    m.my = xs_warp_sum(m.my);
    m.mx2 = xs_warp_sum(m.mx2);
    m.my2 = xs_warp_sum(m.my2);
    m.mxy = xs_warp_sum(m.mxy);
    *out = m;
}


__device__ __forceinline__ int fexpo(float v) { return (int)((__float_as_uint(v) >> 23) & 0xff) - 127; }

// bilinear background at (x, y), src/back.c:685-731
__device__ __forceinline__ float back_at(const float *b, int nx, int ny, int backw, int backh, int x, int y) {
    int xl, yl, pos;
    double dx, dy, cdx;
    float b0, b1, b2, b3;
    dx = (double)x / backw - 0.5;
    dy = (double)y / backh - 0.5;
    dx -= (xl = (int)dx);
    dy -= (yl = (int)dy);
    if (xl < 0) {
        xl = 0;
        dx -= 1.0;
    } else if (xl >= nx - 1) {
        xl = nx < 2 ? 0 : nx - 2;
        dx += 1.0;
    }
    if (yl < 0) {
        yl = 0;
        dy -= 1.0;
    } else if (yl >= ny - 1) {
        yl = ny < 2 ? 0 : ny - 2;
        dy += 1.0;
    }
    pos = yl * nx + xl;
    cdx = 1 - dx;
    b += pos;
    b0 = *b;
    b1 = nx < 2 ? b0 : *(++b);
    b2 = ny < 2 ? *b : *(b += nx);
    b3 = nx < 2 ? *b : *(--b);
    return (float)((1 - dy) * (cdx * b0 + dx * b1) + dy * (dx * b2 + cdx * b3));
}

// ---------------------------------------------------------------------------
// Device-side parameters of one extraction
// ---------------------------------------------------------------------------
struct FrameParams {
    int w, h;
    int bw, bh, nbx, nby;           // meshes
    int nfx, nfy;                   // mesh filter window
    float fthresh;                  // BACK_FILTTHRESH
    int back_type;
    float back_value;
    int thresh_type;
    double detect_thresh, analysis_thresh;
    int conv_w, conv_h, filter_flag;
    int minarea, debminarea, nthresh;
    double mincont;
    int clean_flag;
    double clean_param;
    double satur_level, gain, mag_zeropoint, aperture;
    int naper;                      // PHOT_APERTURES diameters (>= 1); aperture = apertures[0]
    double apertures[SEXGPU_MAXAPER];
    double autoparam0, autoparam1;
    int mask_type, numbering;
    int wtype;                      // weight map: 0 none, 1 MAP_VAR, 2 MAP_RMS, 3 MAP_WEIGHT
    int wthr;                       // thresholds follow the local rms (weight map, relative thresholds)
    double seeing, pixscale;        // SEEING_FWHM, PIXEL_SCALE (CLASS_STAR)
    int bp_local, bp_thick;         // BACKPHOTO_TYPE LOCAL, BACKPHOTO_THICK
    int loop_cap;                   // > 0: cap on union-find walks and retries (failure tests); 0: built-in caps
};

// scalars computed on the device during one extraction
struct FrameScalars {
    float backmean, backsig, dthresh, thresh;
    float sigfac;                   // weight-map scale factor (1 without a map)
    int e0cd;                       // exponent of dthresh (all object cd >= dthresh)
    int status;                     // SX_ST_* bits
    int npix_above;
    int nroots;
    int nrootpix;
    int nobj;                       // objects after deblending
    int nsurv;                      // after CLEAN
    int e0sub;                      // smallest exponent of a non-zero |sub|
    int kitems[2], kchunks[2];      // queued Kron boxes and their work items (pass 1, 2)
    int nvbig;                      // CLEAN victims when too many for the one-block sort, else 0
    int nbig;                       // raw objects of more than 256 objects (their list: k_obj_partition)
    unsigned long long levpix;      // sum of the deblending level of every raw-object pixel
};

// ---------------------------------------------------------------------------
// Weight maps (restated after the SExtractor manual and src/weight.c:91-125;
// the reference has no weighted path).  Relative variance of a weight value:
// MAP_VAR v, MAP_RMS v^2, MAP_WEIGHT 1/v; calibrated variance: MAP_VAR
// v*sigfac^2, MAP_RMS v^2, MAP_WEIGHT sigfac^2/v.  NaN, a variance or rms at
// or above BIG and a weight at or below 0 are unusable (BIG).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ float sx_rel_var(float v, int wtype) {
    float r;
    if (wtype == 1)
        r = v;
    else if (wtype == 2)
        r = v < 1e30f ? v * v : 1e30f;
    else
        r = v > 0.0f ? 1.0f / v : 1e30f;
    return r < 1e30f ? r : 1e30f;
}

__host__ __device__ __forceinline__ float sx_calib_var(float v, int wtype, float sigfac2) {
    float r;
    if (wtype == 1)
        r = v < 1e30f ? v * sigfac2 : 1e30f;
    else if (wtype == 2)
        r = v < 1e30f ? v * v : 1e30f;
    else
        r = v > 0.0f ? sigfac2 / v : 1e30f;
    return r < 1e30f ? r : 1e30f;
}

// detection / analysis threshold at a pixel of calibrated variance var
__device__ __forceinline__ float sx_pix_thr(bool wthr, double fac, float var, float global) {
    return wthr ? (float)(fac * sqrt((double)var)) : global;
}

