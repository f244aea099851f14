/*
 * orc_xsum.h -- exact, order-free sums of float terms (TEST INFRASTRUCTURE ONLY).
 *
 * A sum is kept as an exact value  v * 2^(e - 23)  with v a signed 128-bit
 * integer and e the smallest binary exponent of any non-zero term seen so far.
 * Adding a term of smaller exponent rescales v (an exact left shift).  The
 * exact value does not depend on the order in which terms are added or partial
 * sums are merged, so every implementation that rounds it once gives the same
 * float/double.  Denormal terms (exponent field 0) are treated as zero.
 * If a rescale would overflow 126 bits the sum is marked invalid (ovf = 1).
 *
 * The CUDA kernels implement the same definition independently
 * (gpu-sextractor_b200/csrc/xsum.cuh); tests compare the two.
 */
#ifndef ORC_XSUM_H
#define ORC_XSUM_H
#include <stdint.h>

typedef struct {
    __int128 v;
    int e;      /* exponent of the unit: value = v * 2^(e-23) */
    int ovf;
} xsum_t;

#define XS_EMPTY 1000

static inline void xs_init(xsum_t *s) { s->v = 0; s->e = XS_EMPTY; s->ovf = 0; }

static inline int xs_bits(__int128 v)
{
    unsigned __int128 m = v < 0 ? (unsigned __int128)(-v) : (unsigned __int128)v;
    int k = 0;
    while (m) { m >>= 1; k++; }
    return k;
}

static inline void xs_rescale(xsum_t *s, int e)
{
    if (e >= s->e)
        return;
    if (s->v != 0) {
        int sh = s->e - e;
        if (sh > 125 || xs_bits(s->v) + sh > 125) {
            s->ovf = 1;
            s->v = 0;
        } else
            s->v = (__int128)((unsigned __int128)s->v << sh);
    }
    s->e = e;
}

static inline void xs_add(xsum_t *s, float f)
{
    union { float f; uint32_t u; } c;
    int ef;
    __int128 t;
    c.f = f;
    ef = (int)((c.u >> 23) & 0xff);
    if (ef == 0)
        return;
    ef -= 127;
    if (ef < s->e)
        xs_rescale(s, ef);
    {
        int sh = ef - s->e;
        uint32_t m = (c.u & 0x7fffff) | 0x800000;
        if (sh > 100) {
            s->ovf = 1;
            return;
        }
        t = (__int128)((unsigned __int128)m << sh);
    }
    if (c.u >> 31)
        s->v -= t;
    else
        s->v += t;
}

static inline void xs_merge(xsum_t *s, const xsum_t *o)
{
    xsum_t b = *o;
    if (o->ovf)
        s->ovf = 1;
    if (b.e == XS_EMPTY)
        return;
    if (s->e == XS_EMPTY) {
        s->v = b.v;
        s->e = b.e;
        return;
    }
    if (b.e < s->e)
        xs_rescale(s, b.e);
    else if (s->e < b.e)
        xs_rescale(&b, s->e);
    if (b.ovf)
        s->ovf = 1;
    s->v += b.v;
}

/* Round to the nearest double (ties to even). */
static inline double xs_double(const xsum_t *s)
{
    unsigned __int128 mag;
    uint64_t top;
    int neg, k, sc;
    double d;
    if (s->v == 0 || s->e == XS_EMPTY)
        return 0.0;
    neg = s->v < 0;
    mag = neg ? (unsigned __int128)(-s->v) : (unsigned __int128)s->v;
    k = 127;
    while (!((mag >> k) & 1))
        k--;
    if (k <= 63) {
        d = (double)(uint64_t)mag;
        sc = 0;
    } else {
        int drop = k - 63;
        unsigned __int128 rem = mag & ((((unsigned __int128)1) << drop) - 1);
        top = (uint64_t)(mag >> drop);
        if (rem)
            top |= 1;
        d = (double)top;
        sc = drop;
    }
    d = __builtin_ldexp(d, sc + s->e - 23);
    return neg ? -d : d;
}

static inline float xs_float(const xsum_t *s) { return (float)xs_double(s); }

#endif
