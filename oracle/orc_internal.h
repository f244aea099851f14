/*
 * orc_internal.h -- oracle internals (TEST INFRASTRUCTURE ONLY, see oracle.h).
 * Constants restate src/define.h:37,56,172-177 and src/cuda/cudatypes.h:30-45.
 */
#ifndef ORC_INTERNAL_H
#define ORC_INTERNAL_H

#include <stdint.h>

#define ORC_BIG                 1e+30
void orc_local_stats(const float *buf, int n, float *bkg, float *sig);
#define ORC_BIGF                1e+30f
#define ORC_PI                  3.1415926535898
#define ORC_EPS                 (1e-4)
#define ORC_BACK_MINGOODFRAC    0.5
#define ORC_QUANTIF_NSIGMA      5
#define ORC_QUANTIF_NMAXLEVELS  4096
#define ORC_QUANTIF_AMIN        4
#define ORC_MAXDEBAREA          3
#define ORC_CLEAN_ZONE          10.0
#define ORC_APER_OVERSAMP       5
#define ORC_KRON_NSIG           (3 * 2.0)
#define ORC_CROWD_THRESHOLD     0.1

#define ORC_OBJ_CROWDED   0x0001
#define ORC_OBJ_MERGED    0x0002
#define ORC_OBJ_SATUR     0x0004
#define ORC_OBJ_TRUNC     0x0008
#define ORC_OBJ_APERT_PB  0x0010

float orc_back_at(const float *b, int nx, int ny, int backw, int backh, int x, int y);

/* exponent e0 such that 2^e0 <= v < 2^(e0+1), for v > 0 */
static inline int orc_expo(float v)
{
    union { float f; uint32_t u; } c;
    c.f = v;
    return (int)((c.u >> 23) & 0xff) - 127;
}

#endif
