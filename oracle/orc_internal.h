/*
 * orc_internal.h -- oracle internals (TEST INFRASTRUCTURE ONLY, see oracle.h).
 * Constants restate src/define.h:37,56,172-177 and src/cuda/cudatypes.h:30-45.
 */
#ifndef ORC_INTERNAL_H
#define ORC_INTERNAL_H

#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include "oracle.h"

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

/* one object of an extraction: its pixels, decisions and measurements
 * (orc_extract.c), shared with the FP64 twin of the measurements
 * (orc_fp64.c) */
typedef struct {
    int root, level;
    float node_dthresh;
    float dthr, athr;      /* the raw object's detection / analysis thresholds */
    float dbkg;            /* local background (BACKPHOTO_TYPE LOCAL), else 0 */
    int nnode;             /* pixels of the branch at its own level */
    int *nodepix;
    int n;                 /* final pixels (raster order) */
    int *pix;
    /* preanalysis */
    int xmin, xmax, ymin, ymax, dnpix, flags, singuflag;
    float fdflux, dflux, fdpeak, dpeak;
    double mx, my, mx2, my2, mxy;
    float a, b, theta, abcor, cxx, cyy, cxy;
    /* examineiso */
    int npix, peakx, peaky, iso[ORC_NISO];
    float flux, fluxerr, peak, bkg, thresh, mthresh, fwhm;
    double poserr_mx2, poserr_my2, poserr_mxy;
    /* clean */
    int master, final_master, fdnpix;
    /* endobject */
    float flux_isocor, fluxerr_isocor, flux_aper, fluxerr_aper, mag_aper, magerr_aper;
    float kron, flux_auto, fluxerr_auto, mag_auto, magerr_auto;
    float mag_iso, magerr_iso, fluxerr_iso;
    float elong, ellip, polar;
    float class_star;
    float aper[ORC_MAXAPER][4];  /* every aperture: flux, error, mag, mag error */
} obj_t;

typedef struct {
    int w, h;
    const float *sub, *cd;
    const orc_config *cfg;
    float dthresh, thresh, backsig;
    const float *back;
    int nbx, nby, bw, bh;
    int minarea, debminarea;
    /* weight map: calibrated variance per pixel (ORC_BIGF where unusable),
     * NULL without one; wthr: thresholds follow the local rms */
    const float *var;
    int wthr;
} frame_t;

/* Pixel thresholds with a weight map (SExtractor manual, weight maps: a
 * relative threshold is taken against the local rms): DETECT_THRESH (or
 * ANALYSIS_THRESH) x sqrt(variance); the global value otherwise. */
static inline int pix_bad(const frame_t *F, size_t p) { return F->var && !(F->var[p] < ORC_BIGF); }
static inline float pix_dthr(const frame_t *F, size_t p)
{
    return F->wthr ? (float)(F->cfg->detect_thresh * sqrt((double)F->var[p])) : F->dthresh;
}
static inline float pix_athr(const frame_t *F, size_t p)
{
    return F->wthr ? (float)(F->cfg->analysis_thresh * sqrt((double)F->var[p])) : F->thresh;
}


/* orc_fp64.c: the FP64 twin of the measurements of the catalogue rows */
void orc_measure64(const frame_t *F, const int *alloc, const obj_t *objs, int nobj, const int *rows, int nrows,
                   orc_object64 *out);

#endif
