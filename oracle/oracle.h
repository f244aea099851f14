/*
 * oracle.h -- CPU oracle for the per-field extraction path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py use it, and only as the checker.
 *
 * What it restates (file:line of the reference project, baoxuezhao/GPU-SExtractor):
 *   background      src/back.c:214-279 (backstat), :297-339 (backhisto),
 *                   :347-432 (backguess), :434-557 (filterback),
 *                   :739-773 (makebackspline), :790-900 (subbackline),
 *                   :685-731 (back), :156-193 (thresholds in makeback);
 *                   mesh geometry src/field.c:124-135
 *   filter          src/filter.c:39-95 (convolve), :101-185 (getconv)
 *   detection       src/cuda/cudadetection.cu:36-60 (threshold), :156-276 (8-conn CCL),
 *                   :677-897 (sort/minarea prune), :899-1105 (fdpeak/fdflux)
 *   deblending      src/cuda/cudadeblend.cu:199-217 (multi-thresholds),
 *                   :223-258 (level seeds), :400-483 (MINCONT pruning),
 *                   :1262-1360 (gatherup), :1425-1776 (cut_branch)
 *   analysis        src/cuda/cudaanalyse.cu:1686-1903 (preanalyse full),
 *                   :1906-2124 (preanalyse robust), :2176-2581 (examineiso),
 *                   :62-98 (isocor), :104-287 (aper), :293-592 (auto/Kron),
 *                   :2604-2900 (endobject, SATUR)
 *   CLEAN           src/clean.c:89-180 (test arithmetic), :234-287 (mergeobject);
 *                   pair rule of src/cuda/cudaclean.cu:120-175
 *
 * Parity status: the background and filter stages are pinned bit-exactly
 * against the reference's own back.c/filter.c compiled from source
 * (oracle/Makefile -> oracle/_ref).  The detection, deblending, analysis and
 * CLEAN stages have no CPU implementation left in the reference and no golden
 * vectors in its tests: for those stages parity is unpinned beyond the
 * independent checks in tests/ (scipy connected components, exhaustive small
 * cases).
 */
#ifndef SEX_ORACLE_H
#define SEX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NISO 8

#define ORC_MAXAPER 16

typedef struct {
    /* background (src/preflist.h:48-59) */
    int     back_size;          /* BACK_SIZE, square meshes */
    int     back_filtersize;    /* BACK_FILTERSIZE, square window */
    double  back_filtthresh;    /* BACK_FILTTHRESH */
    int     back_type;          /* 0 AUTO, 1 MANUAL (absolute) */
    double  back_value;         /* BACK_VALUE */
    /* thresholds (src/preflist.h:35,81,135) */
    int     thresh_type;        /* 0 RELATIVE (sigmas), 1 ABSOLUTE (ADU) */
    double  detect_thresh;      /* DETECT_THRESH */
    double  analysis_thresh;    /* ANALYSIS_THRESH */
    /* filter */
    int     filter_flag;        /* FILTER */
    int     conv_w, conv_h;     /* normalised mask size */
    const float *conv;          /* normalised mask, row-major */
    /* detection / deblending */
    int     detect_minarea;     /* DETECT_MINAREA */
    int     deblend_nthresh;    /* DEBLEND_NTHRESH */
    double  deblend_mincont;    /* DEBLEND_MINCONT */
    /* cleaning */
    int     clean_flag;         /* CLEAN: 1 on; 0 off; 2 off, with the CLEAN inputs (mthresh) measured */
    double  clean_param;        /* CLEAN_PARAM */
    /* photometry */
    double  satur_level;        /* SATUR_LEVEL */
    double  gain;               /* GAIN */
    double  mag_zeropoint;      /* MAG_ZEROPOINT */
    double  phot_aperture;      /* PHOT_APERTURES (diameter, one aperture) */
    double  phot_autoparams[2]; /* PHOT_AUTOPARAMS */
    int     mask_type;          /* 0 NONE, 1 BLANK, 2 CORRECT */
    /* weighting */
    int     weight_type;        /* 0 NONE, 1 MAP_VAR, 2 MAP_RMS, 3 MAP_WEIGHT, 4 BACKGROUND */
    /* catalog order: 0 completion order, 1 first-pixel order */
    int     numbering;
    /* star/galaxy classification (src/preflist.h:132, SEEING_FWHM; PIXEL_SCALE) */
    double  seeing_fwhm;
    double  pixel_scale;        /* <= 0: 1 */
    const struct orc_nnw *nnw;  /* network, or NULL: CLASS_STAR 0 */
    /* photometry background (src/preflist.h BACKPHOTO_TYPE, BACKPHOTO_THICK) */
    int     back_photo_type;    /* 0 GLOBAL, 1 LOCAL */
    int     back_photo_thick;   /* annulus thickness (pixels) */
    /* several PHOT_APERTURES diameters: naper of phot_apertures[] (0: the
       single phot_aperture); the row's FLUX_APER columns hold the first */
    int     naper;
    double  phot_apertures[ORC_MAXAPER];
} orc_config;

/* Star/galaxy network (src/types.h:930 brainstruct; src/neurro.c) */
#define ORC_NNW_LAYERS 3
#define ORC_NNW_NEURONS 10
typedef struct orc_nnw {
    int32_t nlayers;
    int32_t nn[ORC_NNW_LAYERS];
    double  inbias[ORC_NNW_NEURONS], inscale[ORC_NNW_NEURONS];
    double  outbias[ORC_NNW_NEURONS], outscale[ORC_NNW_NEURONS];
    double  w[ORC_NNW_LAYERS - 1][ORC_NNW_NEURONS][ORC_NNW_NEURONS];
    double  b[ORC_NNW_LAYERS - 1][ORC_NNW_NEURONS];
} orc_nnw;

/* One catalog row; 0-based pixel coordinates unless stated. */
typedef struct {
    int32_t number;             /* NUMBER (1-based) */
    int32_t root;               /* raw object (0-based, first-pixel order) */
    int32_t level;              /* deblending level of the kept branch */
    int32_t fdnpix, dnpix, npix;
    int32_t xmin, xmax, ymin, ymax;
    int32_t peakx, peaky;       /* 1-based (FITS) */
    int32_t flags;
    int32_t iso[ORC_NISO];
    float   fdflux, dflux, flux, fluxerr, fdpeak, dpeak, peak;
    double  mx, my, mx2, my2, mxy;
    float   a, b, theta, abcor, cxx, cyy, cxy;
    float   class_star;         /* CLASS_STAR (0 without a network) */
    double  poserr_mx2, poserr_my2, poserr_mxy;
    float   bkg, thresh, dthresh, mthresh, fwhm;
    float   flux_iso, fluxerr_iso, mag_iso, magerr_iso;
    float   flux_isocor, fluxerr_isocor;
    float   flux_aper, fluxerr_aper, mag_aper, magerr_aper;
    float   kronfactor, flux_auto, fluxerr_auto, mag_auto, magerr_auto;
    float   elong, ellip, polar;
    float   aper[ORC_MAXAPER][4];  /* every aperture: flux, error, mag, mag error */
} orc_object;

typedef struct {
    /* background results */
    int     nbackx, nbacky;
    float   backmean, backsig;  /* global medians of the filtered mesh maps */
    float   dthresh, thresh;    /* detection / analysis thresholds (ADU) */
    /* counts */
    int64_t npix_above;         /* pixels with cd >= dthresh */
    int32_t nraw;               /* raw objects (area >= minarea) */
    int64_t nraw_pix;           /* pixels in raw objects */
    int32_t ndetected;          /* objects after deblending */
    int32_t nobj;               /* objects after CLEAN (catalog rows) */
    float   sigfac;             /* weight-map scale (1 without a weight map) */
} orc_summary;

/* Background only.  img is modified in place (background subtracted).
 * back/sigma (nbackx*nbacky floats each, may be NULL) receive the filtered
 * mesh maps; dback/dsigma the y-spline 2nd derivatives. */
int orc_background(float *img, int w, int h, const orc_config *cfg,
                   float *back, float *sigma, float *dback, float *dsigma,
                   orc_summary *sum);

/* Detection filter: cd = mask (x) sub, zero outside the frame. */
void orc_filter(const float *sub, int w, int h, const float *mask, int mw, int mh,
                float *cd);

/* Full extraction.  img (w*h) is the raw frame and is left unchanged; var
 * (w*h, may be NULL) is the weight map of weight_type (variance, rms or
 * weight values).
 * out_objects receives up to max_objects rows; segmap (w*h int32, may be NULL)
 * receives NUMBER per pixel (0 = sky).  Returns the number of rows or <0. */
int orc_extract(const float *img, const float *var, int w, int h, const orc_config *cfg,
                orc_object *out_objects, int max_objects, int32_t *segmap,
                float *sub_out, float *cd_out, orc_summary *sum);

/* Read and normalise a .conv mask (src/filter.c:101-185).
 * Returns number of elements, or <0 on error. */
int orc_getconv(const char *path, float *mask, int maxn, int *mw, int *mh);
/* background map (w*h), src/back.c:790 subbackline's backline */
int orc_background_map(const float *img, int w, int h, const orc_config *cfg, float *out);
/* background rms map (w*h), src/back.c:938 backrmsline */
int orc_background_rms(const float *img, int w, int h, const orc_config *cfg, float *rms);
/* src/back.c:568 localback for objects given by their boxes (4 ints each:
   xmin, xmax, ymin, ymax) over a background-subtracted frame: dbkg per object */
void orc_localback(const float *sub, int w, int h, int thick, const int *box, int nobj, float *dbkg);

/* Unit-level entry points (compared with the reference's own photom.c,
 * clean.c and neurro.c by the tests). */
typedef struct {
    double  mx, my;                       /* in: position (0-based pixels) */
    float   a, b, cxx, cyy, cxy, dbkg;    /* in: shape, local background */
    float   flux_aper, fluxerr_aper, mag_aper, magerr_aper;   /* out */
    float   kron, flux_auto, fluxerr_auto, mag_auto, magerr_auto;
    int32_t flags;                        /* out: CROWDED, APERT_PB */
} orc_phot_obj;
/* aperture (PHOT_APERTURES) and AUTO photometry over a background-subtracted
 * frame holding no other object */
int orc_photometry(const float *sub, int w, int h, const orc_config *cfg, float backsig, orc_phot_obj *o, int n);
/* FLUX_ISOCOR / FLUXERR_ISOCOR (src/photom.c:719) */
void orc_isocor(float flux, float fluxerr, int fdnpix, float dthresh, float *flux_isocor, float *fluxerr_isocor);
/* star/galaxy network response to net->nn[0] inputs (src/neurro.c:57) */
double orc_nnw_response(const orc_nnw *net, const double *input);
typedef struct {
    double  mx, my;
    float   a, b, cxx, cyy, cxy, abcor, dthresh, mthresh;
    /* merged by CLEAN into the survivor (src/clean.c:234-287) */
    int32_t fdnpix, dnpix;
    float   fdflux, dflux, flux, fluxerr, fdpeak, dpeak, peak;
    int32_t peakx, peaky, xmin, xmax, ymin, ymax, flags;
    int32_t master;                       /* out: -1 survivor, else its survivor */
} orc_clean_obj;
int orc_clean_objects(orc_clean_obj *o, int n, int w, int h, double clean_param);

/* The FP64 oracle (orc_fp64.c): the floating-point catalogue columns of an
 * extraction, recomputed in double over the same objects (the FP32 oracle's
 * segmentation, deblending, CLEAN and areas); one row per catalogue row. */
typedef struct {
    int32_t number;
    double  fdflux, dflux, flux, fluxerr, fdpeak, dpeak, peak;
    double  mx, my, mx2, my2, mxy;
    double  a, b, theta, abcor, cxx, cyy, cxy;
    double  class_star;
    double  poserr_mx2, poserr_my2, poserr_mxy;
    double  bkg, thresh, fwhm;
    double  flux_iso, fluxerr_iso, mag_iso, magerr_iso;
    double  flux_isocor, fluxerr_isocor;
    double  flux_aper, fluxerr_aper, mag_aper, magerr_aper;
    double  kronfactor, flux_auto, fluxerr_auto, mag_auto, magerr_auto;
    double  elong, ellip, polar;
} orc_object64;
/* the next orc_extract also writes the FP64 rows into out (up to max rows) */
void orc_set_fp64_rows(orc_object64 *out, int max);

/* Small helpers exposed for unit tests. */
float   orc_hmedian(float *ra, int n);
int     orc_median_walk(const int64_t *histo, int lcut, int hcut,
                        int64_t *lowsum, int64_t *highsum);
int     orc_median_mergepath(const int64_t *histo, int lcut, int hcut,
                             int64_t *lowsum, int64_t *highsum);
double  orc_xsum_floats(const float *v, int n, int e0);

#ifdef __cplusplus
}
#endif
#endif
