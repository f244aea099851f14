/*
 * sexgpu_compat.h -- the reference's own CUDA entry points, implemented on
 * libsexgpu (library libsexgpu_compat.so).
 *
 * The reference's host code drives its GPU library through thirteen
 * extern "C" functions (src/cuda/cudainit.h, cudaback.h, cudafilter.h,
 * cudadetection.h, cudadeblend.h, cudaanalyse.h, cudaclean.h), called from
 * makeback() (src/back.c:104) and scanimage() (src/scan.c:78-147).  This
 * library exports the same thirteen names with the same arguments and the same
 * order of calls, so src/scan.c and src/back.c link against it unchanged.
 *
 * Semantics kept from the reference:
 *   - one frame at a time, process-global state (there is no context
 *     argument); the frame pointer given to init_device receives the
 *     background-subtracted image in clear_device;
 *   - back_estimate computes the background and subtracts it on the device;
 *     the caller derives dthresh/thresh from backsig (src/back.c:156-193) and
 *     passes them to run_detection;
 *   - parcel_out returns the number of objects after deblending; analyse_gpu,
 *     run_clean and endobject_gpu refer to objects by that index;
 *   - run_clean writes -1 for every object that survives CLEAN and the index of
 *     the object that absorbed it otherwise (src/scan.c:152);
 *   - endobject_gpu fills one output record per object, in object index
 *     order (src/types.h:417-455, NAPER = 1); NUMBER is left to the caller
 *     (src/scan.c:154); ALPHA/DELTA_J2000 are 0 as in the reference; CLASS_STAR
 *     (sprob) is computed when a network was given with sexgpu_compat_set_nnw
 *     (0 otherwise);
 *   - errors print "*Error*: ..." to stderr and exit the process, as the
 *     reference's checkCudaErrors/exit(-1) do (a handler can replace that).
 *
 * The pointer arguments the reference passes for its own structures
 * (prefstruct, brainstruct, obj2struct, wcsstruct) are accepted and not read:
 * their layouts belong to the reference's headers.  The photometry settings
 * the reference's endobject reads from prefstruct (MAG_ZEROPOINT,
 * PHOT_APERTURES, PHOT_AUTOPARAMS, MASK_TYPE) and BACK_VALUE for an absolute
 * background are given once with sexgpu_compat_configure; without that call
 * they have SExtractor's default values (0, 5, 2.5/3.5, CORRECT, 0).
 */
#ifndef SEXGPU_COMPAT_H
#define SEXGPU_COMPAT_H

#include <stddef.h>

#include "sexgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* src/types.h:417-455 (outobjstruct, NAPER = 1): one catalogue record */
typedef struct __attribute__((aligned(16))) {
    int number;
    double alpha2000;
    double delta2000;
    float sposx;
    float sposy;
    float flux_iso;
    float fluxerr_iso;
    float mag_iso;
    float magerr_iso;
    float flux_isocor;
    float fluxerr_isocor;
    float flux_aper[1];
    float fluxerr_aper[1];
    float mag_aper[1];
    float magerr_aper[1];
    float flux_auto;
    float fluxerr_auto;
    float mag_auto;
    float magerr_auto;
    float theta;
    double poserr_mx2;
    double poserr_my2;
    double poserr_mxy;
    short flag;
    float elong;
    float ellip;
    float sprob;
    float peak;
    float kronfactor;
    float bkg;
    float fwhm;
} sexgpu_outobj;

/* settings the reference reads from its prefstruct; see above */
void sexgpu_compat_configure(double mag_zeropoint, double phot_aperture, double autoparam0, double autoparam1,
                             int mask_type, double back_value);
/* device the state is created on (default 0); before init_device */
void sexgpu_compat_set_device(int device);
/* CLASS_STAR: the reference's brainstruct (read by getnnw, src/neurro.c)
 * in this library's layout, and prefs.seeing_fwhm; endobject_gpu's pixscale
 * argument gives the pixel scale.  NULL: CLASS_STAR (sprob) stays 0. */
void sexgpu_compat_set_nnw(const sexgpu_nnw *net, double seeing_fwhm);
/* called instead of exit() on an error, with the message */
void sexgpu_compat_set_error_handler(void (*handler)(const char *msg));

/* src/cuda/cudainit.h:11 -- copy the frame to the device */
void init_device(int width, int height, float *img);
/* src/cuda/cudainit.h:12 -- background-subtracted frame back into img */
void clear_device(float *img);
/* src/cuda/cudaback.h:5 -- background maps, subtraction, global mean/sigma */
void back_estimate(int back_size, float backfthresh, float *backmean, float *backsig, int nbackfx, int nbackfy,
                   int backtype);
/* src/cuda/cudafilter.h:11 -- square detection mask (normalised by getconv) */
void cudaFilter(float *mask, unsigned int mask_width);
/* src/cuda/cudadetection.h:11,15,16 -- filter, threshold, raw objects */
void init_detection(void);
void run_detection(float dthresh, float thresh, int minarea, size_t *numValidObj, size_t *numValidPix);
void clear_detection(void);
/* src/cuda/cudadeblend.h:11,16,23 -- multi-threshold deblending */
void init_deblend(float basethresh, int nthresh, size_t numValidObj, size_t numValidPix);
int parcel_out(float basethresh, int nthresh, int deb_minarea, size_t numValidObj, size_t numValidPix,
               double deblend_mincont);
void clear_deblend(int nthresh);
/* src/cuda/cudaanalyse.h:13 -- per-object analysis */
void analyse_gpu(double flagobj_poserr_mx2, int flagobj_peakx, int flagobj_iso_0, float flagobj_fwhm, float backsig,
                 double gain, double ngamma, float thresh, float dthresh, double satur_level, int plistexist_var,
                 int plistoff_var, int prefs_weightgain_flag, int prefs_ext_minarea, int prefs_clean_flag,
                 int detect_type, int nbackx, int nbacky, int backw, int backh, int width, int numobj);
/* src/cuda/cudaclean.h:4 -- CLEAN; returns the number of surviving objects */
int run_clean(int *masterIndex, double clean_param, int clean_stacksize, int numobj);
/* src/cuda/cudaanalyse.h:39 -- photometry and FLAGS, one record per object */
void endobject_gpu(void *prefs, void *brain, void *flagobj2, sexgpu_outobj *outobj, void *wcs, int fymin, int fymax,
                   int width, int height, float backsig, float thresh, double satur, double pixscale, double ngamma,
                   double gain, int numobj);

#ifdef __cplusplus
}
#endif

#endif
