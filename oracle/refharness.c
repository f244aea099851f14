/*
 * refharness.c -- drives the reference's own CPU background and filter code
 * (src/back.c, src/filter.c, src/misc.c of baoxuezhao/GPU-SExtractor, compiled
 * unmodified from the reference tree by oracle/Makefile into oracle/_ref/).
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/ to pin the oracle restatement
 * (orc_back.c, orc_extract.c:orc_filter/orc_getconv) against the reference.
 *
 * The reference's makeback() (src/back.c:43) calls back_estimate(), which in
 * the reference is the CUDA driver src/cuda/cudaback.cu:1212.  This file
 * supplies a CPU back_estimate() that runs the reference's own backstat,
 * backhisto, backguess, filterback and makebackspline over every mesh of the
 * frame (the mesh loop of cudaback.cu:1212-1375), so the whole background
 * path below makeback() is reference code.  The other symbols below are stubs
 * for reference functions this path never calls.
 */
#include "config.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "define.h"
#include "globals.h"
#include "prefs.h"
#include "back.h"
#include "field.h"
#include "filter.h"

prefstruct prefs;
char gstr[MAXCHAR];
static picstruct *cur_field;

/* error() and warning() are the reference's own (src/fits/fitsmisc.c) */



/* CPU replacement of the reference's CUDA back_estimate(): every mesh of the
 * frame in raster order, partial meshes at the right/bottom edges, then the
 * reference's filterback() and makebackspline(). */
void back_estimate(int back_size, float backfthresh, float *backmean, float *backsigma,
                   int nbackfx, int nbackfy, int back_type)
{
    picstruct *field = cur_field;
    int w = field->width, h = field->height, bw = field->backw, bh = field->backh;
    int nx = field->nbackx, ny = field->nbacky, j, i;
    backstruct *bm = (backstruct *)calloc(nx, sizeof(backstruct));
    float *buf = (float *)malloc(sizeof(float) * (size_t)w * bh);
    (void)back_size; (void)backfthresh; (void)nbackfx; (void)nbackfy; (void)back_type;
    (void)backmean; (void)backsigma;

    field->back = (float *)malloc(sizeof(float) * field->nback);
    field->sigma = (float *)malloc(sizeof(float) * field->nback);
    for (j = 0; j < ny; j++) {
        int rows = (j == ny - 1 && h % bh) ? h % bh : bh;
        memcpy(buf, field->strip + (size_t)j * bh * w, sizeof(float) * (size_t)w * rows);
        memset(bm, 0, sizeof(backstruct) * nx);
        backstat(bm, buf, (size_t)w * rows, nx, w, bw);
        for (i = 0; i < nx; i++)
            if (bm[i].mean > -BIG) {
                bm[i].histo = (LONG *)calloc(bm[i].nlevels + 1, sizeof(LONG));
            }
        backhisto(bm, buf, (size_t)w * rows, nx, w, bw);
        for (i = 0; i < nx; i++) {
            backguess(&bm[i], field->back + j * nx + i, field->sigma + j * nx + i);
            free(bm[i].histo);
            bm[i].histo = NULL;
        }
    }
    free(buf);
    free(bm);
    filterback(field);
    field->dback = makebackspline(field, field->back);
    field->dsigma = makebackspline(field, field->sigma);
}

/* Background of one frame through the reference's makeback() and
 * subbackline().  img (w*h) is background-subtracted in place. */
int ref_background(float *img, int w, int h, int back_size, int back_filtersize,
                   double back_filtthresh, int back_type, double back_value,
                   double detect_thresh, double analysis_thresh,
                   float *back_out, float *sigma_out, float *stats_out)
{
    picstruct field;
    int y;

    memset(&field, 0, sizeof(field));
    memset(&prefs, 0, sizeof(prefs));
    prefs.backfthresh = back_filtthresh;
    prefs.ndthresh = prefs.nthresh = 1;
    prefs.dthresh[0] = detect_thresh;
    prefs.thresh[0] = analysis_thresh;
    prefs.thresh_type[0] = prefs.thresh_type[1] = THRESH_RELATIVE;
    prefs.back_val[0] = prefs.back_val[1] = back_value;
    prefs.detect_type = CCD;
    prefs.verbose_type = QUIET;

    field.width = w;
    field.height = h;
    field.flags = DETECT_FIELD;
    field.pixscale = 1.0;
    field.ngamma = 4.0 / log(10.0);
    /* src/field.c:124-135 */
    field.backw = back_size < w ? back_size : w;
    field.backh = back_size < h ? back_size : h;
    field.nbackp = field.backw * field.backh;
    field.nbackx = (w - 1) / field.backw + 1;
    field.nbacky = (h - 1) / field.backh + 1;
    field.nback = field.nbackx * field.nbacky;
    field.nbackfx = field.nbackx > 1 ? back_filtersize : 1;
    field.nbackfy = field.nbacky > 1 ? back_filtersize : 1;
    field.back_type = back_type ? BACK_ABSOLUTE : BACK_RELATIVE;
    field.strip = img;
    field.stripheight = h;
    field.ymin = 0;
    field.ymax = h;
    field.backline = (PIXTYPE *)malloc(sizeof(PIXTYPE) * w);
    cur_field = &field;

    makeback(&field);
    for (y = 0; y < h; y++)
        subbackline(&field, y, img + (size_t)y * w);

    if (back_out)
        memcpy(back_out, field.back, sizeof(float) * field.nback);
    if (sigma_out)
        memcpy(sigma_out, field.sigma, sizeof(float) * field.nback);
    if (stats_out) {
        stats_out[0] = field.backmean;
        stats_out[1] = field.backsig;
        stats_out[2] = field.dthresh;
        stats_out[3] = field.thresh;
    }
    free(field.back);
    free(field.sigma);
    free(field.dback);
    free(field.dsigma);
    free(field.backline);
    return 0;
}

/* The reference's LOCAL photometry background, localback() (src/back.c:568),
 * for objects given by their boxes (xmin, xmax, ymin, ymax per object) over a
 * background-subtracted frame held whole in memory (strip = frame). */
int ref_localback(const float *sub, int w, int h, int thick, const int *box, int nobj, float *dbkg)
{
    picstruct field;
    objstruct obj;
    int i;
    memset(&field, 0, sizeof(field));
    memset(&prefs, 0, sizeof(prefs));
    prefs.pback_size = thick;
    field.width = w;
    field.height = h;
    field.strip = (PIXTYPE *)sub;
    field.stripheight = h;
    field.ymin = 0;
    field.ymax = h;
    for (i = 0; i < nobj; i++) {
        memset(&obj, 0, sizeof(obj));
        obj.xmin = box[4 * i];
        obj.xmax = box[4 * i + 1];
        obj.ymin = box[4 * i + 2];
        obj.ymax = box[4 * i + 3];
        localback(&field, &obj);
        dbkg[i] = obj.dbkg;
    }
    return 0;
}

/* The background map of the reference: makeback(), then subbackline()
 * (src/back.c:790) for every row, keeping the backline it fills (what
 * src/readimage.c:114 writes to the BACKGROUND check image).  img is not
 * modified. */
int ref_background_map(const float *img, int w, int h, int back_size, int back_filtersize, double back_filtthresh,
                       int back_type, double back_value, float *out)
{
    picstruct field;
    int y;
    float *copy = (float *)malloc(sizeof(float) * (size_t)w * h);
    memcpy(copy, img, sizeof(float) * (size_t)w * h);
    memset(&field, 0, sizeof(field));
    memset(&prefs, 0, sizeof(prefs));
    prefs.backfthresh = back_filtthresh;
    prefs.ndthresh = prefs.nthresh = 1;
    prefs.dthresh[0] = prefs.thresh[0] = 1.5;
    prefs.thresh_type[0] = prefs.thresh_type[1] = THRESH_RELATIVE;
    prefs.back_val[0] = prefs.back_val[1] = back_value;
    prefs.detect_type = CCD;
    prefs.verbose_type = QUIET;
    field.width = w;
    field.height = h;
    field.flags = DETECT_FIELD;
    field.pixscale = 1.0;
    field.ngamma = 4.0 / log(10.0);
    field.backw = back_size < w ? back_size : w;
    field.backh = back_size < h ? back_size : h;
    field.nbackp = field.backw * field.backh;
    field.nbackx = (w - 1) / field.backw + 1;
    field.nbacky = (h - 1) / field.backh + 1;
    field.nback = field.nbackx * field.nbacky;
    field.nbackfx = field.nbackx > 1 ? back_filtersize : 1;
    field.nbackfy = field.nbacky > 1 ? back_filtersize : 1;
    field.back_type = back_type ? BACK_ABSOLUTE : BACK_RELATIVE;
    field.strip = copy;
    field.stripheight = h;
    field.ymin = 0;
    field.ymax = h;
    field.backline = (PIXTYPE *)malloc(sizeof(PIXTYPE) * w);
    cur_field = &field;
    makeback(&field);
    for (y = 0; y < h; y++) {
        subbackline(&field, y, copy + (size_t)y * w);
        memcpy(out + (size_t)y * w, field.backline, sizeof(float) * w);
    }
    free(field.back);
    free(field.sigma);
    free(field.dback);
    free(field.dsigma);
    free(field.backline);
    free(copy);
    return 0;
}

/* The background rms map of the reference: makeback(), then backrmsline()
 * (src/back.c:938) for every row.  img is not modified. */
int ref_background_rms(const float *img, int w, int h, int back_size, int back_filtersize,
                       double back_filtthresh, float *rms)
{
    picstruct field;
    int y;
    float *copy = (float *)malloc(sizeof(float) * (size_t)w * h);
    memcpy(copy, img, sizeof(float) * (size_t)w * h);
    memset(&field, 0, sizeof(field));
    memset(&prefs, 0, sizeof(prefs));
    prefs.backfthresh = back_filtthresh;
    prefs.ndthresh = prefs.nthresh = 1;
    prefs.dthresh[0] = prefs.thresh[0] = 1.5;
    prefs.thresh_type[0] = prefs.thresh_type[1] = THRESH_RELATIVE;
    prefs.detect_type = CCD;
    prefs.verbose_type = QUIET;
    field.width = w;
    field.height = h;
    field.flags = DETECT_FIELD;
    field.pixscale = 1.0;
    field.ngamma = 4.0 / log(10.0);
    field.backw = back_size < w ? back_size : w;
    field.backh = back_size < h ? back_size : h;
    field.nbackp = field.backw * field.backh;
    field.nbackx = (w - 1) / field.backw + 1;
    field.nbacky = (h - 1) / field.backh + 1;
    field.nback = field.nbackx * field.nbacky;
    field.nbackfx = field.nbackx > 1 ? back_filtersize : 1;
    field.nbackfy = field.nbacky > 1 ? back_filtersize : 1;
    field.back_type = BACK_RELATIVE;
    field.strip = copy;
    field.stripheight = h;
    field.ymin = 0;
    field.ymax = h;
    field.backline = (PIXTYPE *)malloc(sizeof(PIXTYPE) * w);
    cur_field = &field;
    makeback(&field);
    for (y = 0; y < h; y++)
        backrmsline(&field, y, rms + (size_t)y * w);
    free(field.back);
    free(field.sigma);
    free(field.dback);
    free(field.dsigma);
    free(field.backline);
    free(copy);
    return 0;
}

/* Read a .conv file with the reference's getconv(); returns the mask size. */
int ref_getconv(const char *path, float *mask, int maxn, int *mw, int *mh)
{
    int n;
    thefilter = (filterstruct *)calloc(1, sizeof(filterstruct));
    if (getconv((char *)path) != RETURN_OK)
        return -1;
    n = thefilter->convw * thefilter->convh;
    if (n > maxn)
        return -2;
    memcpy(mask, thefilter->conv, sizeof(float) * n);
    *mw = thefilter->convw;
    *mh = thefilter->convh;
    free(thefilter->conv);
    free(thefilter);
    thefilter = NULL;
    return n;
}

/* Filter a background-subtracted frame with the reference's convolve(). */
int ref_convolve(float *sub, int w, int h, const float *mask, int mw, int mh, float *cd)
{
    picstruct field;
    int y;
    memset(&field, 0, sizeof(field));
    thefilter = (filterstruct *)calloc(1, sizeof(filterstruct));
    thefilter->conv = (float *)mask;
    thefilter->convw = mw;
    thefilter->convh = mh;
    thefilter->nconv = mw * mh;
    field.width = w;
    field.height = h;
    field.strip = sub;
    field.stripheight = h;
    field.ymin = 0;
    field.ymax = h;
    for (y = 0; y < h; y++) {
        field.y = y;
        convolve(&field, cd + (size_t)y * w);
    }
    free(thefilter);
    thefilter = NULL;
    return 0;
}
