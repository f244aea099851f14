/*
 * refscan.c -- the reference's own host extraction code linked unchanged
 * against libsexgpu_compat.so (TEST INFRASTRUCTURE ONLY: the drop-in check).
 *
 * oracle/Makefile compiles the reference's src/scan.c, src/back.c and
 * src/misc.c unmodified and links them with this driver and
 * gpu-sextractor_b200/libsexgpu_compat.so into oracle/_ref/ref_scan.  The
 * driver does for one frame what the reference's makeit() does
 * (src/makeit.c:164-228): it fills prefs and the field the way readprefs(),
 * useprefs() and newfield() would (src/prefs.c:446-470, src/field.c:124-135),
 * copies the frame to the device with init_device() (src/makeit.c:189), then
 * calls the reference's makeback() (src/makeit.c:195) and scanimage()
 * (:207).  scanimage() drives the thirteen entry points and prints the
 * catalogue through the reference's printobj() (src/scan.c:331) into the
 * output file.  The one call it adds is sexgpu_compat_configure(): the
 * photometry settings the library cannot read from the reference's
 * prefstruct (its layout belongs to the reference's headers).
 *
 * usage: ref_scan frame.f32 W H mask.f32 MW MH out.cat BACK_SIZE
 *        BACK_FILTERSIZE BACK_FILTTHRESH DETECT_THRESH ANALYSIS_THRESH MINAREA
 *        NTHRESH MINCONT CLEAN CLEAN_PARAM GAIN SATUR
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
#include "sexgpu_compat.h"

/* globals the reference defines in files this driver does not link
 * (src/globals.c, src/catout.c, src/neurro.c, src/fits/fitsmisc.c) */
prefstruct prefs;
objstruct flagobj;
obj2struct flagobj2;
brainstruct *brain;
FILE *ascfile;
char gstr[MAXCHAR];

void error(int num, char *msg1, char *msg2)
{
    fprintf(stderr, "\n> %s%s\n\n", msg1, msg2);
    exit(num);
}

void warning(char *msg1, char *msg2) { fprintf(stderr, "\n> WARNING: %s%s\n\n", msg1, msg2); }

static void *slurp(const char *path, size_t bytes)
{
    FILE *f = fopen(path, "rb");
    void *p = malloc(bytes);
    if (!f || !p || fread(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(2);
    }
    fclose(f);
    return p;
}

int main(int argc, char **argv)
{
    picstruct field;
    int w, h, mw, mh, back_size, nbackf;
    if (argc != 20) {
        fprintf(stderr, "usage: see the header of oracle/refscan.c\n");
        return 2;
    }
    w = atoi(argv[2]);
    h = atoi(argv[3]);
    mw = atoi(argv[5]);
    mh = atoi(argv[6]);
    back_size = atoi(argv[8]);
    nbackf = atoi(argv[9]);

    /* readprefs()/useprefs(): the settings of this run */
    memset(&prefs, 0, sizeof(prefs));
    prefs.backfthresh = atof(argv[10]);
    prefs.ndthresh = prefs.nthresh = 1;
    prefs.dthresh[0] = atof(argv[11]);
    prefs.thresh[0] = atof(argv[12]);
    prefs.thresh_type[0] = prefs.thresh_type[1] = THRESH_RELATIVE;
    prefs.ext_minarea = atoi(argv[13]);
    prefs.deb_maxarea = prefs.ext_minarea < MAXDEBAREA ? prefs.ext_minarea : MAXDEBAREA; /* src/prefs.c:463 */
    prefs.deblend_nthresh = atoi(argv[14]);
    prefs.deblend_mincont = atof(argv[15]);
    prefs.clean_flag = atoi(argv[16]);
    prefs.clean_param = atof(argv[17]);
    prefs.clean_stacksize = 3000;
    prefs.detect_type = CCD;
    prefs.verbose_type = QUIET;
    prefs.mag_zeropoint = 0.0;
    prefs.apert[0] = 5.0;
    prefs.autoparam[0] = 2.5;
    prefs.autoparam[1] = 3.5;
    prefs.mask_type = MASK_CORRECT;

    /* the detection filter, as getconv() leaves it (src/filter.c:101) */
    thefilter = (filterstruct *)calloc(1, sizeof(filterstruct));
    thefilter->conv = (float *)slurp(argv[4], sizeof(float) * (size_t)mw * mh);
    thefilter->convw = mw;
    thefilter->convh = mh;
    thefilter->nconv = mw * mh;

    /* newfield(): the frame, held whole in memory (src/makeit.c:181-184) */
    memset(&field, 0, sizeof(field));
    field.width = w;
    field.height = h;
    field.flags = DETECT_FIELD;
    field.pixscale = 1.0;
    field.gain = atof(argv[18]);
    field.satur_level = atof(argv[19]);
    field.ngamma = 4.0 / log(10.0);
    field.backw = back_size < w ? back_size : w;
    field.backh = back_size < h ? back_size : h;
    field.nbackp = field.backw * field.backh;
    field.nbackx = (w - 1) / field.backw + 1;
    field.nbacky = (h - 1) / field.backh + 1;
    field.nback = field.nbackx * field.nbacky;
    field.nbackfx = field.nbackx > 1 ? nbackf : 1;
    field.nbackfy = field.nbacky > 1 ? nbackf : 1;
    field.back_type = BACK_RELATIVE;
    field.strip = (PIXTYPE *)slurp(argv[1], sizeof(float) * (size_t)w * h);
    field.stripheight = h;
    field.ymin = 0;
    field.ymax = h;

    /* the one call a maintainer adds to makeit(): photometry settings */
    sexgpu_compat_configure(prefs.mag_zeropoint, prefs.apert[0], prefs.autoparam[0], prefs.autoparam[1], 2, 0.0);

    if (!(ascfile = fopen(argv[7], "w"))) {
        fprintf(stderr, "cannot write %s\n", argv[7]);
        return 2;
    }
    init_device(w, h, field.strip); /* src/makeit.c:189 */
    makeback(&field);               /* src/makeit.c:195 */
    scanimage(&field, NULL, 0);     /* src/makeit.c:207 */
    fclose(ascfile);
    return 0;
}
