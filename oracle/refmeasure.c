/*
 * refmeasure.c -- drives the reference's own CPU measurement code, compiled
 * unmodified from the reference tree into oracle/_ref/libsexref.so:
 *
 *   src/clean.c        clean(), addcleanobj(), mergeobject()   (CLEAN)
 *   src/photom.c       computeaperflux(), computeautoflux(),
 *                      computeisocorflux()                     (photometry)
 *   src/neurro.c       neurinit(), getnnw(), neurresp()        (CLASS_STAR net)
 *   src/fits/fitsbody.c read_body()                            (FITS pixels)
 *
 * TEST INFRASTRUCTURE ONLY: tests/ use it to pin the oracle's CLEAN,
 * photometry, network and FITS conversion against the reference itself.
 * Each function sets up the reference structures (picstruct, objstruct,
 * prefstruct, tabstruct) the way the reference's own callers do and calls
 * the reference function; nothing of the reference's arithmetic is restated
 * here.
 */
#include "config.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "define.h"
#include "globals.h"
#include "prefs.h"
#include "clean.h"
#include "photom.h"
#include "neurro.h"
#include "fits/fitscat.h"

/* src/fits/fitscat.c:32 defines it and src/prefs.c:393 sets it from the
 * host byte order; fitscat.c itself is not compiled into this harness */
int bswapflag;

/* ------------------------------------------------------------------------ */
/* CLEAN.  Objects are given in the order an extraction completes them.  Each
 * one enters clean() against the list of the survivors so far
 * (src/clean.c:89-177); if it is not eaten it joins the list through
 * addcleanobj() (:189-228), as the upstream scan loop does.  Objects are never
 * expired from the list: the loop that wrote out objects the scan line had
 * passed lived in the deleted body of src/scan.c.
 *
 * in/out: the ref_clean_obj array (attributes of the objects; on return the
 * survivors carry their merged attributes); survive[i] = 1 if object i is
 * in the final list. */
typedef struct {
    double mx, my;
    float a, b, cxx, cyy, cxy, abcor, dthresh, mthresh;
    int fdnpix, dnpix;
    float fdflux, dflux, flux, fluxerr, fdpeak, dpeak, peak;
    int peakx, peaky, xmin, xmax, ymin, ymax, flags;
    int master;
} ref_clean_obj;

int ref_clean(ref_clean_obj *co, int n, double clean_param, int *survive)
{
    objliststruct objlist;
    objstruct *obj = (objstruct *)calloc(n + 1, sizeof(objstruct));
    picstruct field;
    int i, k;
    if (!obj)
        return -1;
    memset(&prefs, 0, sizeof(prefs));
    memset(&field, 0, sizeof(field));
    prefs.clean_flag = 1;
    prefs.clean_param = clean_param;
    prefs.clean_stacksize = n + 1;
    prefs.blank_flag = 0;
    for (i = 0; i < n; i++) {
        objstruct *o = obj + i;
        o->number = i;
        o->mx = co[i].mx;
        o->my = co[i].my;
        o->a = co[i].a;
        o->b = co[i].b;
        o->cxx = co[i].cxx;
        o->cyy = co[i].cyy;
        o->cxy = co[i].cxy;
        o->abcor = co[i].abcor;
        o->dthresh = co[i].dthresh;
        o->mthresh = co[i].mthresh;
        o->fdnpix = co[i].fdnpix;
        o->dnpix = co[i].dnpix;
        o->fdflux = co[i].fdflux;
        o->dflux = co[i].dflux;
        o->flux = co[i].flux;
        o->fluxerr = co[i].fluxerr;
        o->fdpeak = co[i].fdpeak;
        o->dpeak = co[i].dpeak;
        o->peak = co[i].peak;
        o->peakx = co[i].peakx;
        o->peaky = co[i].peaky;
        o->xmin = co[i].xmin;
        o->xmax = co[i].xmax;
        o->ymin = co[i].ymin;
        o->ymax = co[i].ymax;
        o->flag = co[i].flags;
    }
    objlist.obj = obj;
    objlist.nobj = n;
    objlist.plist = NULL;
    objlist.npix = 0;
    initclean();
    for (i = 0; i < n; i++)
        if (clean(&field, &field, i, &objlist))
            addcleanobj(obj + i);
    for (i = 0; i < n; i++)
        survive[i] = 0;
    for (k = 0; k < cleanobjlist->nobj; k++) {
        objstruct *o = cleanobjlist->obj + k;
        i = o->number;
        survive[i] = 1;
        co[i].fdnpix = o->fdnpix;
        co[i].dnpix = o->dnpix;
        co[i].fdflux = o->fdflux;
        co[i].dflux = o->dflux;
        co[i].flux = o->flux;
        co[i].fluxerr = o->fluxerr;
        co[i].fdpeak = o->fdpeak;
        co[i].dpeak = o->dpeak;
        co[i].peak = o->peak;
        co[i].peakx = o->peakx;
        co[i].peaky = o->peaky;
        co[i].xmin = o->xmin;
        co[i].xmax = o->xmax;
        co[i].ymin = o->ymin;
        co[i].ymax = o->ymax;
        co[i].flags = o->flag;
    }
    if (cleanobjlist->nobj)
        free(cleanobjlist->obj);
    cleanobjlist->nobj = 0;
    endclean();
    free(obj);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Photometry.  The frame (background-subtracted, CCD detection type, no
 * weight map) is held whole in memory (strip = frame, as the reference's
 * makeit.c:181-184 reads it).  For every object, computeaperflux() with the
 * first aperture, then computeautoflux(), with the object's position, shape
 * and local background. */
typedef struct {
    double mx, my;
    float a, b, cxx, cyy, cxy, dbkg;
    float flux_aper, fluxerr_aper, mag_aper, magerr_aper;
    float kron, flux_auto, fluxerr_auto, mag_auto, magerr_auto;
    int flags;
} ref_phot_obj;

int ref_photometry(float *sub, int w, int h, double aperture, double autoparam0, double autoparam1, int mask_type,
                   double gain, double mag_zeropoint, float backsig, ref_phot_obj *po, int n)
{
    picstruct field;
    objstruct obj;
    int i;
    memset(&field, 0, sizeof(field));
    memset(&prefs, 0, sizeof(prefs));
    memset(&outobj2, 0, sizeof(outobj2));
    memset(&flagobj2, 0, sizeof(flagobj2));
    prefs.detect_type = CCD;
    prefs.mask_type = mask_type == 2 ? MASK_CORRECT : mask_type == 1 ? MASK_BLANK : MASK_NONE;
    prefs.apert[0] = aperture;
    prefs.naper = 1;
    prefs.flux_apersize = prefs.fluxerr_apersize = prefs.mag_apersize = prefs.magerr_apersize = 1;
    prefs.autoparam[0] = autoparam0;
    prefs.autoparam[1] = autoparam1;
    prefs.autoaper[0] = prefs.autoaper[1] = 0.0;
    prefs.mag_zeropoint = mag_zeropoint;
    prefs.weightgain_flag = 0;
    /* the catalogue asks for MAG_AUTO and MAGERR_AUTO (src/photom.c:677-684) */
    *((char *)&flagobj2.mag_auto) = 1;
    *((char *)&flagobj2.magerr_auto) = 1;
    field.width = w;
    field.height = h;
    field.strip = sub;
    field.stripheight = h;
    field.ymin = 0;
    field.ymax = h;
    field.backsig = backsig;
    field.gain = gain;
    field.ngamma = 4.0 / log(10.0);
    for (i = 0; i < n; i++) {
        memset(&obj, 0, sizeof(obj));
        obj.mx = po[i].mx;
        obj.my = po[i].my;
        obj.a = po[i].a;
        obj.b = po[i].b;
        obj.cxx = po[i].cxx;
        obj.cyy = po[i].cyy;
        obj.cxy = po[i].cxy;
        obj.dbkg = po[i].dbkg;
        computeaperflux(&field, NULL, &obj, 0);
        computeautoflux(&field, NULL, NULL, NULL, &obj);
        po[i].flux_aper = outobj2.flux_aper[0];
        po[i].fluxerr_aper = outobj2.fluxerr_aper[0];
        po[i].mag_aper = outobj2.mag_aper[0];
        po[i].magerr_aper = outobj2.magerr_aper[0];
        po[i].kron = outobj2.kronfactor;
        po[i].flux_auto = outobj2.flux_auto;
        po[i].fluxerr_auto = outobj2.fluxerr_auto;
        po[i].mag_auto = outobj2.mag_auto;
        po[i].magerr_auto = outobj2.magerr_auto;
        po[i].flags = obj.flag;
    }
    return 0;
}

/* FLUX_ISOCOR / FLUXERR_ISOCOR through computeisocorflux() for objects
 * given by their isophotal flux, variance sum, fdnpix and detection
 * threshold. */
int ref_isocor(const float *flux, const float *fluxerr, const int *fdnpix, const float *dthresh, int n,
               float *flux_isocor, float *fluxerr_isocor)
{
    picstruct field;
    objstruct obj;
    int i;
    memset(&field, 0, sizeof(field));
    memset(&outobj2, 0, sizeof(outobj2));
    memset(&flagobj2, 0, sizeof(flagobj2));
    *((char *)&flagobj2.fluxerr_isocor) = 1;
    for (i = 0; i < n; i++) {
        memset(&obj, 0, sizeof(obj));
        obj.flux = flux[i];
        obj.fluxerr = fluxerr[i];
        obj.fdnpix = fdnpix[i];
        obj.dthresh = dthresh[i];
        computeisocorflux(&field, &obj);
        flux_isocor[i] = outobj2.flux_isocor;
        fluxerr_isocor[i] = outobj2.fluxerr_isocor;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* The star/galaxy network: the reference reads the .nnw file with getnnw()
 * (src/neurro.c:96) into its brainstruct and evaluates neurresp() (:57) on
 * each input vector (nin values per row); out receives the first output. */
int ref_neurresp(const char *nnw_path, const double *input, int nrows, double *out, int *nn_out)
{
    int i, l;
    double o[NEURONS];
    neurinit();
    strncpy(prefs.nnw_name, nnw_path, MAXCHAR - 1);
    getnnw();
    for (l = 0; l < 3; l++)
        nn_out[l] = l < brain->layersnb ? brain->nn[l] : 0;
    for (i = 0; i < nrows; i++) {
        double in[NEURONS];
        memcpy(in, input + (size_t)i * brain->nn[0], sizeof(double) * brain->nn[0]);
        neurresp(in, o);
        out[i] = o[0];
    }
    neurclose();
    return 0;
}

/* ------------------------------------------------------------------------ */
/* FITS data block to PIXTYPE through read_body() (src/fits/fitsbody.c:195):
 * the block (big-endian, as stored in the file) is read from path, with the
 * BITPIX, BSCALE, BZERO and BLANK of its header.  bitsgn is the header's
 * BITSGN keyword; without one the reference's header reader sets 1
 * (src/fits/fitshead.c:159), which makes BITPIX 8 pixels signed. */
int ref_read_body(const char *path, int bitpix, double bscale, double bzero, int blankflag, int blank, int bitsgn,
                  size_t n, float *out)
{
    catstruct cat;
    tabstruct tab;
    short ashort = 1;
    memset(&cat, 0, sizeof(cat));
    memset(&tab, 0, sizeof(tab));
    bswapflag = *((char *)&ashort);  /* as src/prefs.c:393 */
    strncpy(cat.filename, path, MAXCHARS - 1);
    if (!(cat.file = fopen(path, "rb")))
        return -1;
    tab.cat = &cat;
    tab.bitpix = bitpix;
    tab.bytepix = bitpix > 0 ? bitpix / 8 : -bitpix / 8;
    tab.bitsgn = bitsgn;
    tab.bscale = bscale;
    tab.bzero = bzero;
    tab.blankflag = blankflag;
    tab.blank = blank;
    tab.compress_type = COMPRESS_NONE;
    read_body(&tab, out, n);
    fclose(cat.file);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* The layout of the reference's catalogue record, outobjstruct
 * (src/types.h:417-455): sizeof, then the offset of every member in order. */
#include <stddef.h>
int ref_outobj_layout(int *out, int max)
{
    const int v[] = {(int)sizeof(outobjstruct), (int)offsetof(outobjstruct, number),
        (int)offsetof(outobjstruct, alpha2000), (int)offsetof(outobjstruct, delta2000),
        (int)offsetof(outobjstruct, sposx), (int)offsetof(outobjstruct, sposy),
        (int)offsetof(outobjstruct, flux_iso), (int)offsetof(outobjstruct, fluxerr_iso),
        (int)offsetof(outobjstruct, mag_iso), (int)offsetof(outobjstruct, magerr_iso),
        (int)offsetof(outobjstruct, flux_isocor), (int)offsetof(outobjstruct, fluxerr_isocor),
        (int)offsetof(outobjstruct, flux_aper), (int)offsetof(outobjstruct, fluxerr_aper),
        (int)offsetof(outobjstruct, mag_aper), (int)offsetof(outobjstruct, magerr_aper),
        (int)offsetof(outobjstruct, flux_auto), (int)offsetof(outobjstruct, fluxerr_auto),
        (int)offsetof(outobjstruct, mag_auto), (int)offsetof(outobjstruct, magerr_auto),
        (int)offsetof(outobjstruct, theta), (int)offsetof(outobjstruct, poserr_mx2),
        (int)offsetof(outobjstruct, poserr_my2), (int)offsetof(outobjstruct, poserr_mxy),
        (int)offsetof(outobjstruct, flag), (int)offsetof(outobjstruct, elong),
        (int)offsetof(outobjstruct, ellip), (int)offsetof(outobjstruct, sprob),
        (int)offsetof(outobjstruct, peak), (int)offsetof(outobjstruct, kronfactor),
        (int)offsetof(outobjstruct, bkg), (int)offsetof(outobjstruct, fwhm)};
    int i, n = (int)(sizeof(v) / sizeof(v[0]));
    for (i = 0; i < n && i < max; i++)
        out[i] = v[i];
    return n;
}
