/*
 * orc_fp64.c -- the FP64 oracle: the catalogue's floating-point columns of an
 * extraction recomputed in double precision (TEST INFRASTRUCTURE ONLY).
 *
 * The FP32 oracle (orc_extract.c) decides everything that is not a
 * floating-point measurement: the segmentation, the deblending tree and its
 * cut, the pixel sets of the objects (node pixels at their branch level,
 * final pixels after gatherup), CLEAN's victims and masters, the local
 * background, the isophotal areas and FLAGS.  Those decisions must equal the
 * reference's (they are held bit-exact against the GPU).  This file then
 * measures the same objects again with every accumulator in long double and
 * every derived quantity in double: preanalysis moments, ellipse and abcor
 * (src/cuda/cudaanalyse.cu:1686-1903), examineiso fluxes, errors and FWHM
 * (:2176-2581), ISOCOR (:62-98), APER (:104-287), AUTO/Kron (:293-592),
 * CLASS_STAR's network (src/neurro.c:57) and magnitudes (:638-656).  The
 * geometry of the apertures (which pixels and sub-pixels fall inside) follows
 * the double positions and shapes, so a pixel on an aperture boundary may
 * count differently from the FP32 catalogue; the error report shows that as
 * what it is, a difference from the FP64 result.
 *
 * The steps and their order are those of orc_extract.c (which cites the
 * reference's lines); only the types change.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "orc_internal.h"

typedef long double acc_t;

/* measurements of one object in double */
typedef struct {
    double fdflux, dflux, fdpeak, dpeak;
    double mx, my, mx2, my2, mxy, a, b, theta, abcor, cxx, cyy, cxy;
    int singuflag;
    double flux, fluxerr, peak, bkg, thresh, fwhm;
    double poserr_mx2, poserr_my2, poserr_mxy;
    double flux_isocor, fluxerr_isocor, flux_aper, fluxerr_aper, mag_aper, magerr_aper;
    double kron, flux_auto, fluxerr_auto, mag_auto, magerr_auto;
    double mag_iso, magerr_iso, fluxerr_iso, elong, ellip, polar, class_star;
} m64_t;

/* preanalyse (orc_extract.c) in double over one pixel list */
static void pre64(const frame_t *F, const obj_t *o, m64_t *t, const int *pix, int n, double dthresh, int robust)
{
    int w = F->w, k, xmin = 2 * 1048576, ymin = 2 * 1048576, xmax = 0, ymax = 0, area2 = 0, dnpix = 0;
    double peak = -ORC_BIG, cpeak = -ORC_BIG, dthresh2, xm, ym, xm2, ym2, xym, temp, temp2, theta, pmx2, pmy2;
    double darea, t1t2, rv;
    acc_t srv = 0, smx = 0, smy = 0, smx2 = 0, smy2 = 0, smxy = 0;
    for (k = 0; k < n; k++) {
        int p = pix[k], x = p % w, y = p / w;
        double val = F->sub[p], cval = F->cd[p];
        if (peak < val) peak = val;
        if (cpeak < cval) cpeak = cval;
        srv += cval;
        if (xmin > x) xmin = x;
        if (xmax < x) xmax = x;
        if (ymin > y) ymin = y;
        if (ymax < y) ymax = y;
    }
    rv = (double)srv;
    t->fdflux = rv;
    t->fdpeak = cpeak;
    t->dpeak = peak;
    dthresh2 = (dthresh + peak) / 2.0;
    for (k = 0; k < n; k++) {
        int p = pix[k];
        double x = p % w - xmin, y = p / w - ymin, cval = F->cd[p], val = F->sub[p];
        if (val > dthresh) dnpix++;
        if (val > dthresh2) area2++;
        smx += cval * x;
        smy += cval * y;
        smx2 += cval * x * x;
        smy2 += cval * y * y;
        smxy += cval * x * y;
    }
    xm = (double)(smx / srv);
    ym = (double)(smy / srv);
    if (robust && (o->flags & ORC_OBJ_MERGED)) {
        double xn = t->mx - xmin, yn = t->my - ymin;
        xm2 = (double)(smx2 / srv) + xn * xn - 2 * xm * xn;
        ym2 = (double)(smy2 / srv) + yn * yn - 2 * ym * yn;
        xym = (double)(smxy / srv) + xn * yn - xm * yn - xn * ym;
        xm = xn;
        ym = yn;
    } else {
        xm2 = (double)(smx2 / srv) - xm * xm;
        ym2 = (double)(smy2 / srv) - ym * ym;
        xym = (double)(smxy / srv) - xm * ym;
    }
    t->singuflag = 0;
    if ((temp2 = xm2 * ym2 - xym * xym) < 0.00694) {
        xm2 += 0.0833333;
        ym2 += 0.0833333;
        temp2 = xm2 * ym2 - xym * xym;
        t->singuflag = 1;
    }
    if (fabs(temp = xm2 - ym2) > 0.0)
        theta = atan2(2.0 * xym, temp) / 2.0;
    else
        theta = ORC_PI / 4.0;
    temp = sqrt(0.25 * temp * temp + xym * xym);
    pmy2 = pmx2 = 0.5 * (xm2 + ym2);
    pmx2 += temp;
    pmy2 -= temp;
    t->dflux = 0;
    {
        acc_t stv = 0;
        for (k = 0; k < n; k++)
            stv += F->sub[pix[k]];
        t->dflux = (double)stv;
    }
    t->mx = xm + xmin;
    t->my = ym + ymin;
    t->mx2 = xm2;
    t->my2 = ym2;
    t->mxy = xym;
    t->a = sqrt(pmx2);
    t->b = sqrt(pmy2);
    t->theta = theta * 180.0 / ORC_PI;
    t->cxx = ym2 / temp2;
    t->cyy = xm2 / temp2;
    t->cxy = -2 * xym / temp2;
    darea = (double)area2 - dnpix;
    t1t2 = dthresh / dthresh2;
    if (t1t2 > 0.0) {
        t->abcor = (darea < 0.0 ? darea : -1.0) / (2 * ORC_PI * log(t1t2 < 1.0 ? t1t2 : 0.99) * t->a * t->b);
        if (t->abcor > 1.0)
            t->abcor = 1.0;
    } else
        t->abcor = 1.0;
}

/* examineiso (orc_extract.c) in double; areas, peaks' positions and the
 * local background come from the FP32 object */
static void exam64(const frame_t *F, const obj_t *o, m64_t *t)
{
    const orc_config *cfg = F->cfg;
    int k, w = F->w;
    double backnoise2 = (double)F->backsig * F->backsig, peak = -ORC_BIG, dbkg = o->dbkg;
    acc_t esum = 0, emx2 = 0, emy2 = 0, emxy = 0, stv = 0, svar = 0;
    t->bkg = orc_back_at(F->back, F->nbx, F->nby, F->bw, F->bh, (int)(t->mx + 0.5), (int)(t->my + 0.5));
    if (cfg->back_photo_type == 1 && o->bkg != orc_back_at(F->back, F->nbx, F->nby, F->bw, F->bh,
                                                           (int)(o->mx + 0.5), (int)(o->my + 0.5)))
        t->bkg += dbkg;
    for (k = 0; k < o->n; k++) {
        int p = o->pix[k];
        double pix = F->sub[p], cdpix = F->cd[p], err, x, y;
        if (pix > peak) peak = pix;
        stv += pix;
        if (F->var) svar += F->var[p];
        err = F->var ? (double)F->var[p] : backnoise2;
        if (cfg->gain > 0.0 && cdpix > 0.0)
            err += cdpix / cfg->gain;
        x = p % w - t->mx;
        y = p / w - t->my;
        esum += err;
        emx2 += err * x * x;
        emy2 += err * y * y;
        emxy += err * x * y;
    }
    {
        double flux2 = t->fdflux * t->fdflux, ex = (double)(emx2 / flux2), ey = (double)(emy2 / flux2),
               exy = (double)(emxy / flux2), es = (double)(esum * 0.08333 / flux2);
        if (t->singuflag && (ex * ey - exy * exy) < es * es) {
            ex += es;
            ey += es;
        }
        t->poserr_mx2 = ex;
        t->poserr_my2 = ey;
        t->poserr_mxy = exy;
    }
    {
        double sigtv = F->var ? (double)svar : (double)o->n * backnoise2, tvd = (double)stv;
        if (cfg->back_photo_type == 1)
            tvd -= o->n * dbkg;
        if (cfg->gain > 0.0 && tvd > 0.0)
            sigtv += tvd / cfg->gain;
        t->flux = tvd;
        t->fluxerr = sigtv;
    }
    t->thresh = (double)o->athr - dbkg;
    t->peak = peak - dbkg;
    /* FWHM */
    {
        double thresh0 = t->peak / 5.0;
        if (thresh0 < t->thresh)
            thresh0 = t->thresh;
        t->fwhm = 0.0;
        if (thresh0 > 0.0) {
            acc_t s = 0, sx = 0, sy = 0, sxx = 0, sxy = 0;
            double sat = cfg->satur_level - dbkg, d, b, bmax;
            for (k = 0; k < o->n; k++) {
                int p = o->pix[k];
                double pv = F->sub[p] - dbkg;
                if (pv > thresh0 && pv < sat) {
                    double dx = p % w - t->mx, dy = p / w - t->my, lpix = log(pv), inverr2 = pv * pv;
                    double d2 = dx * dx + dy * dy;
                    s += inverr2;
                    sx += d2 * inverr2;
                    sxx += d2 * d2 * inverr2;
                    sy += lpix * inverr2;
                    sxy += lpix * d2 * inverr2;
                }
            }
            d = (double)(s * sxx - sx * sx);
            if (fabs(d) > 0.0) {
                b = -(double)(s * sxy - sx * sy) / d;
                if (b < (bmax = 1 / (13 * t->a * t->b)))
                    b = bmax;
                t->fwhm = 1.6651 / sqrt(b);
                if (t->fwhm > 0.0)
                    t->fwhm -= 1 / (4 * t->fwhm);
            }
        }
    }
}

/* aperflux (orc_extract.c) in double */
static void aper64(const frame_t *F, const int *alloc, const obj_t *o, m64_t *t, int self)
{
    const orc_config *cfg = F->cfg;
    double raper = cfg->phot_aperture / 2.0, raper2 = raper * raper, rintlim = raper - 0.75, rintlim2, rextlim2;
    double scale = 1.0 / ORC_APER_OVERSAMP, scale2 = scale * scale, off = 0.5 * (scale - 1.0), area = 0.0;
    double var = (double)F->backsig * F->backsig;
    acc_t tv = 0, sigtv = 0;
    int x, y, xmin, xmax, ymin, ymax, w = F->w, h = F->h;
    rintlim2 = rintlim > 0.0 ? rintlim * rintlim : 0.0;
    rextlim2 = (raper + 0.75) * (raper + 0.75);
    xmin = (int)(t->mx - raper + 0.499999);
    xmax = (int)(t->mx + raper + 1.499999);
    ymin = (int)(t->my - raper + 0.499999);
    ymax = (int)(t->my + raper + 1.499999);
    if (xmin < 0) xmin = 0;
    if (xmax > w) xmax = w;
    if (ymin < 0) ymin = 0;
    if (ymax > h) ymax = h;
    for (y = ymin; y < ymax; y++)
        for (x = xmin; x < xmax; x++) {
            double dx = x - t->mx, dy = y - t->my, r2 = dx * dx + dy * dy, locarea, pix, pvar;
            int tt, x2, y2, sx, sy;
            if (r2 >= rextlim2)
                continue;
            if (r2 > rintlim2) {
                locarea = 0.0;
                for (sy = 0; sy < ORC_APER_OVERSAMP; sy++) {
                    double ddy = dy + off + sy * scale;
                    for (sx = 0; sx < ORC_APER_OVERSAMP; sx++) {
                        double ddx = dx + off + sx * scale;
                        if (ddx * ddx + ddy * ddy < raper2)
                            locarea += scale2;
                    }
                }
            } else
                locarea = 1.0;
            area += locarea;
            pix = F->sub[(size_t)y * w + x];
            tt = alloc[(size_t)y * w + x];
            pvar = F->var ? (double)F->var[(size_t)y * w + x] : var;
            if ((tt >= 0 && tt != self) || pix <= -ORC_BIG) {
                if (cfg->mask_type == 2 && (x2 = (int)(2 * t->mx + 0.49999 - x)) >= 0 && x2 < w
                    && (y2 = (int)(2 * t->my + 0.49999 - y)) >= 0 && y2 < h
                    && ((tt = alloc[(size_t)y2 * w + x2]) == self || tt == -1)
                    && F->sub[(size_t)y2 * w + x2] > -ORC_BIG) {
                    pix = F->sub[(size_t)y2 * w + x2];
                    if (F->var)
                        pvar = F->var[(size_t)y2 * w + x2];
                } else {
                    pix = 0.0;
                    if (F->var)
                        pvar = 0.0;
                }
            }
            sigtv += pvar * locarea;
            tv += locarea * pix;
        }
    {
        double tvd = (double)tv - area * o->dbkg, sig = (double)sigtv;
        if (cfg->gain > 0.0 && tvd > 0.0)
            sig += tvd / cfg->gain;
        t->flux_aper = tvd;
        t->fluxerr_aper = sqrt(sig);
        t->mag_aper = tvd > 0.0 ? -2.5 * log10(tvd) + cfg->mag_zeropoint : 99.0;
        t->magerr_aper = tvd > 0.0 ? 1.086 * sqrt(sig) / tvd : 99.0;
    }
}

/* autoflux (orc_extract.c) in double */
static void auto64(const frame_t *F, const int *alloc, const obj_t *o, m64_t *t, int self)
{
    const orc_config *cfg = F->cfg;
    double cx2, cy2, cxy, dxlim, dylim, klim2, var = (double)F->backsig * F->backsig, tvd, sig;
    acc_t r1 = 0, v1 = 0, tv = 0, svar = 0;
    int x, y, xmin, xmax, ymin, ymax, area = 0, areab = 0, w = F->w, h = F->h;
    cx2 = t->cxx;
    cy2 = t->cyy;
    cxy = t->cxy;
    dxlim = cx2 - cxy * cxy / (4.0 * cy2);
    dxlim = dxlim > 0.0 ? ORC_KRON_NSIG / sqrt(dxlim) : 0.0;
    dylim = cy2 - cxy * cxy / (4.0 * cx2);
    dylim = dylim > 0.0 ? ORC_KRON_NSIG / sqrt(dylim) : 0.0;
    klim2 = ORC_KRON_NSIG * ORC_KRON_NSIG;
    if (!(ORC_KRON_NSIG * sqrt(t->a * t->b) > 0.0)) {
        cx2 = cy2 = 1.0;
        cxy = 0.0;
        dxlim = dylim = 0.0;
        klim2 = 0.0;
    }
    xmin = (int)floor(t->mx - dxlim + 0.5);
    xmax = (int)floor(t->mx + dxlim + 0.5) + 1;
    ymin = (int)floor(t->my - dylim + 0.5);
    ymax = (int)floor(t->my + dylim + 0.5) + 1;
    if (xmin < 0) xmin = 0;
    if (xmax > w) xmax = w;
    if (ymin < 0) ymin = 0;
    if (ymax > h) ymax = h;
    for (y = ymin; y < ymax; y++)
        for (x = xmin; x < xmax; x++) {
            double dx = x - t->mx, dy = y - t->my, r2 = cx2 * dx * dx + cy2 * dy * dy + cxy * dx * dy, pix;
            int tt;
            if (r2 > klim2)
                continue;
            pix = F->sub[(size_t)y * w + x];
            tt = alloc[(size_t)y * w + x];
            if ((tt == self || tt == -1) && pix > -ORC_BIG) {
                area++;
                r1 += sqrt(r2) * pix;
                v1 += pix;
            } else
                areab++;
        }
    area += areab;
    if (!area) {
        t->kron = t->flux_auto = t->fluxerr_auto = 0.0;
        t->mag_auto = t->magerr_auto = 99.0;
        return;
    }
    if (r1 > 0 && v1 > 0) {
        t->kron = cfg->phot_autoparams[0] * (double)(r1 / v1);
        if (t->kron < cfg->phot_autoparams[1])
            t->kron = cfg->phot_autoparams[1];
    } else
        t->kron = cfg->phot_autoparams[1];
    if (t->kron * sqrt(t->a * t->b) > 0.0) {
        cx2 = t->cxx;
        cy2 = t->cyy;
        cxy = t->cxy;
        dxlim = cx2 - cxy * cxy / (4.0 * cy2);
        dxlim = dxlim > 0.0 ? t->kron / sqrt(dxlim) : 0.0;
        dylim = cy2 - cxy * cxy / (4.0 * cx2);
        dylim = dylim > 0.0 ? t->kron / sqrt(dylim) : 0.0;
        klim2 = t->kron * t->kron;
    } else {
        cx2 = cy2 = 1.0;
        cxy = 0.0;
        dxlim = dylim = klim2 = 0.0;
        t->kron = 0.0;
    }
    xmin = (int)floor(t->mx - dxlim + 0.5);
    xmax = (int)floor(t->mx + dxlim + 0.5) + 1;
    ymin = (int)floor(t->my - dylim + 0.5);
    ymax = (int)floor(t->my + dylim + 0.5) + 1;
    if (xmin < 0) xmin = 0;
    if (xmax > w) xmax = w;
    if (ymin < 0) ymin = 0;
    if (ymax > h) ymax = h;
    area = 0;
    for (y = ymin; y < ymax; y++)
        for (x = xmin; x < xmax; x++) {
            double dx = x - t->mx, dy = y - t->my, pix, pvar;
            int tt, x2, y2;
            if (cx2 * dx * dx + cy2 * dy * dy + cxy * dx * dy > klim2)
                continue;
            area++;
            pix = F->sub[(size_t)y * w + x];
            tt = alloc[(size_t)y * w + x];
            pvar = F->var ? F->var[(size_t)y * w + x] : 0.0;
            if ((tt >= 0 && tt != self) || pix <= -ORC_BIG) {
                if (cfg->mask_type == 2 && (x2 = (int)(2 * t->mx + 0.49999 - x)) >= 0 && x2 < w
                    && (y2 = (int)(2 * t->my + 0.49999 - y)) >= 0 && y2 < h
                    && ((tt = alloc[(size_t)y2 * w + x2]) == -1 || tt == self)
                    && F->sub[(size_t)y2 * w + x2] > -ORC_BIG) {
                    pix = F->sub[(size_t)y2 * w + x2];
                    if (F->var)
                        pvar = F->var[(size_t)y2 * w + x2];
                } else {
                    pix = 0.0;
                    pvar = 0.0;
                }
            }
            tv += pix;
            svar += pvar;
        }
    tvd = (double)tv - area * (double)o->dbkg;
    sig = F->var ? (double)svar : (double)area * var;
    if (cfg->gain > 0.0 && tvd > 0.0)
        sig += tvd / cfg->gain;
    t->flux_auto = tvd;
    t->fluxerr_auto = sqrt(sig);
    t->mag_auto = tvd > 0.0 ? -2.5 * log10(tvd) + cfg->mag_zeropoint : 99.0;
    t->magerr_auto = tvd > 0.0 ? 1.086 * t->fluxerr_auto / tvd : 99.0;
    if (tvd <= 0.0)
        t->kron = 0.0;
}

/* the network response (nnw_response of orc_extract.c) */
static double nnw64(const orc_nnw *net, double *in)
{
    double nx[ORC_NNW_NEURONS];
    int i, k, l, last = net->nlayers - 1;
    for (i = 0; i < net->nn[0]; i++)
        in[i] = in[i] * net->inscale[i] + net->inbias[i];
    for (l = 0; l < last; l++) {
        for (k = 0; k < net->nn[l + 1]; k++) {
            double sum = net->b[l][k];
            for (i = 0; i < net->nn[l]; i++)
                sum += net->w[l][i][k] * in[i];
            nx[k] = 1.0 / (1.0 + exp(-sum));
        }
        for (k = 0; k < net->nn[l + 1]; k++)
            in[k] = nx[k];
    }
    return (in[0] - net->outbias[0]) / net->outscale[0];
}

static void end64(const frame_t *F, const int *alloc, const obj_t *o, m64_t *t, int self)
{
    const orc_config *cfg = F->cfg;
    double ati;
    t->elong = t->a / t->b;
    t->ellip = 1 - t->b / t->a;
    t->polar = (t->a * t->a - t->b * t->b) / (t->a * t->a + t->b * t->b);
    t->fluxerr_iso = sqrt(t->fluxerr);
    ati = (t->flux > 0.0) ? (o->fdnpix * (double)o->dthr / t->flux) : 0.0;
    if (ati > 1.0)
        ati = 1.0;
    else if (ati < 0.0)
        ati = 0.0;
    t->flux_isocor = t->flux / (1.0 - 0.196099 * ati - 0.751208 * ati * ati);
    if (t->flux > 0.0) {
        double sigtv = t->fluxerr / (t->flux * t->flux);
        double dati = o->fdnpix ? ati * sqrt(sigtv + 1.0 / o->fdnpix) : 0.0;
        dati = 0.196099 * dati + 0.751208 * 2 * ati * dati;
        t->fluxerr_isocor = sqrt(sigtv + dati * dati) * t->flux;
    } else
        t->fluxerr_isocor = sqrt(t->fluxerr);
    aper64(F, alloc, o, t, self);
    auto64(F, alloc, o, t, self);
    t->mag_iso = t->flux > 0.0 ? -2.5 * log10(t->flux) + cfg->mag_zeropoint : 99.0;
    t->magerr_iso = t->flux > 0.0 ? 1.086 * t->fluxerr_iso / t->flux : 99.0;
    t->class_star = 0.0;
    if (cfg->nnw) {
        double in[ORC_NNW_NEURONS], fwhm = cfg->seeing_fwhm, fac2;
        double pixscale = cfg->pixel_scale > 0.0 ? cfg->pixel_scale : 1.0;
        int i, j = 0;
        fac2 = fwhm / pixscale;
        fac2 *= fac2;
        in[j] = log10(o->iso[0] ? o->iso[0] / fac2 : 0.01);
        in[++j] = o->athr > 0.0 ? log10(t->peak > 0.0 ? t->peak / o->athr : 0.1) : -1.0;
        for (i = 1; i < ORC_NISO; i++)
            in[++j] = log10(o->iso[i] ? o->iso[i] / fac2 : 0.01);
        in[++j] = log10(fwhm);
        t->class_star = nnw64(cfg->nnw, in);
    }
}

/* The twin of every object, then of the catalogue rows: objs[] as
 * orc_extract leaves them after CLEAN (final_master set), alloc the
 * allocation map of the photometry, rows[k] the object index of catalogue
 * row k. */
void orc_measure64(const frame_t *F, const int *alloc, const obj_t *objs, int nobj, const int *rows, int nrows,
                   orc_object64 *out)
{
    m64_t *t = (m64_t *)calloc(nobj + 1, sizeof(m64_t));
    int i, k;
    for (i = 0; i < nobj; i++) {
        const obj_t *o = &objs[i];
        pre64(F, o, &t[i], o->nodepix, o->nnode, o->node_dthresh, 0);
        if (o->level > 0)
            pre64(F, o, &t[i], o->pix, o->n, o->dthr, 1);
        exam64(F, o, &t[i]);
    }
    /* CLEAN merges (mergeobject, src/clean.c:234-287) with the FP32 masters */
    for (i = 0; i < nobj; i++) {
        int m = objs[i].final_master;
        if (m < 0)
            continue;
        t[m].fdflux += t[i].fdflux;
        t[m].dflux += t[i].dflux;
        t[m].flux += t[i].flux;
        t[m].fluxerr += t[i].fluxerr;
        if (t[i].fdpeak > t[m].fdpeak) t[m].fdpeak = t[i].fdpeak;
        if (t[i].dpeak > t[m].dpeak) t[m].dpeak = t[i].dpeak;
        if (t[i].peak > t[m].peak) t[m].peak = t[i].peak;
    }
    for (k = 0; k < nrows; k++) {
        const int i2 = rows[k];
        const obj_t *o = &objs[i2];
        m64_t *q = &t[i2];
        orc_object64 *r = &out[k];
        end64(F, alloc, o, q, i2);
        memset(r, 0, sizeof(*r));
        r->number = k + 1;
        r->fdflux = q->fdflux; r->dflux = q->dflux; r->flux = q->flux; r->fluxerr = q->fluxerr;
        r->fdpeak = q->fdpeak; r->dpeak = q->dpeak; r->peak = q->peak;
        r->mx = q->mx; r->my = q->my; r->mx2 = q->mx2; r->my2 = q->my2; r->mxy = q->mxy;
        r->a = q->a; r->b = q->b; r->theta = q->theta; r->abcor = q->abcor;
        r->cxx = q->cxx; r->cyy = q->cyy; r->cxy = q->cxy; r->class_star = q->class_star;
        r->poserr_mx2 = q->poserr_mx2; r->poserr_my2 = q->poserr_my2; r->poserr_mxy = q->poserr_mxy;
        r->bkg = q->bkg; r->thresh = q->thresh; r->fwhm = q->fwhm;
        r->flux_iso = q->flux; r->fluxerr_iso = q->fluxerr_iso; r->mag_iso = q->mag_iso; r->magerr_iso = q->magerr_iso;
        r->flux_isocor = q->flux_isocor; r->fluxerr_isocor = q->fluxerr_isocor;
        r->flux_aper = q->flux_aper; r->fluxerr_aper = q->fluxerr_aper; r->mag_aper = q->mag_aper;
        r->magerr_aper = q->magerr_aper;
        r->kronfactor = q->kron; r->flux_auto = q->flux_auto; r->fluxerr_auto = q->fluxerr_auto;
        r->mag_auto = q->mag_auto; r->magerr_auto = q->magerr_auto;
        r->elong = q->elong; r->ellip = q->ellip; r->polar = q->polar;
    }
    free(t);
}
