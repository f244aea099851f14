/*
 * orc_extract.c -- oracle: filter, detection, deblending, analysis, CLEAN,
 * photometry/FLAGS and catalog order.  TEST INFRASTRUCTURE ONLY (oracle.h).
 *
 * Straight-line single-threaded C.  Each step names the reference file:line
 * whose arithmetic it restates.  Where the reference is order-dependent
 * (floating sums in an unspecified scan order) or buggy, the rule used here is
 * stated at that step; the CUDA path follows the same rules.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "orc_internal.h"
#include "orc_xsum.h"

/* ------------------------------------------------------------------------ */
/* Detection filter: src/filter.c:39-95.  For every output pixel the mask is
 * walked row-major and each in-frame term is added to a float accumulator
 * started at 0; out-of-frame terms are skipped (the frame is zero-padded).  */
void orc_filter(const float *sub, int w, int h, const float *mask, int mw, int mh, float *cd)
{
    int x, y, i, j, mw2 = mw / 2, mh2 = mh / 2;
    for (y = 0; y < h; y++)
        for (x = 0; x < w; x++) {
            float acc = 0.0f;
            for (j = 0; j < mh; j++) {
                int yy = y + j - mh2;
                if (yy < 0 || yy >= h)
                    continue;
                for (i = 0; i < mw; i++) {
                    int xx = x + i - mw2;
                    if (xx < 0 || xx >= w)
                        continue;
                    acc += mask[j * mw + i] * sub[(size_t)yy * w + xx];
                }
            }
            cd[(size_t)y * w + x] = acc;
        }
}

/* ------------------------------------------------------------------------ */
/* union-find with the root of every set equal to its smallest element
 * (src/cuda/cudadetection.cu:235-276 converge to the minimum linear index). */
static int uf_find(int *p, int a)
{
    int r = a, t;
    while (p[r] != r)
        r = p[r];
    while (p[a] != r) {
        t = p[a];
        p[a] = r;
        a = t;
    }
    return r;
}

static void uf_union(int *p, int a, int b)
{
    a = uf_find(p, a);
    b = uf_find(p, b);
    if (a < b)
        p[b] = a;
    else if (b < a)
        p[a] = b;
}

/* ------------------------------------------------------------------------ */
typedef struct {
    int n;          /* pixels */
    int *pix;       /* linear pixel indices, raster order */
    int xmin, xmax, ymin, ymax;
    float fdpeak;
    xsum_t fdflux;
    int firstpix;   /* smallest index */
    int lastrow_x;  /* x of the first pixel on row ymax */
    float dthresh, thresh;  /* smallest detection / analysis threshold of its pixels */
} root_t;

typedef struct {
    int level, label;      /* label = smallest pixel index of the branch at its level */
    int npix;
    float fdflux;
    float dthresh;
    int parent;            /* node index at level-1 */
} node_t;

/* ------------------------------------------------------------------------ */
/* Branch CCL inside one root at threshold t: labels lab[k] (index into the
 * root's raster-ordered pixel list) get the smallest member position; -1 for
 * pixels below t.  bmap maps bbox positions to list positions (-1 outside). */
static void level_ccl(const frame_t *F, const root_t *R, const int *bmap, int bw,
                      float t, int *par, int *lab)
{
    int k, q, x, y, bx, by;
    static const int dx[4] = {-1, -1, 0, 1}, dy[4] = {0, -1, -1, -1};
    for (k = 0; k < R->n; k++)
        par[k] = (F->cd[R->pix[k]] >= t) ? k : -1;
    for (k = 0; k < R->n; k++) {
        if (par[k] < 0)
            continue;
        x = R->pix[k] % F->w;
        y = R->pix[k] / F->w;
        bx = x - R->xmin;
        by = y - R->ymin;
        for (q = 0; q < 4; q++) {
            int nx = bx + dx[q], ny = by + dy[q], m;
            if (nx < 0 || ny < 0 || nx >= bw || ny > R->ymax - R->ymin)
                continue;
            m = bmap[ny * bw + nx];
            if (m >= 0 && par[m] >= 0)
                uf_union(par, k, m);
        }
    }
    for (k = 0; k < R->n; k++)
        lab[k] = par[k] >= 0 ? uf_find(par, k) : -1;
}

/* cudaanalyse.cu:1686-1903 (preanalyse_full_kernel) and :1906-2124
 * (preanalyse_robust_kernel), restated on one pixel list.  robust != 0 uses
 * the previous barycentre (OBJ_MERGED branch of :2059-2070).  The five moment
 * sums and rv/tv are exact order-free sums of the float terms the reference
 * accumulates; singuflag keeps the value set by the singularity fix. */
static void preanalyse(const frame_t *F, obj_t *o, const int *pix, int n, double dthresh, int robust)
{
    float peak, cpeak, val, cval;
    double dthresh2, t1t2, darea, xm, ym, xm2, ym2, xym, temp, temp2, theta, pmx2, pmy2, mx, my, mx2, my2, mxy, rvd;
    int k, x, y, xmin, xmax, ymin, ymax, area2, dnpix;
    float rv;
    xsum_t srv, stv, smx, smy, smx2, smy2, smxy;
    int w = F->w, h = F->h, flag = o->flags;

    xs_init(&srv);
    peak = cpeak = -ORC_BIG;
    ymin = xmin = 2 * 1048576;
    ymax = xmax = 0;
    for (k = 0; k < n; k++) {
        int p = pix[k];
        x = p % w;
        y = p / w;
        if (peak < (val = F->sub[p]))
            peak = val;
        if (cpeak < (cval = F->cd[p]))
            cpeak = cval;
        xs_add(&srv, cval);
        if (xmin > x) xmin = x;
        if (xmax < x) xmax = x;
        if (ymin > y) ymin = y;
        if (ymax < y) ymax = y;
    }
    rv = xs_float(&srv);
    if (!robust && o->level > 0)
        flag |= ORC_OBJ_MERGED;
    if (xmin == 0 || xmax == w - 1 || ymin == 0 || ymax == h - 1)
        flag |= ORC_OBJ_TRUNC;
    o->fdflux = rv;
    o->fdpeak = cpeak;
    o->dpeak = peak;
    o->xmin = xmin;
    o->xmax = xmax;
    o->ymin = ymin;
    o->ymax = ymax;

    xs_init(&stv); xs_init(&smx); xs_init(&smy); xs_init(&smx2); xs_init(&smy2); xs_init(&smxy);
    dthresh2 = (dthresh + peak) / 2.0;
    area2 = dnpix = 0;
    for (k = 0; k < n; k++) {
        int p = pix[k];
        x = p % w - xmin;
        y = p / w - ymin;
        cval = F->cd[p];
        xs_add(&stv, val = F->sub[p]);
        if (val > dthresh)
            dnpix++;
        if (val > dthresh2)
            area2++;
        xs_add(&smx, cval * x);
        xs_add(&smy, cval * y);
        xs_add(&smx2, cval * x * x);
        xs_add(&smy2, cval * y * y);
        xs_add(&smxy, cval * x * y);
    }
    mx = xs_double(&smx);
    my = xs_double(&smy);
    mx2 = xs_double(&smx2);
    my2 = xs_double(&smy2);
    mxy = xs_double(&smxy);
    rvd = rv;
    xm = mx / rvd;
    ym = my / rvd;
    if (robust && (flag & ORC_OBJ_MERGED)) {
        double xn = o->mx - xmin, yn = o->my - ymin;
        xm2 = mx2 / rvd + xn * xn - 2 * xm * xn;
        ym2 = my2 / rvd + yn * yn - 2 * ym * yn;
        xym = mxy / rvd + xn * yn - xm * yn - xn * ym;
        xm = xn;
        ym = yn;
    } else {
        xm2 = mx2 / rvd - xm * xm;
        ym2 = my2 / rvd - ym * ym;
        xym = mxy / rvd - xm * ym;
    }
    o->singuflag = 0;
    if ((temp2 = xm2 * ym2 - xym * xym) < 0.00694) {
        xm2 += 0.0833333;
        ym2 += 0.0833333;
        temp2 = xm2 * ym2 - xym * xym;
        o->singuflag = 1;
    }
    if ((fabs(temp = xm2 - ym2)) > 0.0)
        theta = atan2(2.0 * xym, temp) / 2.0;
    else
        theta = ORC_PI / 4.0;
    temp = sqrt(0.25 * temp * temp + xym * xym);
    pmy2 = pmx2 = 0.5 * (xm2 + ym2);
    pmx2 += temp;
    pmy2 -= temp;
    o->dnpix = dnpix;
    o->dflux = xs_float(&stv);
    o->mx = xm + xmin;
    o->my = ym + ymin;
    o->mx2 = xm2;
    o->my2 = ym2;
    o->mxy = xym;
    o->a = (float)sqrt(pmx2);
    o->b = (float)sqrt(pmy2);
    o->theta = theta * 180.0 / ORC_PI;
    o->cxx = (float)(ym2 / temp2);
    o->cyy = (float)(xm2 / temp2);
    o->cxy = (float)(-2 * xym / temp2);
    darea = (double)area2 - dnpix;
    t1t2 = dthresh / dthresh2;
    if (t1t2 > 0.0) {
        o->abcor = (darea < 0.0 ? darea : -1.0) / (2 * ORC_PI * log(t1t2 < 1.0 ? t1t2 : 0.99) * o->a * o->b);
        if (o->abcor > 1.0)
            o->abcor = 1.0;
    } else
        o->abcor = 1.0;
    o->flags = flag;
}

/* ------------------------------------------------------------------------ */
/* Deblend one root: src/cuda/cudadeblend.cu:199-217 (thresholds), :579-727
 * (per-level branches), :1425-1776 (pruning), :1262-1360 (gatherup).
 * Appends the kept branches of this root to objs (in level, label order). */
static int deblend_root(const frame_t *F, int r, root_t *R, obj_t **objs, int *nobj, int *cap)
{
    const orc_config *cfg = F->cfg;
    int N = cfg->deblend_nthresh, L, k, i, j;
    int bw = R->xmax - R->xmin + 1, bh = R->ymax - R->ymin + 1;
    int *bmap, *par, *lab, *prevlab, *owner;
    float *thr;
    node_t *nodes = NULL;
    int nnodes = 0, capn = 0;
    int *lvstart = (int *)malloc(sizeof(int) * (N + 1));
    int *ok, *flagv, *nson;
    double value0;
    float fdflux0 = xs_float(&R->fdflux);
    int nkept = 0, first_obj = *nobj;

    bmap = (int *)malloc(sizeof(int) * (size_t)bw * bh);
    for (k = 0; k < bw * bh; k++)
        bmap[k] = -1;
    for (k = 0; k < R->n; k++) {
        int p = R->pix[k];
        bmap[(p / F->w - R->ymin) * bw + (p % F->w - R->xmin)] = k;
    }
    par = (int *)malloc(sizeof(int) * R->n);
    lab = (int *)malloc(sizeof(int) * R->n);
    prevlab = (int *)malloc(sizeof(int) * R->n);
    owner = (int *)malloc(sizeof(int) * R->n);

    /* multi-thresholds, cudadeblend.cu:199-217 */
    thr = (float *)malloc(sizeof(float) * (N + 1));
    thr[0] = R->dthresh;
    for (i = 1; i < N; i++) {
        double d0 = R->dthresh, dp = R->fdpeak;
        thr[i] = d0 * pow(dp / d0, (double)i / N);
    }

    /* level 0: the root itself */
    capn = 16;
    nodes = (node_t *)malloc(sizeof(node_t) * capn);
    nodes[0].level = 0;
    nodes[0].label = 0;
    nodes[0].npix = R->n;
    nodes[0].fdflux = fdflux0;
    nodes[0].dthresh = R->dthresh;
    nodes[0].parent = -1;
    nnodes = 1;
    lvstart[0] = 0;
    for (k = 0; k < R->n; k++)
        prevlab[k] = 0; /* list position 0 is the smallest index */
    /* per-level branches, src/cuda/cudadeblend.cu:609-727 with the minimum
     * area prefs.deb_maxarea (src/scan.c:90, src/prefs.c:463) */
    for (L = 1; L < N; L++) {
        int *cnt, *nodeof;
        xsum_t *fs;
        lvstart[L] = nnodes;
        level_ccl(F, R, bmap, bw, thr[L], par, lab);
        cnt = (int *)calloc(R->n, sizeof(int));
        nodeof = (int *)malloc(sizeof(int) * R->n);
        fs = (xsum_t *)malloc(sizeof(xsum_t) * R->n);
        for (k = 0; k < R->n; k++)
            xs_init(&fs[k]);
        for (k = 0; k < R->n; k++)
            if (lab[k] >= 0) {
                cnt[lab[k]]++;
                xs_add(&fs[lab[k]], F->cd[R->pix[k]]);
            }
        for (k = 0; k < R->n; k++) {
            nodeof[k] = -1;
            if (lab[k] == k && cnt[k] >= F->debminarea) {
                if (nnodes == capn) {
                    capn *= 2;
                    nodes = (node_t *)realloc(nodes, sizeof(node_t) * capn);
                }
                nodes[nnodes].level = L;
                nodes[nnodes].label = k;
                nodes[nnodes].npix = cnt[k];
                nodes[nnodes].fdflux = xs_float(&fs[k]);
                nodes[nnodes].dthresh = thr[L];
                nodes[nnodes].parent = prevlab[k];
                nodeof[k] = nnodes;
                nnodes++;
            }
        }
        /* labels of this level become node ids for the next level's parents */
        for (k = 0; k < R->n; k++)
            prevlab[k] = (lab[k] >= 0) ? nodeof[lab[k]] : -1;
        free(cnt);
        free(nodeof);
        free(fs);
    }
    lvstart[N] = nnodes;

    /* pruning, cudadeblend.cu:422-483 and the level loop of :1425-1470 */
    ok = (int *)malloc(sizeof(int) * nnodes);
    flagv = (int *)malloc(sizeof(int) * nnodes);
    nson = (int *)malloc(sizeof(int) * nnodes);
    for (k = 0; k < nnodes; k++)
        ok[k] = 1;
    value0 = (double)fdflux0 * cfg->deblend_mincont;
    for (L = N - 1; L >= 1; L--) {
        for (k = lvstart[L - 1]; k < lvstart[L]; k++)
            nson[k] = 0;
        for (k = lvstart[L]; k < lvstart[L + 1]; k++) {
            int p = nodes[k].parent;
            float lhs;
            ok[p] &= ok[k];
            lhs = nodes[k].fdflux - nodes[k].dthresh * (float)(unsigned)nodes[k].npix;
            flagv[k] = (lhs > value0);
            if (flagv[k])
                nson[p]++;
        }
        for (k = lvstart[L]; k < lvstart[L + 1]; k++) {
            int p = nodes[k].parent, ns = nson[p];
            if (ns > 1)
                ok[p] = 0;
            ok[k] = (ns > 1 && ok[k] == 1 && flagv[k] == 1) ? 1 : 0;
        }
    }

    /* kept branches in (level, label) order; ownership of their pixels */
    for (k = 0; k < R->n; k++)
        owner[k] = -1;
    for (L = 0; L < N; L++) {
        int any = 0;
        for (k = lvstart[L]; k < lvstart[L + 1]; k++)
            any |= ok[k];
        if (!any)
            continue;
        if (L > 0)
            level_ccl(F, R, bmap, bw, thr[L], par, lab);
        else
            for (k = 0; k < R->n; k++)
                lab[k] = 0;
        for (k = lvstart[L]; k < lvstart[L + 1]; k++) {
            obj_t *o;
            int cntp = 0;
            if (!ok[k])
                continue;
            if (*nobj == *cap) {
                *cap *= 2;
                *objs = (obj_t *)realloc(*objs, sizeof(obj_t) * (*cap));
            }
            o = &(*objs)[*nobj];
            memset(o, 0, sizeof(*o));
            o->root = r;
            o->level = L;
            o->node_dthresh = nodes[k].dthresh;
            o->dthr = R->dthresh;
            o->athr = R->thresh;
            o->nodepix = (int *)malloc(sizeof(int) * nodes[k].npix);
            for (j = 0; j < R->n; j++)
                if (lab[j] == nodes[k].label) {
                    o->nodepix[cntp++] = R->pix[j];
                    owner[j] = nkept;
                }
            o->nnode = cntp;
            (*nobj)++;
            nkept++;
        }
    }
    /* preanalyse_full of every kept branch over its own level pixels
     * (cudadeblend.cu:1670-1712), with the branch threshold */
    for (i = first_obj; i < *nobj; i++) {
        obj_t *o = &(*objs)[i];
        o->flags = 0;
        preanalyse(F, o, o->nodepix, o->nnode, o->node_dthresh, 0);
    }
    /* gatherup, cudadeblend.cu:1262-1360: unassigned pixels go to the kept
     * branch of smallest distance (first in order on ties) */
    for (k = 0; k < R->n; k++) {
        if (owner[k] >= 0)
            continue;
        {
            int p = R->pix[k], x = p % F->w, y = p / F->w, iclst = 0;
            float distmin = 1e+31f, dx, dy, dist;
            for (i = 0; i < nkept; i++) {
                obj_t *o = &(*objs)[first_obj + i];
                dx = x - o->mx;
                dy = y - o->my;
                dist = 0.5 * (o->cxx * dx * dx + o->cyy * dy * dy + o->cxy * dx * dy) / o->abcor;
                if (dist < distmin) {
                    distmin = dist;
                    iclst = i;
                }
            }
            owner[k] = iclst;
        }
    }
    /* final pixel lists (raster order) */
    for (i = 0; i < nkept; i++) {
        obj_t *o = &(*objs)[first_obj + i];
        int c = 0;
        for (k = 0; k < R->n; k++)
            if (owner[k] == i)
                c++;
        o->n = c;
        o->pix = (int *)malloc(sizeof(int) * (c ? c : 1));
        c = 0;
        for (k = 0; k < R->n; k++)
            if (owner[k] == i)
                o->pix[c++] = R->pix[k];
    }
    free(bmap); free(par); free(lab); free(prevlab); free(owner); free(thr);
    free(nodes); free(lvstart); free(ok); free(flagv); free(nson);
    return nkept;
}

/* ------------------------------------------------------------------------ */
static int cmp_float_desc(const void *a, const void *b)
{
    float fa = *(const float *)a, fb = *(const float *)b;
    return (fa < fb) - (fa > fb);
}

/* examineiso, src/cuda/cudaanalyse.cu:2176-2581 (GLOBAL background, CCD). */
/* src/back.c:568-660 (localback): the mode of the background-subtracted
   pixels in a rectangular annulus around the object's box, collected in the
   reference's order (per row the left and right strips, then the rows above,
   then the rows below); 0 when the annulus leaves the frame or holds no
   valid pixel.  *applied tells whether the reference adds the mode to the
   object's background (only when it was measured). */
static float localback(const float *sub, int w, int h, int pbs, int xmin, int xmax, int ymin, int ymax,
                       int *applied)
{
    const int oxsize = xmax - xmin + 1, oysize = ymax - ymin + 1;
    const int bxnml = oxsize < w / 2 ? oxsize / 4 : (w - oxsize) / 4;
    const int bynml = oysize < h / 2 ? oysize / 4 : (h - oysize) / 4;
    const int ixmin = xmin - bxnml, ixmax = xmax + 1 + bxnml, iymin = ymin - bynml, iymax = ymax + 1 + bynml;
    const int bxmin = ixmin - pbs, bxmax = ixmax + pbs, bymin = iymin - pbs, bymax = iymax + pbs;
    float *buf, bkg = 0.0f, sig = 0.0f, pix;
    int n = 0, x, y;
    *applied = 0;
    if (!(bymin >= 0 && bymax < h && bxmin >= 0 && bxmax < w))
        return 0.0f;
    buf = (float *)malloc(sizeof(float) * ((size_t)(bxmax - bxmin) * (bymax - bymin)));
    for (y = bymin; y < bymax; y++) {
        for (x = bxmin; x < bxmin + pbs; x++)
            if ((pix = sub[(size_t)y * w + x]) > -ORC_BIGF)
                buf[n++] = pix;
        for (x = ixmax; x < ixmax + pbs; x++)
            if ((pix = sub[(size_t)y * w + x]) > -ORC_BIGF)
                buf[n++] = pix;
    }
    for (y = bymin; y < iymin; y++)
        for (x = ixmin; x < ixmax; x++)
            if ((pix = sub[(size_t)y * w + x]) > -ORC_BIGF)
                buf[n++] = pix;
    for (y = iymax; y < bymax; y++)
        for (x = ixmin; x < ixmax; x++)
            if ((pix = sub[(size_t)y * w + x]) > -ORC_BIGF)
                buf[n++] = pix;
    if (n) {
        orc_local_stats(buf, n, &bkg, &sig);
        *applied = 1;
    }
    free(buf);
    return bkg;
}

static void examineiso(const frame_t *F, obj_t *o)
{
    const orc_config *cfg = F->cfg;
    int k, i, w = F->w, area = 0, errflag = 1, cleanflag = cfg->clean_flag;
    double esum = 0, emx2 = 0, emy2 = 0, emxy = 0, err, backnoise2, dbacknoise2, xm, ym, x, y, var, sigtv, tvd;
    float peak = -ORC_BIG, cdpeak = -ORC_BIG, pix, cdpix;
    float threshs[ORC_NISO];
    float *heap = NULL;
    xsum_t stv, svar;

    o->bkg = orc_back_at(F->back, F->nbx, F->nby, F->bw, F->bh, (int)(o->mx + 0.5), (int)(o->my + 0.5));
    o->dbkg = 0.0f;
    if (cfg->back_photo_type == 1) {
        int applied;
        o->dbkg = localback(F->sub, F->w, F->h, cfg->back_photo_thick, o->xmin, o->xmax, o->ymin, o->ymax, &applied);
        if (applied)
            o->bkg += o->dbkg;
    }
    dbacknoise2 = F->backsig * F->backsig;
    xm = o->mx;
    ym = o->my;
    var = backnoise2 = F->backsig * F->backsig;
    if (cleanflag) {
        if (o->n < F->minarea) {
            o->mthresh = 0.0;
            cleanflag = 0;
        } else
            heap = (float *)malloc(sizeof(float) * o->n);
    } else
        o->mthresh = 0.0;
    xs_init(&stv);
    xs_init(&svar);
    o->peakx = o->peaky = 0;
    for (k = 0; k < o->n; k++) {
        int p = o->pix[k], ix = p % w, iy = p / w;
        pix = F->sub[p];
        if (pix > peak)
            peak = pix;
        cdpix = F->cd[p];
        if (cdpix > cdpeak) {
            cdpeak = cdpix;
            o->peakx = ix + 1;
            o->peaky = iy + 1;
        }
        if (pix > pix_athr(F, p))
            area++;
        xs_add(&stv, pix);
        if (F->var)
            xs_add(&svar, F->var[p]);
        if (errflag) {
            err = F->var ? (double)F->var[p] : dbacknoise2;
            if (cfg->gain > 0.0 && cdpix > 0.0)
                err += cdpix / cfg->gain;
            x = ix - xm;
            y = iy - ym;
            esum += err;
            emx2 += err * x * x;
            emy2 += err * y * y;
            emxy += err * x * y;
        }
        if (cleanflag)
            heap[k] = cdpix - o->dthr;
    }
    /* mthresh: the minarea-th largest (cd - dthresh), the value the reference
     * heap of src/cuda/cudaanalyse.cu:2331-2365 intends to select */
    if (cleanflag) {
        qsort(heap, o->n, sizeof(float), cmp_float_desc);
        o->mthresh = heap[F->minarea - 1];
        free(heap);
    }
    {
        double flux2 = o->fdflux * o->fdflux;
        emx2 /= flux2;
        emy2 /= flux2;
        emxy /= flux2;
        esum *= 0.08333 / flux2;
        if (o->singuflag && (emx2 * emy2 - emxy * emxy) < esum * esum) {
            emx2 += esum;
            emy2 += esum;
        }
        o->poserr_mx2 = emx2;
        o->poserr_my2 = emy2;
        o->poserr_mxy = emxy;
    }
    /* sigtv accumulates the constant var once per pixel (exact n*var); with a
     * weight map, the pixels' variances (an exact sum) */
    sigtv = F->var ? xs_double(&svar) : (double)o->n * var;
    tvd = xs_double(&stv);
    if (cfg->back_photo_type == 1)
        tvd -= o->n * o->dbkg;  /* int * float: a float product, cudaanalyse.cu:2462 */
    if (cfg->gain > 0.0 && tvd > 0.0)
        sigtv += tvd / cfg->gain;
    o->npix = area;
    o->flux = tvd;
    o->fluxerr = sigtv;
    o->thresh = o->athr - o->dbkg;
    o->peak = peak - o->dbkg;
    if (o->peak > 0.0 && o->thresh > 0.0)
        for (i = 0; i < ORC_NISO; i++)
            threshs[i] = o->thresh * pow((double)o->peak / o->thresh, (double)i / ORC_NISO);
    else
        for (i = 0; i < ORC_NISO; i++)
            threshs[i] = 0.0;
    for (i = 0; i < ORC_NISO; i++)
        o->iso[i] = 0;
    for (k = 0; k < o->n; k++) {
        float v = F->sub[o->pix[k]];
        for (i = 0; i < ORC_NISO && v > threshs[i]; i++)
            o->iso[i]++;
    }
    /* FWHM, cudaanalyse.cu:2521-2578 */
    {
        float thresh0 = o->peak / 5.0;
        if (thresh0 < o->thresh)
            thresh0 = o->thresh;
        if (thresh0 > 0.0) {
            double mx = o->mx, my = o->my, s = 0, sx = 0, sy = 0, sxx = 0, sxy = 0, dx, dy, d2, lpix, pv, b, inverr2, sat, d, bmax;
            sat = (double)(cfg->satur_level - (double)o->dbkg);
            for (k = 0; k < o->n; k++) {
                int p = o->pix[k];
                pv = F->sub[p] - (double)o->dbkg;
                if (pv > thresh0 && pv < sat) {
                    dx = p % w - mx;
                    dy = p / w - my;
                    lpix = log(pv);
                    inverr2 = pv * pv;
                    s += inverr2;
                    d2 = dx * dx + dy * dy;
                    sx += d2 * inverr2;
                    sxx += d2 * d2 * inverr2;
                    sy += lpix * inverr2;
                    sxy += lpix * d2 * inverr2;
                }
            }
            d = s * sxx - sx * sx;
            if (fabs(d) > 0.0) {
                b = -(s * sxy - sx * sy) / d;
                if (b < (bmax = 1 / (13 * o->a * o->b)))
                    b = bmax;
                o->fwhm = (float)(1.6651 / sqrt(b));
                if (o->fwhm > 0.0)
                    o->fwhm -= 1 / (4 * o->fwhm);
            } else
                o->fwhm = 0.0;
        } else
            o->fwhm = 0.0;
    }
}

/* ------------------------------------------------------------------------ */
/* CLEAN: pair test of src/clean.c:108-132 on pre-merge attributes, over all
 * pairs closer than CLEAN_ZONE*(a_i+a_j) (the reference GPU scans an index
 * window instead, src/cuda/cudaclean.cu:120-175); each victim records the
 * smallest index of the objects that eat it. */
static void clean_pair(const frame_t *F, obj_t *o, const double *amp, const double *alpha,
                       int i, int j, int *master)
{
    double beta = F->cfg->clean_param, val;
    float dx, dy, rlim;
    obj_t *oi = &o[i], *oj = &o[j];
    dx = oi->mx - oj->mx;
    dy = oi->my - oj->my;
    rlim = oi->a + oj->a;
    rlim *= rlim;
    if (!(dx * dx + dy * dy < rlim * ORC_CLEAN_ZONE * ORC_CLEAN_ZONE))
        return;
    if (oi->fdflux < oj->fdflux) {
        val = 1 + alpha[j] * (oj->cxx * dx * dx + oj->cyy * dy * dy + oj->cxy * dx * dy);
        if (val > 1.0 && ((float)(val < 1e10 ? amp[j] * (beta == 1.0 ? 1.0 / val : pow(val, -beta)) : 0.0)
                          > oi->mthresh))
            if (master[i] < 0 || j < master[i])
                master[i] = j;
    } else {
        val = 1 + alpha[i] * (oi->cxx * dx * dx + oi->cyy * dy * dy + oi->cxy * dx * dy);
        if (val > 1.0 && ((float)(val < 1e10 ? amp[i] * (beta == 1.0 ? 1.0 / val : pow(val, -beta)) : 0.0)
                          > oj->mthresh))
            if (master[j] < 0 || i < master[j])
                master[j] = i;
    }
}

/* Victims are merged into the end of their master chain (src/clean.c:234-287,
 * mergeobject), victims taken in increasing index order. */
static void merge_into(obj_t *m, const obj_t *s)
{
    m->fdnpix += s->fdnpix;
    m->dnpix += s->dnpix;
    m->fdflux += s->fdflux;
    m->dflux += s->dflux;
    m->flux += s->flux;
    m->fluxerr += s->fluxerr;
    if (s->fdpeak > m->fdpeak) {
        m->fdpeak = s->fdpeak;
        m->peakx = s->peakx;
        m->peaky = s->peaky;
    }
    if (s->dpeak > m->dpeak)
        m->dpeak = s->dpeak;
    if (s->peak > m->peak)
        m->peak = s->peak;
    if (s->xmin < m->xmin) m->xmin = s->xmin;
    if (s->xmax > m->xmax) m->xmax = s->xmax;
    if (s->ymin < m->ymin) m->ymin = s->ymin;
    if (s->ymax > m->ymax) m->ymax = s->ymax;
    m->flags |= (s->flags & (~(ORC_OBJ_MERGED | ORC_OBJ_CROWDED)));
}

static void run_clean(const frame_t *F, obj_t *o, int n)
{
    double beta = F->cfg->clean_param;
    double *amp = (double *)malloc(sizeof(double) * (n + 1));
    double *alpha = (double *)malloc(sizeof(double) * (n + 1));
    int *master = (int *)malloc(sizeof(int) * (n + 1));
    int i, gx, gy, *head, *next, cx, cy;
    const double cell = 32.0;

    /* src/clean.c:105-107 */
    for (i = 0; i < n; i++) {
        double unitarea = ORC_PI * o[i].a * o[i].b, q;
        amp[i] = o[i].fdflux / (2 * unitarea * o[i].abcor);
        q = amp[i] / o[i].dthr;
        alpha[i] = ((beta == 1.0 ? q : pow(q, 1.0 / beta)) - 1) * unitarea / o[i].fdnpix;
        master[i] = -1;
    }
    /* candidate pairs from a grid: a pair can only pass the zone test if
     * its distance is below 20*max(a_i, a_j); the object of larger a (lower
     * index on ties) searches. */
    gx = (int)(F->w / cell) + 2;
    gy = (int)(F->h / cell) + 2;
    head = (int *)malloc(sizeof(int) * gx * gy);
    next = (int *)malloc(sizeof(int) * (n + 1));
    for (i = 0; i < gx * gy; i++)
        head[i] = -1;
    for (i = n - 1; i >= 0; i--) {
        cx = (int)floor(o[i].mx / cell);
        cy = (int)floor(o[i].my / cell);
        if (cx < 0) cx = 0;
        if (cy < 0) cy = 0;
        if (cx >= gx) cx = gx - 1;
        if (cy >= gy) cy = gy - 1;
        next[i] = head[cy * gx + cx];
        head[cy * gx + cx] = i;
    }
    for (i = 0; i < n; i++) {
        double rad = 20.0 * o[i].a * 1.001 + 2.0;
        int x0 = (int)floor((o[i].mx - rad) / cell), x1 = (int)floor((o[i].mx + rad) / cell);
        int y0 = (int)floor((o[i].my - rad) / cell), y1 = (int)floor((o[i].my + rad) / cell);
        if (x0 < 0) x0 = 0;
        if (y0 < 0) y0 = 0;
        if (x1 >= gx) x1 = gx - 1;
        if (y1 >= gy) y1 = gy - 1;
        for (cy = y0; cy <= y1; cy++)
            for (cx = x0; cx <= x1; cx++) {
                int j;
                for (j = head[cy * gx + cx]; j >= 0; j = next[j]) {
                    if (j == i)
                        continue;
                    if (o[j].a < o[i].a || (o[j].a == o[i].a && j > i)) {
                        if (i < j)
                            clean_pair(F, o, amp, alpha, i, j, master);
                        else
                            clean_pair(F, o, amp, alpha, j, i, master);
                    }
                }
            }
    }
    for (i = 0; i < n; i++) {
        int m = master[i];
        while (m >= 0 && master[m] >= 0)
            m = master[m];
        o[i].master = master[i];
        o[i].final_master = m;
    }
    for (i = 0; i < n; i++)
        if (o[i].final_master >= 0)
            merge_into(&o[o[i].final_master], &o[i]);
    free(amp); free(alpha); free(master); free(head); free(next);
}

/* ------------------------------------------------------------------------ */
#define ALLOC_OTHER 0x7fffffff

/* src/cuda/cudaanalyse.cu:104-287 (computeaperflux, one aperture, CCD).
 * Pixels at or below -BIG (blank or NaN input pixels) are replaced like
 * pixels of other objects, as the CPU computeaperflux does (src/photom.c:128-
 * 145): the GPU kernel drops that test and would sum the -BIG sentinel. */
static void aperflux(const frame_t *F, const int *alloc, obj_t *o, int self, double diameter, int k)
{
    const orc_config *cfg = F->cfg;
    float r2, raper, raper2, rintlim, rintlim2, rextlim2, dx, dx1, dy, dy2, offsetx, offsety, scalex, scaley, scale2, locarea;
    double tv, sigtv, area, pix, var, pvar;
    int x, y, x2, y2, xmin, xmax, ymin, ymax, sx, sy, corrflag, w = F->w, h = F->h, t;

    corrflag = (cfg->mask_type == 2);
    var = F->backsig * F->backsig;
    raper = diameter / 2.0;
    raper2 = raper * raper;
    rintlim = raper - 0.75;
    rintlim2 = (rintlim > 0.0) ? rintlim * rintlim : 0.0;
    rextlim2 = (raper + 0.75) * (raper + 0.75);
    tv = sigtv = area = 0.0;
    scaley = scalex = 1.0 / ORC_APER_OVERSAMP;
    scale2 = scalex * scaley;
    offsetx = 0.5 * (scalex - 1.0);
    offsety = 0.5 * (scaley - 1.0);
    xmin = (int)(o->mx - raper + 0.499999);
    xmax = (int)(o->mx + raper + 1.499999);
    ymin = (int)(o->my - raper + 0.499999);
    ymax = (int)(o->my + raper + 1.499999);
    if (xmin < 0) { xmin = 0; o->flags |= ORC_OBJ_APERT_PB; }
    if (xmax > w) { xmax = w; o->flags |= ORC_OBJ_APERT_PB; }
    if (ymin < 0) { ymin = 0; o->flags |= ORC_OBJ_APERT_PB; }
    if (ymax > h) { ymax = h; o->flags |= ORC_OBJ_APERT_PB; }
    for (y = ymin; y < ymax; y++)
        for (x = xmin; x < xmax; x++) {
            dx = x - o->mx;
            dy = y - o->my;
            if ((r2 = dx * dx + dy * dy) < rextlim2) {
                if (r2 > rintlim2) {
                    dx += offsetx;
                    dy += offsety;
                    locarea = 0.0;
                    for (sy = ORC_APER_OVERSAMP; sy--; dy += scaley) {
                        dx1 = dx;
                        dy2 = dy * dy;
                        for (sx = ORC_APER_OVERSAMP; sx--; dx1 += scalex)
                            if (dx1 * dx1 + dy2 < raper2)
                                locarea += scale2;
                    }
                } else
                    locarea = 1.0;
                area += locarea;
                pix = F->sub[(size_t)y * w + x];
                t = alloc[(size_t)y * w + x];
                /* with a weight map the variance of the pixel actually used,
                 * 0 for a pixel replaced by 0 (src/photom.c:128-145) */
                pvar = F->var ? (double)F->var[(size_t)y * w + x] : var;
                if ((t >= 0 && t != self) || pix <= -ORC_BIG) {
                    if (corrflag && (x2 = (int)(2 * o->mx + 0.49999 - x)) >= 0 && x2 < w
                        && (y2 = (int)(2 * o->my + 0.49999 - y)) >= 0 && y2 < h
                        && ((t = alloc[(size_t)y2 * w + x2]) == self || t == -1)
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
        }
    tv -= area * o->dbkg;
    if (cfg->gain > 0.0 && tv > 0.0)
        sigtv += tv / cfg->gain;
    o->aper[k][0] = tv;
    o->aper[k][1] = sqrt(sigtv);
    o->aper[k][2] = tv > 0.0 ? -2.5 * log10(tv) + cfg->mag_zeropoint : 99.0;
    o->aper[k][3] = tv > 0.0 ? 1.086 * sqrt(sigtv) / tv : 99.0;
    if (k == 0) {
        o->flux_aper = o->aper[0][0];
        o->fluxerr_aper = o->aper[0][1];
        o->mag_aper = o->aper[0][2];
        o->magerr_aper = o->aper[0][3];
    }
}

#define RINT(x) (int)(floor(x + 0.5))

/* src/cuda/cudaanalyse.cu:293-592 (computeautoflux, CCD, no weights).  The
 * sums r1, v1 and tv are exact order-free sums of the float terms the kernel
 * accumulates.  In the flux pass, pixels at or below -BIG count as bad and are
 * replaced as in the CPU computeautoflux (src/photom.c:640-657). */
static void autoflux(const frame_t *F, const int *alloc, obj_t *o, int self)
{
    const orc_config *cfg = F->cfg;
    double sigtv, tv, r1, v1, var;
    float dx, dy, cx2, cy2, cxy, r2, klim2, dxlim, dylim, pix;
    int area, areab, x, y, x2, y2, xmin, xmax, ymin, ymax, corrflag, t, w = F->w, h = F->h;
    xsum_t sr1, sv1, stv, svar;
    const double autoaper0 = 0.0, autoaper1 = 0.0;

    var = F->backsig * F->backsig;
    corrflag = (cfg->mask_type == 2);
    if (ORC_KRON_NSIG * sqrtf(o->a * o->b) > autoaper0 / 2.0) {
        cx2 = o->cxx;
        cy2 = o->cyy;
        cxy = o->cxy;
        dxlim = cx2 - cxy * cxy / (4.0 * cy2);
        dxlim = dxlim > 0.0 ? ORC_KRON_NSIG / sqrtf(dxlim) : 0.0;
        dylim = cy2 - cxy * cxy / (4.0 * cx2);
        dylim = dylim > 0.0 ? ORC_KRON_NSIG / sqrtf(dylim) : 0.0;
        klim2 = ORC_KRON_NSIG * ORC_KRON_NSIG;
    } else {
        cx2 = cy2 = 1.0;
        cxy = 0.0;
        dxlim = dylim = autoaper0 / 2.0;
        klim2 = dxlim * dxlim;
    }
    if ((xmin = RINT(o->mx - dxlim)) < 0) { xmin = 0; o->flags |= ORC_OBJ_APERT_PB; }
    if ((xmax = RINT(o->mx + dxlim) + 1) > w) { xmax = w; o->flags |= ORC_OBJ_APERT_PB; }
    if ((ymin = RINT(o->my - dylim)) < 0) { ymin = 0; o->flags |= ORC_OBJ_APERT_PB; }
    if ((ymax = RINT(o->my + dylim) + 1) > h) { ymax = h; o->flags |= ORC_OBJ_APERT_PB; }
    xs_init(&sr1);
    xs_init(&sv1);
    area = areab = 0;
    for (y = ymin; y < ymax; y++)
        for (x = xmin; x < xmax; x++) {
            dx = x - o->mx;
            dy = y - o->my;
            if ((r2 = cx2 * dx * dx + cy2 * dy * dy + cxy * dx * dy) <= klim2) {
                pix = F->sub[(size_t)y * w + x];
                t = alloc[(size_t)y * w + x];
                if ((t == self || t == -1) & (pix > -ORC_BIG)) {
                    area++;
                    xs_add(&sr1, sqrtf(r2) * pix);
                    xs_add(&sv1, pix);
                } else
                    areab++;
            }
        }
    area += areab;
    r1 = xs_double(&sr1);
    v1 = xs_double(&sv1);
    if (area) {
        if (r1 > 0.0 && v1 > 0.0) {
            o->kron = cfg->phot_autoparams[0] * r1 / v1;
            if (o->kron < cfg->phot_autoparams[1])
                o->kron = cfg->phot_autoparams[1];
        } else
            o->kron = cfg->phot_autoparams[1];
        if ((float)areab / area > ORC_CROWD_THRESHOLD)
            o->flags |= ORC_OBJ_CROWDED;
        if (o->kron * sqrtf(o->a * o->b) > autoaper1 / 2.0) {
            cx2 = o->cxx;
            cy2 = o->cyy;
            cxy = o->cxy;
            dxlim = cx2 - cxy * cxy / (4.0 * cy2);
            dxlim = dxlim > 0.0 ? o->kron / sqrtf(dxlim) : 0.0;
            dylim = cy2 - cxy * cxy / (4.0 * cx2);
            dylim = dylim > 0.0 ? o->kron / sqrtf(dylim) : 0.0;
            klim2 = o->kron * o->kron;
        } else {
            cx2 = cy2 = 1.0;
            cxy = 0.0;
            dxlim = dylim = autoaper1 / 2.0;
            klim2 = dxlim * dxlim;
            o->kron = 0.0;
        }
        if ((xmin = RINT(o->mx - dxlim)) < 0) { xmin = 0; o->flags |= ORC_OBJ_APERT_PB; }
        if ((xmax = RINT(o->mx + dxlim) + 1) > w) { xmax = w; o->flags |= ORC_OBJ_APERT_PB; }
        if ((ymin = RINT(o->my - dylim)) < 0) { ymin = 0; o->flags |= ORC_OBJ_APERT_PB; }
        if ((ymax = RINT(o->my + dylim) + 1) > h) { ymax = h; o->flags |= ORC_OBJ_APERT_PB; }
        area = areab = 0;
        xs_init(&stv);
        xs_init(&svar);
        for (y = ymin; y < ymax; y++)
            for (x = xmin; x < xmax; x++) {
                dx = x - o->mx;
                dy = y - o->my;
                if ((cx2 * dx * dx + cy2 * dy * dy + cxy * dx * dy) <= klim2) {
                    float pvar;
                    area++;
                    pix = F->sub[(size_t)y * w + x];
                    t = alloc[(size_t)y * w + x];
                    pvar = F->var ? F->var[(size_t)y * w + x] : 0.0f;
                    if ((t >= 0 && t != self) || pix <= -ORC_BIG) {
                        areab++;
                        if (corrflag && (x2 = (int)(2 * o->mx + 0.49999 - x)) >= 0 && x2 < w
                            && (y2 = (int)(2 * o->my + 0.49999 - y)) >= 0 && y2 < h
                            && ((t = alloc[(size_t)y2 * w + x2]) == -1 || t == self)
                            && F->sub[(size_t)y2 * w + x2] > -ORC_BIG) {
                            pix = F->sub[(size_t)y2 * w + x2];
                            if (F->var)
                                pvar = F->var[(size_t)y2 * w + x2];
                        } else {
                            pix = 0.0;
                            pvar = 0.0f;
                        }
                    }
                    xs_add(&stv, pix);
                    if (F->var)
                        xs_add(&svar, pvar);
                }
            }
        if ((float)areab > ORC_CROWD_THRESHOLD * area)
            o->flags |= ORC_OBJ_CROWDED;
        tv = xs_double(&stv);
        sigtv = F->var ? xs_double(&svar) : (double)area * var;
        tv -= area * (double)o->dbkg;
        if (cfg->gain > 0.0 && tv > 0.0)
            sigtv += tv / cfg->gain;
    } else
        tv = sigtv = 0.0;
    o->flux_auto = tv;
    o->fluxerr_auto = sqrt(sigtv);
    o->mag_auto = o->flux_auto > 0.0 ? -2.5 * log10(o->flux_auto) + cfg->mag_zeropoint : 99.0;
    o->magerr_auto = o->flux_auto > 0.0 ? 1.086 * o->fluxerr_auto / o->flux_auto : 99.0;
    if (tv <= 0.0)
        o->kron = 0.0;
}

/* endobject, src/cuda/cudaanalyse.cu:2604-2900 (the parts that feed the catalog) */
/* CLASS_STAR: src/cuda/cudaanalyse.cu:2901-2920 (inputs) and :599-632 /
   src/neurro.c neurresp (response, logistic units, double arithmetic) */
/* src/neurro.c:57-78 (neurresp): the network's layers in double with
 * logistic units (src/neurro.c:85-89); in[] holds nn[0] inputs and is
 * overwritten; returns the first output */
static double nnw_response(const orc_nnw *net, double *in)
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

static float class_star(const orc_config *cfg, const obj_t *o)
{
    const orc_nnw *net = cfg->nnw;
    double in[ORC_NNW_NEURONS], fac2, fwhm = cfg->seeing_fwhm;
    double pixscale = cfg->pixel_scale > 0.0 ? cfg->pixel_scale : 1.0;
    int i, j = 0;
    fac2 = fwhm / pixscale;
    fac2 *= fac2;
    in[j] = log10(o->iso[0] ? o->iso[0] / fac2 : 0.01);
    in[++j] = o->athr > 0.0 ? log10(o->peak > 0.0 ? o->peak / o->athr : 0.1) : -1.0;
    for (i = 1; i < ORC_NISO; i++)
        in[++j] = log10(o->iso[i] ? o->iso[i] / fac2 : 0.01);
    in[++j] = log10(fwhm);
    return (float)nnw_response(net, in);
}

/* computeisocorflux, src/cuda/cudaanalyse.cu:62-98 (src/photom.c:719) */
static void isocorflux(obj_t *o)
{
    double ati = (o->flux > 0.0) ? (o->fdnpix * o->dthr / o->flux) : 0.0;
    if (ati > 1.0)
        ati = 1.0;
    else if (ati < 0.0)
        ati = 0.0;
    o->flux_isocor = o->flux / (1.0 - 0.196099 * ati - 0.751208 * ati * ati);
    if (o->flux > 0.0) {
        double dati, sigtv;
        sigtv = o->fluxerr / (o->flux * o->flux);
        dati = o->fdnpix ? ati * sqrt(sigtv + 1.0 / o->fdnpix) : 0.0;
        dati = 0.196099 * dati + 0.751208 * 2 * ati * dati;
        o->fluxerr_isocor = sqrt(sigtv + dati * dati) * o->flux;
    } else
        o->fluxerr_isocor = sqrt(o->fluxerr);
}

static void endobject(const frame_t *F, const int *alloc, obj_t *o, int self)
{
    const orc_config *cfg = F->cfg;
    o->elong = o->a / o->b;
    o->ellip = 1 - o->b / o->a;
    o->polar = (o->a * o->a - o->b * o->b) / (o->a * o->a + o->b * o->b);
    o->fluxerr_iso = sqrt(o->fluxerr);
    isocorflux(o);
    {
        /* every PHOT_APERTURES diameter, in order */
        int k, na = cfg->naper > 0 ? cfg->naper : 1;
        for (k = 0; k < na; k++)
            aperflux(F, alloc, o, self, cfg->naper > 0 ? cfg->phot_apertures[k] : cfg->phot_aperture, k);
    }
    autoflux(F, alloc, o, self);
    if (o->peak + o->bkg >= cfg->satur_level)
        o->flags |= ORC_OBJ_SATUR;
    o->mag_iso = o->flux > 0.0 ? -2.5 * log10(o->flux) + cfg->mag_zeropoint : 99.0;
    o->magerr_iso = o->flux > 0.0 ? 1.086 * o->fluxerr_iso / o->flux : 99.0;
    o->class_star = cfg->nnw ? class_star(cfg, o) : 0.0f;
}

/* ------------------------------------------------------------------------ */
/* rows of the FP64 twin asked for by orc_set_fp64_rows (one extraction) */
static orc_object64 *g_out64;
static int g_max64;

void orc_set_fp64_rows(orc_object64 *out, int max)
{
    g_out64 = out;
    g_max64 = max;
}

typedef struct {
    int ymax, lastx, idx;
} okey_t;

static int cmp_okey(const void *a, const void *b)
{
    const okey_t *p = (const okey_t *)a, *q = (const okey_t *)b;
    if (p->ymax != q->ymax) return p->ymax < q->ymax ? -1 : 1;
    if (p->lastx != q->lastx) return p->lastx < q->lastx ? -1 : 1;
    return (p->idx > q->idx) - (p->idx < q->idx);
}

/* ------------------------------------------------------------------------ */
/* Weight maps.  The reference keeps weight_to_var (src/weight.c:91-125) but
 * no weighted background, threshold or measurement; this restates them after
 * the SExtractor manual (weight maps): unusable pixels (variance or rms at or
 * above BIG, weight at or below 0, NaN) are blank for the background and the
 * detection; the relative map is scaled by sigfac^2 (MAP_VAR, MAP_WEIGHT) with
 * sigfac the median over usable meshes of (mesh rms of the frame) /
 * sqrt(mesh mean of the relative variance), or used as it is (MAP_RMS). */
static float rel_var(float v, int wtype)
{
    float r;
    if (wtype == 1)
        r = v;
    else if (wtype == 2)
        r = v < ORC_BIGF ? v * v : ORC_BIGF;
    else
        r = v > 0.0f ? 1.0f / v : ORC_BIGF;
    return r < ORC_BIGF ? r : ORC_BIGF;  /* NaN and overflow too */
}

/* src/weight.c:104-118 with the scale factor */
static float calib_var(float v, int wtype, float sigfac2)
{
    float r;
    if (wtype == 1)
        r = v < ORC_BIGF ? v * sigfac2 : ORC_BIGF;
    else if (wtype == 2)
        r = v < ORC_BIGF ? v * v : ORC_BIGF;
    else
        r = v > 0.0f ? sigfac2 / v : ORC_BIGF;
    return r < ORC_BIGF ? r : ORC_BIGF;
}

/* sigfac from the frame's filtered mesh rms map `sigma` */
static float weight_sigfac(const float *wmap, int wtype, int w, int h, int bw, int bh, int nx, int ny,
                           const float *sigma)
{
    float *ratio = (float *)malloc(sizeof(float) * nx * ny), f;
    int nr = 0, mx, my, x, y;
    if (wtype == 2) {
        free(ratio);
        return 1.0f;
    }
    for (my = 0; my < ny; my++) {
        int mh = (my == ny - 1 && h % bh) ? h % bh : bh;
        for (mx = 0; mx < nx; mx++) {
            int mw = (mx == nx - 1 && w % bw) ? w % bw : bw, n = 0;
            xsum_t sv;
            double vmean;
            float sm = sigma[my * nx + mx];
            xs_init(&sv);
            for (y = 0; y < mh; y++)
                for (x = 0; x < mw; x++) {
                    float r = rel_var(wmap[(size_t)(my * bh + y) * w + mx * bw + x], wtype);
                    if (r < ORC_BIGF) {
                        xs_add(&sv, r);
                        n++;
                    }
                }
            if ((float)n < (float)(mw * mh * ORC_BACK_MINGOODFRAC))
                continue;
            vmean = xs_double(&sv) / n;
            if (vmean > 0.0 && sm > 0.0f)
                ratio[nr++] = (float)(sm / sqrt(vmean));
        }
    }
    f = nr ? orc_hmedian(ratio, nr) : 1.0f;
    free(ratio);
    return f;
}

/* LOCAL photometry background of objects given by their boxes (xmin, xmax,
   ymin, ymax per object, 0-based) over a background-subtracted frame */
void orc_localback(const float *sub, int w, int h, int thick, const int *box, int nobj, float *dbkg)
{
    int i, applied;
    for (i = 0; i < nobj; i++)
        dbkg[i] = localback(sub, w, h, thick, box[4 * i], box[4 * i + 1], box[4 * i + 2], box[4 * i + 3], &applied);
}

int orc_extract(const float *img, const float *var, int w, int h, const orc_config *cfg,
                orc_object *out, int max_objects, int32_t *segmap,
                float *sub_out, float *cd_out, orc_summary *sum)
{
    orc_summary S;
    frame_t F;
    float *sub, *cd, *back;
    int *lab, *alloc;
    size_t N = (size_t)w * h, p;
    int nroots = 0, r, i, k, nobj = 0, cap = 1024, nout = 0;
    float *wvar;
    root_t *roots;
    int *rootid;
    obj_t *objs;
    (void)var;

    memset(&S, 0, sizeof(S));
    S.sigfac = 1.0f;
    sub = (float *)malloc(sizeof(float) * N);
    cd = (float *)malloc(sizeof(float) * N);
    memcpy(sub, img, sizeof(float) * N);
    wvar = NULL;
    if (var && cfg->weight_type >= 1 && cfg->weight_type <= 3) {
        /* unusable weight: a blank pixel */
        for (p = 0; p < N; p++)
            if (!(rel_var(var[p], cfg->weight_type) < ORC_BIGF))
                sub[p] = -ORC_BIGF;
    } else
        var = NULL;
    {
        int bw = cfg->back_size < w ? cfg->back_size : w, bh = cfg->back_size < h ? cfg->back_size : h;
        int nbx = (w - 1) / bw + 1, nby = (h - 1) / bh + 1;
        float *sig = (float *)malloc(sizeof(float) * nbx * nby);
        back = (float *)malloc(sizeof(float) * nbx * nby);
        orc_background(sub, w, h, cfg, back, sig, NULL, NULL, &S);
        if (cfg->weight_type == 4) {
            /* WEIGHT_TYPE BACKGROUND: variance = (background rms map)^2 */
            wvar = (float *)malloc(sizeof(float) * N);
            orc_background_rms(img, w, h, cfg, wvar);
            for (p = 0; p < N; p++)
                wvar[p] = wvar[p] * wvar[p];
        } else if (var) {
            float sigfac2;
            S.sigfac = weight_sigfac(var, cfg->weight_type, w, h, bw, bh, nbx, nby, sig);
            sigfac2 = S.sigfac * S.sigfac;
            wvar = (float *)malloc(sizeof(float) * N);
            for (p = 0; p < N; p++)
                wvar[p] = calib_var(var[p], cfg->weight_type, sigfac2);
        }
        free(sig);
        F.nbx = nbx;
        F.nby = nby;
        F.bw = bw;
        F.bh = bh;
    }
    if (cfg->filter_flag)
        orc_filter(sub, w, h, cfg->conv, cfg->conv_w, cfg->conv_h, cd);
    else
        memcpy(cd, sub, sizeof(float) * N);
    F.w = w;
    F.h = h;
    F.sub = sub;
    F.cd = cd;
    F.cfg = cfg;
    F.dthresh = S.dthresh;
    F.thresh = S.thresh;
    F.backsig = S.backsig;
    F.back = back;
    F.minarea = cfg->detect_minarea;
    F.debminarea = cfg->detect_minarea < ORC_MAXDEBAREA ? cfg->detect_minarea : ORC_MAXDEBAREA;
    F.var = wvar;
    F.wthr = wvar != NULL && cfg->thresh_type != 1;

    /* thresholding + 8-connected components, src/cuda/cudadetection.cu:36-276 */
    lab = (int *)malloc(sizeof(int) * N);
    for (p = 0; p < N; p++)
        lab[p] = (!pix_bad(&F, p) && cd[p] >= pix_dthr(&F, p)) ? (int)p : -1;
    for (p = 0; p < N; p++) {
        int x = p % w, y = p / w;
        if (lab[p] < 0)
            continue;
        S.npix_above++;
        if (x > 0 && lab[p - 1] >= 0) uf_union(lab, p, p - 1);
        if (y > 0) {
            if (x > 0 && lab[p - w - 1] >= 0) uf_union(lab, p, p - w - 1);
            if (lab[p - w] >= 0) uf_union(lab, p, p - w);
            if (x < w - 1 && lab[p - w + 1] >= 0) uf_union(lab, p, p - w + 1);
        }
    }
    /* raw objects: components of at least DETECT_MINAREA pixels, in order of
     * their first pixel (cudadetection.cu:677-897) */
    {
        int *cnt = (int *)calloc(N, sizeof(int));
        rootid = (int *)malloc(sizeof(int) * N);
        for (p = 0; p < N; p++)
            if (lab[p] >= 0) {
                lab[p] = uf_find(lab, p);
                cnt[lab[p]]++;
            }
        for (p = 0; p < N; p++) {
            rootid[p] = -1;
            if (lab[p] == (int)p && cnt[p] >= F.minarea)
                rootid[p] = nroots++;
        }
        roots = (root_t *)calloc(nroots ? nroots : 1, sizeof(root_t));
        for (p = 0; p < N; p++)
            if (lab[p] == (int)p && rootid[p] >= 0) {
                root_t *R = &roots[rootid[p]];
                R->pix = (int *)malloc(sizeof(int) * cnt[p]);
                R->firstpix = p;
                R->xmin = w;
                R->ymin = h;
                R->xmax = R->ymax = -1;
                R->fdpeak = -ORC_BIG;
                R->dthresh = R->thresh = ORC_BIGF;
                xs_init(&R->fdflux);
            }
        for (p = 0; p < N; p++)
            if (lab[p] >= 0 && rootid[lab[p]] >= 0) {
                root_t *R = &roots[rootid[lab[p]]];
                int x = p % w, y = p / w;
                R->pix[R->n++] = p;
                if (x < R->xmin) R->xmin = x;
                if (x > R->xmax) R->xmax = x;
                if (y < R->ymin) R->ymin = y;
                if (y > R->ymax) { R->ymax = y; R->lastrow_x = x; }
                if (cd[p] > R->fdpeak) R->fdpeak = cd[p];
                xs_add(&R->fdflux, cd[p]);
                if (pix_dthr(&F, p) < R->dthresh) R->dthresh = pix_dthr(&F, p);
                if (pix_athr(&F, p) < R->thresh) R->thresh = pix_athr(&F, p);
            }
        for (p = 0; p < N; p++)
            rootid[p] = (lab[p] >= 0) ? rootid[lab[p]] : -1;
        free(cnt);
    }
    S.nraw = nroots;
    for (r = 0; r < nroots; r++)
        S.nraw_pix += roots[r].n;

    /* deblending */
    objs = (obj_t *)malloc(sizeof(obj_t) * cap);
    for (r = 0; r < nroots; r++)
        deblend_root(&F, r, &roots[r], &objs, &nobj, &cap);
    S.ndetected = nobj;

    /* analysis: robust preanalysis of deblended objects, then examineiso */
    for (i = 0; i < nobj; i++) {
        obj_t *o = &objs[i];
        if (o->level > 0)
            preanalyse(&F, o, o->pix, o->n, o->dthr, 1);
        o->fdnpix = o->n;
        o->master = o->final_master = -1;
        examineiso(&F, o);
    }
    if (cfg->clean_flag == 1)
        run_clean(&F, objs, nobj);

    /* allocation map: object (after CLEAN merges) or OTHER for above
     * threshold pixels outside every object, -1 elsewhere */
    alloc = (int *)malloc(sizeof(int) * N);
    for (p = 0; p < N; p++)
        alloc[p] = (!pix_bad(&F, p) && cd[p] >= pix_dthr(&F, p)) ? ALLOC_OTHER : -1;
    for (i = 0; i < nobj; i++) {
        int m = objs[i].final_master >= 0 ? objs[i].final_master : i;
        for (k = 0; k < objs[i].n; k++)
            alloc[objs[i].pix[k]] = m;
    }
    for (i = 0; i < nobj; i++)
        if (objs[i].final_master < 0)
            endobject(&F, alloc, &objs[i], i);

    /* catalog order and NUMBER */
    {
        okey_t *keys = (okey_t *)malloc(sizeof(okey_t) * (nobj + 1));
        int *number = (int *)calloc(nobj + 1, sizeof(int));
        int ns = 0;
        for (i = 0; i < nobj; i++)
            if (objs[i].final_master < 0) {
                root_t *R = &roots[objs[i].root];
                keys[ns].ymax = cfg->numbering == 0 ? R->ymax : 0;
                keys[ns].lastx = cfg->numbering == 0 ? R->lastrow_x : 0;
                keys[ns].idx = i;
                ns++;
            }
        qsort(keys, ns, sizeof(okey_t), cmp_okey);
        for (k = 0; k < ns; k++)
            number[keys[k].idx] = k + 1;
        if (g_out64) {
            int *rows = (int *)malloc(sizeof(int) * (ns + 1));
            for (k = 0; k < ns; k++)
                rows[k] = keys[k].idx;
            orc_measure64(&F, alloc, objs, nobj, rows, ns < g_max64 ? ns : g_max64, g_out64);
            free(rows);
            g_out64 = NULL;
        }
        for (k = 0; k < ns && nout < max_objects; k++) {
            obj_t *o = &objs[keys[k].idx];
            orc_object *q = &out[nout++];
            memset(q, 0, sizeof(*q));
            q->number = k + 1;
            q->root = o->root;
            q->level = o->level;
            q->fdnpix = o->fdnpix;
            q->dnpix = o->dnpix;
            q->npix = o->npix;
            q->xmin = o->xmin; q->xmax = o->xmax; q->ymin = o->ymin; q->ymax = o->ymax;
            q->peakx = o->peakx; q->peaky = o->peaky;
            q->flags = o->flags;
            for (i = 0; i < ORC_NISO; i++)
                q->iso[i] = o->iso[i];
            q->fdflux = o->fdflux; q->dflux = o->dflux; q->flux = o->flux; q->fluxerr = o->fluxerr;
            q->fdpeak = o->fdpeak; q->dpeak = o->dpeak; q->peak = o->peak;
            q->mx = o->mx; q->my = o->my; q->mx2 = o->mx2; q->my2 = o->my2; q->mxy = o->mxy;
            q->a = o->a; q->b = o->b; q->theta = o->theta; q->abcor = o->abcor;
            q->cxx = o->cxx; q->cyy = o->cyy; q->cxy = o->cxy; q->class_star = o->class_star;
            q->poserr_mx2 = o->poserr_mx2; q->poserr_my2 = o->poserr_my2; q->poserr_mxy = o->poserr_mxy;
            q->bkg = o->bkg; q->thresh = o->thresh; q->dthresh = o->dthr; q->mthresh = o->mthresh;
            q->fwhm = o->fwhm;
            q->flux_iso = o->flux; q->fluxerr_iso = o->fluxerr_iso; q->mag_iso = o->mag_iso; q->magerr_iso = o->magerr_iso;
            q->flux_isocor = o->flux_isocor; q->fluxerr_isocor = o->fluxerr_isocor;
            q->flux_aper = o->flux_aper; q->fluxerr_aper = o->fluxerr_aper;
            q->mag_aper = o->mag_aper; q->magerr_aper = o->magerr_aper;
            q->kronfactor = o->kron; q->flux_auto = o->flux_auto; q->fluxerr_auto = o->fluxerr_auto;
            q->mag_auto = o->mag_auto; q->magerr_auto = o->magerr_auto;
            q->elong = o->elong; q->ellip = o->ellip; q->polar = o->polar;
            memcpy(q->aper, o->aper, sizeof(q->aper));
        }
        if (segmap) {
            for (p = 0; p < N; p++)
                segmap[p] = 0;
            for (i = 0; i < nobj; i++) {
                int m = objs[i].final_master >= 0 ? objs[i].final_master : i;
                for (k = 0; k < objs[i].n; k++)
                    segmap[objs[i].pix[k]] = number[m];
            }
        }
        S.nobj = ns;
        free(keys);
        free(number);
    }
    if (sub_out) memcpy(sub_out, sub, sizeof(float) * N);
    if (cd_out) memcpy(cd_out, cd, sizeof(float) * N);
    if (sum) *sum = S;
    for (i = 0; i < nobj; i++) {
        free(objs[i].nodepix);
        free(objs[i].pix);
    }
    for (r = 0; r < nroots; r++)
        free(roots[r].pix);
    free(objs); free(roots); free(rootid); free(lab); free(alloc); free(sub); free(cd); free(back); free(wvar);
    return nout;
}

/* ------------------------------------------------------------------------ */
/* src/filter.c:101-185 (getconv) */
int orc_getconv(const char *path, float *mask, int maxn, int *mw, int *mh)
{
    FILE *f = fopen(path, "r");
    char str[512], *tok;
    int i = 0, j, n = 0, normflag;
    double sum = 0.0, var = 0.0, pix;
    if (!f)
        return -1;
    if (!fgets(str, sizeof(str), f) || strncmp(str, "CONV", 4)) {
        fclose(f);
        return -2;
    }
    normflag = strstr(str, "NORM") ? (strstr(str, "NONORM") ? 0 : 1) : 1;
    while (fgets(str, sizeof(str), f)) {
        j = 0;
        tok = strtok(str, " \t\n");
        if (tok && tok[0] != '#')
            do {
                j++;
                if (i >= maxn) {
                    fclose(f);
                    return -3;
                }
                mask[i++] = (float)atof(tok);
            } while ((tok = strtok(NULL, " \t\n")));
        if (j > n)
            n = j;
    }
    fclose(f);
    if (n < 1 || i % n)
        return -4;
    *mw = n;
    *mh = i / n;
    for (j = 0; j < i; j++) {
        sum += fabs(pix = mask[j]);
        var += pix * pix;
    }
    var = sqrt(var);
    if (normflag) {
        if (sum == 0.0)
            sum = var;
        for (j = 0; j < i; j++)
            mask[j] /= sum;
    }
    return i;
}

double orc_xsum_floats(const float *v, int n, int e0)
{
    xsum_t s;
    int i;
    (void)e0;
    xs_init(&s);
    for (i = 0; i < n; i++)
        xs_add(&s, v[i]);
    return xs_double(&s);
}

/* ------------------------------------------------------------------------ */
/* Unit-level entry points.  The tests compare them with the reference's own
 * src/photom.c, src/clean.c and src/neurro.c compiled unmodified
 * (oracle/_ref). */

/* Aperture and AUTO photometry (aperflux, autoflux above) of objects given
 * by their position and shape over a background-subtracted frame in which no
 * pixel belongs to another object. */
int orc_photometry(const float *sub, int w, int h, const orc_config *cfg, float backsig, orc_phot_obj *po, int n)
{
    frame_t F;
    obj_t o;
    int i, *alloc = (int *)malloc(sizeof(int) * (size_t)w * h);
    if (!alloc)
        return -1;
    for (i = 0; i < w * h; i++)
        alloc[i] = -1;
    memset(&F, 0, sizeof(F));
    F.w = w;
    F.h = h;
    F.sub = sub;
    F.cfg = cfg;
    F.backsig = backsig;
    for (i = 0; i < n; i++) {
        memset(&o, 0, sizeof(o));
        o.mx = po[i].mx;
        o.my = po[i].my;
        o.a = po[i].a;
        o.b = po[i].b;
        o.cxx = po[i].cxx;
        o.cyy = po[i].cyy;
        o.cxy = po[i].cxy;
        o.dbkg = po[i].dbkg;
        aperflux(&F, alloc, &o, 0, cfg->phot_aperture, 0);
        autoflux(&F, alloc, &o, 0);
        po[i].flux_aper = o.flux_aper;
        po[i].fluxerr_aper = o.fluxerr_aper;
        po[i].mag_aper = o.mag_aper;
        po[i].magerr_aper = o.magerr_aper;
        po[i].kron = o.kron;
        po[i].flux_auto = o.flux_auto;
        po[i].fluxerr_auto = o.fluxerr_auto;
        po[i].mag_auto = o.mag_auto;
        po[i].magerr_auto = o.magerr_auto;
        po[i].flags = o.flags;
    }
    free(alloc);
    return 0;
}

/* Corrected isophotal flux (isocorflux above) from an object's isophotal
 * flux, its variance sum, fdnpix and detection threshold. */
void orc_isocor(float flux, float fluxerr, int fdnpix, float dthresh, float *flux_isocor, float *fluxerr_isocor)
{
    obj_t o;
    memset(&o, 0, sizeof(o));
    o.flux = flux;
    o.fluxerr = fluxerr;
    o.fdnpix = fdnpix;
    o.dthr = dthresh;
    isocorflux(&o);
    *flux_isocor = o.flux_isocor;
    *fluxerr_isocor = o.fluxerr_isocor;
}

/* The star/galaxy network's response to nn[0] inputs (nnw_response above). */
double orc_nnw_response(const orc_nnw *net, const double *input)
{
    double in[ORC_NNW_NEURONS];
    int i;
    for (i = 0; i < net->nn[0] && i < ORC_NNW_NEURONS; i++)
        in[i] = input[i];
    return nnw_response(net, in);
}

/* CLEAN (run_clean above) over objects given by their measurements, in
 * object-index order; on return master[i] is -1 for a survivor, else the
 * survivor it was merged into, and the survivors carry the merged
 * attributes. */
int orc_clean_objects(orc_clean_obj *co, int n, int w, int h, double clean_param)
{
    frame_t F;
    orc_config cfg;
    obj_t *o = (obj_t *)calloc(n + 1, sizeof(obj_t));
    int i;
    if (!o)
        return -1;
    memset(&F, 0, sizeof(F));
    memset(&cfg, 0, sizeof(cfg));
    cfg.clean_param = clean_param;
    F.w = w;
    F.h = h;
    F.cfg = &cfg;
    for (i = 0; i < n; i++) {
        o[i].mx = co[i].mx;
        o[i].my = co[i].my;
        o[i].a = co[i].a;
        o[i].b = co[i].b;
        o[i].cxx = co[i].cxx;
        o[i].cyy = co[i].cyy;
        o[i].cxy = co[i].cxy;
        o[i].abcor = co[i].abcor;
        o[i].dthr = co[i].dthresh;
        o[i].mthresh = co[i].mthresh;
        o[i].fdnpix = co[i].fdnpix;
        o[i].dnpix = co[i].dnpix;
        o[i].fdflux = co[i].fdflux;
        o[i].dflux = co[i].dflux;
        o[i].flux = co[i].flux;
        o[i].fluxerr = co[i].fluxerr;
        o[i].fdpeak = co[i].fdpeak;
        o[i].dpeak = co[i].dpeak;
        o[i].peak = co[i].peak;
        o[i].peakx = co[i].peakx;
        o[i].peaky = co[i].peaky;
        o[i].xmin = co[i].xmin;
        o[i].xmax = co[i].xmax;
        o[i].ymin = co[i].ymin;
        o[i].ymax = co[i].ymax;
        o[i].flags = co[i].flags;
    }
    run_clean(&F, o, n);
    for (i = 0; i < n; i++) {
        co[i].master = o[i].final_master;
        co[i].fdnpix = o[i].fdnpix;
        co[i].dnpix = o[i].dnpix;
        co[i].fdflux = o[i].fdflux;
        co[i].dflux = o[i].dflux;
        co[i].flux = o[i].flux;
        co[i].fluxerr = o[i].fluxerr;
        co[i].fdpeak = o[i].fdpeak;
        co[i].dpeak = o[i].dpeak;
        co[i].peak = o[i].peak;
        co[i].peakx = o[i].peakx;
        co[i].peaky = o[i].peaky;
        co[i].xmin = o[i].xmin;
        co[i].xmax = o[i].xmax;
        co[i].ymin = o[i].ymin;
        co[i].ymax = o[i].ymax;
        co[i].flags = o[i].flags;
    }
    free(o);
    return 0;
}
