/*
 * orc_back.c -- oracle: background estimation and subtraction.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Every function below restates one
 * function of the reference's src/back.c operation for operation, with the same
 * C types, so that it compiles (gcc -ffp-contract=off, x86-64 SSE) to the same
 * IEEE results as the reference's own code.  tests/test_oracle_ref.py checks
 * that claim against the reference sources compiled into oracle/_ref.
 *
 * The mesh loop that the reference deleted from makeback() (the body is
 * commented out at src/back.c:47-88) is restated from the reference's GPU
 * driver src/cuda/cudaback.cu:1212-1375: every mesh is computed from the whole
 * frame (no line subsampling), partial meshes at the right/bottom edges use
 * their actual size.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "orc_internal.h"

typedef struct {
    float mean, sigma;
    int   nlevels;
    float qzero, qscale, lcut, hcut;
    int   npix;
} mesh_t;

/* src/misc.c:30-70 (hmedian, heapsort median; reorders ra). */
float orc_hmedian(float *ra, int n)
{
    int l, j, ir, i;
    float rra;
    if (n < 2)
        return *ra;
    ra--;
    for (l = ((ir = n) >> 1) + 1;;) {
        if (l > 1)
            rra = ra[--l];
        else {
            rra = ra[ir];
            ra[ir] = ra[1];
            if (--ir == 1) {
                ra[1] = rra;
                return n & 1 ? ra[n / 2 + 1] : (float)((ra[n / 2] + ra[n / 2 + 1]) / 2.0);
            }
        }
        for (j = (i = l) << 1; j <= ir;) {
            if (j < ir && ra[j] < ra[j + 1])
                ++j;
            if (rra < ra[j]) {
                ra[i] = ra[j];
                j += (i = j);
            } else
                j = ir + 1;
        }
        ra[i] = rra;
    }
}

/* src/back.c:214-279 (backstat) for a single mesh of bw x bh pixels at
 * (x0, y0); pixels are visited row by row, left to right. */
static void mesh_stat(const float *img, int w, int x0, int y0, int bw, int bh, mesh_t *bm)
{
    double pix, sig, mean, sigma, step;
    float lcut, hcut;
    int x, y, npix;
    const float *row;

    step = sqrt(2 / ORC_PI) * ORC_QUANTIF_NSIGMA / ORC_QUANTIF_AMIN;
    mean = sigma = 0.0;
    npix = 0;
    for (y = 0; y < bh; y++) {
        row = img + (size_t)(y0 + y) * w + x0;
        for (x = 0; x < bw; x++)
            if ((pix = row[x]) > -ORC_BIG) {
                mean += pix;
                sigma += pix * pix;
                npix++;
            }
    }
    if ((float)npix < (float)(bw * bh * ORC_BACK_MINGOODFRAC)) {
        bm->mean = bm->sigma = -ORC_BIG;
        return;
    }
    mean /= (double)npix;
    sigma = (sig = sigma / npix - mean * mean) > 0.0 ? sqrt(sig) : 0.0;
    lcut = bm->lcut = (float)(mean - 2.0 * sigma);
    hcut = bm->hcut = (float)(mean + 2.0 * sigma);
    mean = sigma = 0.0;
    npix = 0;
    for (y = 0; y < bh; y++) {
        row = img + (size_t)(y0 + y) * w + x0;
        for (x = 0; x < bw; x++) {
            pix = row[x];
            if (pix <= hcut && pix >= lcut) {
                mean += pix;
                sigma += pix * pix;
                npix++;
            }
        }
    }
    bm->npix = npix;
    mean /= (double)npix;
    sig = sigma / npix - mean * mean;
    sigma = sig > 0.0 ? sqrt(sig) : 0.0;
    bm->mean = mean;
    bm->sigma = sigma;
    if ((bm->nlevels = (int)(step * npix + 1)) > ORC_QUANTIF_NMAXLEVELS)
        bm->nlevels = ORC_QUANTIF_NMAXLEVELS;
    bm->qscale = sigma > 0.0 ? 2 * ORC_QUANTIF_NSIGMA * sigma / bm->nlevels : 1.0;
    bm->qzero = mean - ORC_QUANTIF_NSIGMA * sigma;
}

/* src/back.c:297-339 (backhisto) for one mesh. */
static void mesh_histo(const float *img, int w, int x0, int y0, int bw, int bh,
                       const mesh_t *bm, int64_t *histo)
{
    float qscale, cste;
    int x, y, bin, nlevels;
    const float *row;

    if (bm->mean <= -ORC_BIG)
        return;
    nlevels = bm->nlevels;
    qscale = bm->qscale;
    cste = 0.499999 - bm->qzero / qscale;
    for (y = 0; y < bh; y++) {
        row = img + (size_t)(y0 + y) * w + x0;
        for (x = 0; x < bw; x++) {
            bin = (int)(row[x] / qscale + cste);
            if (bin >= 0 && bin < nlevels)
                histo[bin]++;
        }
    }
}

/* The two-pointer median walk of src/back.c:370-382, restated on its own so
 * the tests can compare it with the merge-path form used on the GPU.  On
 * return lowsum/highsum hold the two running sums and the return value is the
 * index that hilow points to (hihigh is that index minus one). */
int orc_median_walk(const int64_t *histo, int lcut, int hcut,
                    int64_t *lowsum, int64_t *highsum)
{
    int64_t lo = 0, hi = 0;
    int il = lcut, ih = hcut, i;
    for (i = lcut; i <= hcut; i++) {
        if (lo < hi)
            lo += histo[il++];
        else
            hi += histo[ih--];
    }
    *lowsum = lo;
    *highsum = hi;
    return il;
}

/* The same split found by binary search on the merge path of the two
 * cumulative sums (low prefix A(a), high suffix B(b); A(a) < B(b) takes from
 * the low side, ties take from the high side). */
int orc_median_mergepath(const int64_t *histo, int lcut, int hcut,
                         int64_t *lowsum, int64_t *highsum)
{
    int n = hcut - lcut + 1, lo = 0, hi = n, a, b, k;
    int64_t *A = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    int64_t *B = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    A[0] = B[0] = 0;
    for (k = 0; k < n; k++) {
        A[k + 1] = A[k] + histo[lcut + k];
        B[k + 1] = B[k] + histo[hcut - k];
    }
    /* smallest a in [0,n] such that NOT(A(a) < B(n-1-a)) */
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (A[mid] < B[n - 1 - mid])
            lo = mid + 1;
        else
            hi = mid;
    }
    a = lo;
    b = n - a;
    *lowsum = A[a];
    *highsum = B[b];
    free(A);
    free(B);
    return lcut + a;
}

/* src/back.c:347-432 (backguess).  histo must have at least nlevels+1 entries
 * (the walk may read one bin past hcut). */
static void mesh_guess(const mesh_t *bkg, const int64_t *histo, float *mean, float *sigma)
{
    const int64_t *hilow, *hihigh, *histot;
    unsigned long lowsum, highsum, sum;
    double ftemp, mea, sig, sig1, med, dpix;
    int i, n, lcut, hcut, nlevelsm1;
    int64_t pix;

    if (bkg->mean <= -ORC_BIG) {
        *mean = *sigma = -ORC_BIG;
        return;
    }
    hcut = nlevelsm1 = bkg->nlevels - 1;
    lcut = 0;
    sig = 10.0 * nlevelsm1;
    sig1 = 1.0;
    mea = med = bkg->mean;
    for (n = 100; n-- && (sig >= 0.1) && (fabs(sig / sig1 - 1.0) > ORC_EPS);) {
        sig1 = sig;
        sum = mea = sig = 0.0;
        lowsum = highsum = 0;
        histot = hilow = histo + lcut;
        hihigh = histo + hcut;
        for (i = lcut; i <= hcut; i++) {
            if (lowsum < highsum)
                lowsum += *(hilow++);
            else
                highsum += *(hihigh--);
            sum += (pix = *(histot++));
            mea += (dpix = (double)pix * i);
            sig += dpix * i;
        }
        med = hihigh >= histo ?
              ((hihigh - histo) + 0.5 + ((double)highsum - lowsum)
               / (2.0 * (*hilow > *hihigh ? *hilow : *hihigh))) : 0.0;
        if (sum) {
            mea /= (double)sum;
            sig = sig / sum - mea * mea;
        }
        sig = sig > 0.0 ? sqrt(sig) : 0.0;
        lcut = (ftemp = med - 3.0 * sig) > 0.0 ? (int)(ftemp > 0.0 ? ftemp + 0.5 : ftemp - 0.5) : 0;
        hcut = (ftemp = med + 3.0 * sig) < nlevelsm1 ? (int)(ftemp > 0.0 ? ftemp + 0.5 : ftemp - 0.5)
               : nlevelsm1;
    }
    /* back.c:408 calls the C library abs(int) on the double sig, so the mode
     * branch is taken only when |sig| >= 1 histogram bin. */
    if (abs((int)sig) > 0.0) {
        if (fabs((mea - med) / sig) < 0.3)
            *mean = bkg->qzero + (2.5 * med - 1.5 * mea) * bkg->qscale;
        else
            *mean = bkg->qzero + med * bkg->qscale;
    } else
        *mean = bkg->qzero + mea * bkg->qscale;
    *sigma = sig * bkg->qscale;
}

/* src/back.c:434-557 (filterback) on nx*ny mesh maps, in place. */
static void filter_back(float *back, float *sigma, int nx, int ny, int nfx, int nfy,
                        float fthresh, float *backmean, float *backsig)
{
    float *bmask, *smask, *back2, *sigma2, *sigmat, d2, d2min, med, val, sval;
    int i, j, px, py, np, npx, npx2, npy, npy2, dpx, dpy, x, y, nmin;

    np = nx * ny;
    npx = nfx / 2;
    npy = nfy / 2;
    npy *= nx;
    bmask = (float *)malloc(sizeof(float) * (2 * npx + 1) * (2 * (nfy / 2) + 1));
    smask = (float *)malloc(sizeof(float) * (2 * npx + 1) * (2 * (nfy / 2) + 1));
    back2 = (float *)malloc(sizeof(float) * np);
    sigma2 = (float *)malloc(sizeof(float) * np);
    val = sval = 0.0;
    for (i = 0, py = 0; py < ny; py++)
        for (px = 0; px < nx; px++, i++)
            if ((back2[i] = back[i]) <= -ORC_BIG) {
                d2min = ORC_BIG;
                nmin = 0.0;
                for (j = 0, y = 0; y < ny; y++)
                    for (x = 0; x < nx; x++, j++)
                        if (back[j] > -ORC_BIG) {
                            d2 = (float)(x - px) * (x - px) + (y - py) * (y - py);
                            if (d2 < d2min) {
                                val = back[j];
                                sval = sigma[j];
                                nmin = 1;
                                d2min = d2;
                            } else if (d2 == d2min) {
                                val += back[j];
                                sval += sigma[j];
                                nmin++;
                            }
                        }
                back2[i] = nmin ? val / nmin : 0.0;
                sigma[i] = nmin ? sval / nmin : 1.0;
            }
    memcpy(back, back2, (size_t)np * sizeof(float));
    for (py = 0; py < np; py += nx) {
        npy2 = np - py - nx;
        if (npy2 > npy)
            npy2 = npy;
        if (npy2 > py)
            npy2 = py;
        for (px = 0; px < nx; px++) {
            npx2 = nx - px - 1;
            if (npx2 > npx)
                npx2 = npx;
            if (npx2 > px)
                npx2 = px;
            i = 0;
            for (dpy = -npy2; dpy <= npy2; dpy += nx) {
                y = py + dpy;
                for (dpx = -npx2; dpx <= npx2; dpx++) {
                    x = px + dpx;
                    bmask[i] = back[x + y];
                    smask[i++] = sigma[x + y];
                }
            }
            if (fabs((med = orc_hmedian(bmask, i)) - back[px + py]) >= fthresh) {
                back2[px + py] = med;
                sigma2[px + py] = orc_hmedian(smask, i);
            } else {
                back2[px + py] = back[px + py];
                sigma2[px + py] = sigma[px + py];
            }
        }
    }
    free(bmask);
    free(smask);
    memcpy(back, back2, np * sizeof(float));
    *backmean = orc_hmedian(back2, np);
    free(back2);
    memcpy(sigma, sigma2, np * sizeof(float));
    *backsig = orc_hmedian(sigma2, np);
    if (*backsig <= 0.0) {
        sigmat = sigma2 + np;
        for (i = np; i-- && *(--sigmat) > 0.0;)
            ;
        if (i >= 0 && i < (np - 1))
            *backsig = orc_hmedian(sigmat + 1, np - 1 - i);
        else
            *backsig = 1.0;
    }
    free(sigma2);
}

/* src/back.c:739-773 (makebackspline). */
static void back_spline(const float *map, float *dmap, int nbx, int nby)
{
    int x, y, nbym1 = nby - 1;
    float *u, temp;
    for (x = 0; x < nbx; x++) {
        if (nby > 1) {
            u = (float *)malloc(sizeof(float) * nbym1);
            dmap[x] = u[0] = 0.0;
            for (y = 1; y < nbym1; y++) {
                temp = -1 / (dmap[(size_t)(y - 1) * nbx + x] + 4);
                dmap[(size_t)y * nbx + x] = temp;
                temp *= u[y - 1] - 6 * (map[(size_t)(y + 1) * nbx + x] + map[(size_t)(y - 1) * nbx + x]
                                        - 2 * map[(size_t)y * nbx + x]);
                u[y] = temp;
            }
            dmap[(size_t)nbym1 * nbx + x] = 0.0;
            for (y = nby - 2; y >= 1; y--)
                dmap[(size_t)y * nbx + x] = (dmap[(size_t)y * nbx + x] * dmap[(size_t)(y + 1) * nbx + x] + u[y]) / 6.0;
            free(u);
        } else
            dmap[x] = 0.0;
    }
}

/* src/back.c:790-900 (subbackline) for line y. */
static void sub_back_line(const float *back, const float *dback, int nbx, int nby,
                          int backw, int backh, int back_type, float backmean,
                          int y, float *line, int width)
{
    int i, j, x, yl, nbxm1 = nbx - 1, nx, changepoint;
    float dx, dx0, dy, dy3, cdx, cdy, cdy3, temp, xstep;
    float *node, *dnode, *u;
    const float *blo, *bhi, *dblo, *dbhi, *nd, *dnd;

    if (back_type == 1) {
        for (i = 0; i < width; i++)
            line[i] -= backmean;
        return;
    }
    node = dnode = NULL;
    if (nby > 1) {
        dy = (float)y / backh - 0.5;
        dy -= (yl = (int)dy);
        if (yl < 0) {
            yl = 0;
            dy -= 1.0;
        } else if (yl >= nby - 1) {
            yl = nby < 2 ? 0 : nby - 2;
            dy += 1.0;
        }
        cdy = 1 - dy;
        dy3 = (dy * dy * dy - dy);
        cdy3 = (cdy * cdy * cdy - cdy);
        blo = back + (size_t)nbx * yl;
        bhi = blo + nbx;
        dblo = dback + (size_t)nbx * yl;
        dbhi = dblo + nbx;
        node = (float *)malloc(sizeof(float) * nbx);
        for (x = 0; x < nbx; x++)
            node[x] = cdy * blo[x] + dy * bhi[x] + cdy3 * dblo[x] + dy3 * dbhi[x];
        dnode = (float *)malloc(sizeof(float) * nbx);
        if (nbx > 1) {
            u = (float *)malloc(sizeof(float) * nbxm1);
            dnode[0] = u[0] = 0.0;
            for (x = 1; x < nbxm1; x++) {
                temp = -1 / (dnode[x - 1] + 4);
                dnode[x] = temp;
                temp *= u[x - 1] - 6 * (node[x + 1] + node[x - 1] - 2 * node[x]);
                u[x] = temp;
            }
            dnode[nbxm1] = 0.0;
            for (x = nbx - 2; x >= 1; x--)
                dnode[x] = (dnode[x] * dnode[x + 1] + u[x]) / 6.0;
            free(u);
        }
        nd = node;
        dnd = dnode;
    } else {
        nd = back;
        dnd = dback;
    }
    if (nbx > 1) {
        nx = backw;
        xstep = 1.0 / nx;
        changepoint = nx / 2;
        dx = (xstep - 1) / 2;
        dx0 = ((nx + 1) % 2) * xstep / 2;
        blo = nd;
        bhi = nd + 1;
        dblo = dnd;
        dbhi = dnd + 1;
        for (x = i = 0, j = 0; j < width; j++, i++, dx += xstep) {
            if (i == changepoint && x > 0 && x < nbxm1) {
                blo++;
                bhi++;
                dblo++;
                dbhi++;
                dx = dx0;
            }
            cdx = 1 - dx;
            line[j] -= (float)(cdx * (*blo + (cdx * cdx - 1) * *dblo) + dx * (*bhi + (dx * dx - 1) * *dbhi));
            if (i == nx) {
                x++;
                i = 0;
            }
        }
    } else
        for (j = 0; j < width; j++)
            line[j] -= *nd;
    free(node);
    free(dnode);
}

/* src/back.c:685-731 (back): bilinear background at (x, y). */
float orc_back_at(const float *b, int nx, int ny, int backw, int backh, int x, int y)
{
    int xl, yl, pos;
    double dx, dy, cdx;
    float b0, b1, b2, b3;

    dx = (double)x / backw - 0.5;
    dy = (double)y / backh - 0.5;
    dx -= (xl = (int)dx);
    dy -= (yl = (int)dy);
    if (xl < 0) {
        xl = 0;
        dx -= 1.0;
    } else if (xl >= nx - 1) {
        xl = nx < 2 ? 0 : nx - 2;
        dx += 1.0;
    }
    if (yl < 0) {
        yl = 0;
        dy -= 1.0;
    } else if (yl >= ny - 1) {
        yl = ny < 2 ? 0 : ny - 2;
        dy += 1.0;
    }
    pos = yl * nx + xl;
    cdx = 1 - dx;
    b += pos;
    b0 = *b;
    b1 = nx < 2 ? b0 : *(++b);
    b2 = ny < 2 ? *b : *(b += nx);
    b3 = nx < 2 ? *b : *(--b);
    return (float)((1 - dy) * (cdx * b0 + dx * b1) + dy * (dx * b2 + cdx * b3));
}

/* src/back.c:568-660 (localback), its statistics: the collected annulus
   pixels as one mesh of one column (backstat), their histogram and the mode
   (backguess) */
void orc_local_stats(const float *buf, int n, float *bkg, float *sig)
{
    mesh_t bm;
    int64_t *histo = (int64_t *)calloc(ORC_QUANTIF_NMAXLEVELS + 1, sizeof(int64_t));
    memset(&bm, 0, sizeof(bm));
    mesh_stat(buf, 1, 0, 0, 1, n, &bm);
    mesh_histo(buf, 1, 0, 0, 1, n, &bm, histo);
    mesh_guess(&bm, histo, bkg, sig);
    free(histo);
}

/* The background rms map (src/back.c:938 backrmsline): the filtered sigma
   mesh map through the same y and x splines as the background. */
int orc_background_rms(const float *img, int w, int h, const orc_config *cfg, float *rms)
{
    int bw = cfg->back_size < w ? cfg->back_size : w, bh = cfg->back_size < h ? cfg->back_size : h;
    int nx = (w - 1) / bw + 1, ny = (h - 1) / bh + 1, y;
    size_t p, nb = (size_t)nx * ny;
    float *copy = (float *)malloc(sizeof(float) * (size_t)w * h);
    float *sigma = (float *)malloc(sizeof(float) * nb), *dsigma = (float *)malloc(sizeof(float) * nb);
    memcpy(copy, img, sizeof(float) * (size_t)w * h);
    orc_background(copy, w, h, cfg, NULL, sigma, NULL, dsigma, NULL);
    for (y = 0; y < h; y++) {
        float *line = rms + (size_t)y * w;
        for (p = 0; p < (size_t)w; p++)
            line[p] = -0.0f;
        /* the line minus the interpolated map: -0 - v = -v for every v (zeros
           included), negated back exactly */
        sub_back_line(sigma, dsigma, nx, ny, bw, bh, 0, 0.0f, y, line, w);
        for (p = 0; p < (size_t)w; p++)
            line[p] = -line[p];
    }
    free(copy);
    free(sigma);
    free(dsigma);
    return 0;
}

/* The background map (src/back.c:790 subbackline's backline, the
   BACKGROUND check image): every line of -0 minus the interpolated map,
   negated back exactly (backmean everywhere for an absolute background). */
int orc_background_map(const float *img, int w, int h, const orc_config *cfg, float *out)
{
    int bw = cfg->back_size < w ? cfg->back_size : w, bh = cfg->back_size < h ? cfg->back_size : h;
    int nx = (w - 1) / bw + 1, ny = (h - 1) / bh + 1, y;
    size_t p, nb = (size_t)nx * ny;
    float *copy = (float *)malloc(sizeof(float) * (size_t)w * h);
    float *back = (float *)malloc(sizeof(float) * nb), *dback = (float *)malloc(sizeof(float) * nb);
    orc_summary s;
    memcpy(copy, img, sizeof(float) * (size_t)w * h);
    orc_background(copy, w, h, cfg, back, NULL, dback, NULL, &s);
    for (y = 0; y < h; y++) {
        float *line = out + (size_t)y * w;
        for (p = 0; p < (size_t)w; p++)
            line[p] = -0.0f;
        sub_back_line(back, dback, nx, ny, bw, bh, cfg->back_type, s.backmean, y, line, w);
        for (p = 0; p < (size_t)w; p++)
            line[p] = -line[p];
    }
    free(copy);
    free(back);
    free(dback);
    return 0;
}

int orc_background(float *img, int w, int h, const orc_config *cfg,
                   float *back_out, float *sigma_out, float *dback_out, float *dsigma_out,
                   orc_summary *sum)
{
    int bw, bh, nx, ny, nb, mx, my, nfx, nfy, y;
    float *back, *sigma, *dback, *dsigma, backmean = 0, backsig = 0;
    int64_t *histo;
    mesh_t bm;

    /* mesh geometry: src/field.c:124-135 */
    bw = cfg->back_size < w ? cfg->back_size : w;
    bh = cfg->back_size < h ? cfg->back_size : h;
    nx = (w - 1) / bw + 1;
    ny = (h - 1) / bh + 1;
    nb = nx * ny;
    nfx = nx > 1 ? cfg->back_filtersize : 1;
    nfy = ny > 1 ? cfg->back_filtersize : 1;

    back = (float *)malloc(sizeof(float) * nb);
    sigma = (float *)malloc(sizeof(float) * nb);
    dback = (float *)malloc(sizeof(float) * nb);
    dsigma = (float *)malloc(sizeof(float) * nb);
    histo = (int64_t *)malloc(sizeof(int64_t) * (ORC_QUANTIF_NMAXLEVELS + 1));
    for (my = 0; my < ny; my++) {
        int mh = (my == ny - 1 && h % bh) ? h % bh : bh;
        for (mx = 0; mx < nx; mx++) {
            int mw = (mx == nx - 1 && w % bw) ? w % bw : bw;
            memset(&bm, 0, sizeof(bm));
            mesh_stat(img, w, mx * bw, my * bh, mw, mh, &bm);
            memset(histo, 0, sizeof(int64_t) * (ORC_QUANTIF_NMAXLEVELS + 1));
            mesh_histo(img, w, mx * bw, my * bh, mw, mh, &bm, histo);
            mesh_guess(&bm, histo, back + my * nx + mx, sigma + my * nx + mx);
        }
    }
    free(histo);
    filter_back(back, sigma, nx, ny, nfx, nfy, (float)cfg->back_filtthresh, &backmean, &backsig);
    back_spline(back, dback, nx, ny);
    back_spline(sigma, dsigma, nx, ny);
    if (cfg->back_type == 1)
        backmean = (float)cfg->back_value;
    /* blank (NaN) pixels read as -BIG, as the FITS reader does
     * (src/fits/fitsbody.c:328); the mesh statistics above skip both alike */
    for (size_t p = 0; p < (size_t)w * h; p++)
        if (img[p] != img[p])
            img[p] = -ORC_BIGF;
    for (y = 0; y < h; y++)
        sub_back_line(back, dback, nx, ny, bw, bh, cfg->back_type, backmean, y,
                      img + (size_t)y * w, w);
    if (sum) {
        sum->nbackx = nx;
        sum->nbacky = ny;
        sum->backmean = backmean;
        sum->backsig = backsig;
        /* src/back.c:156-193 (single-entry thresholds) */
        if (cfg->thresh_type == 1) {
            sum->dthresh = (float)cfg->detect_thresh;
            sum->thresh = (float)cfg->analysis_thresh;
        } else {
            sum->dthresh = (float)(cfg->detect_thresh * backsig);
            sum->thresh = (float)(cfg->analysis_thresh * backsig);
        }
    }
    if (back_out) memcpy(back_out, back, sizeof(float) * nb);
    if (sigma_out) memcpy(sigma_out, sigma, sizeof(float) * nb);
    if (dback_out) memcpy(dback_out, dback, sizeof(float) * nb);
    if (dsigma_out) memcpy(dsigma_out, dsigma, sizeof(float) * nb);
    free(back);
    free(sigma);
    free(dback);
    free(dsigma);
    return 0;
}
