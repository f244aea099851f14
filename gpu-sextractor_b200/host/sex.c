/*
 * sex.c -- command-line front end of libsexgpu with the reference's usage:
 *
 *     sex image.fits [-c file.sex] [-KEYWORD value ...]
 *
 * Reference: src/main.c:40 (argument loop :65-121), src/prefs.c:66 (readprefs,
 * `KEY value` lines, '#' comments), src/makeit.c:58 (per-image flow), and the
 * catalogue row of src/scan.c:331-406 (printobj).  The extraction itself is
 * the C ABI call sexgpu_extract_fits() (include/sexgpu.h), which replaces
 * read_body() + makeback() + scanimage(): the image's data block goes to the
 * device as stored and is converted there.
 *
 * Supported keywords (the extraction settings of src/preflist.h):
 *   CATALOG_NAME CATALOG_TYPE (ASCII, ASCII_HEAD, FITS_LDAC) PARAMETERS_NAME
 *   DETECT_MINAREA DETECT_THRESH ANALYSIS_THRESH THRESH_TYPE FILTER FILTER_NAME
 *   DEBLEND_NTHRESH DEBLEND_MINCONT CLEAN CLEAN_PARAM MASK_TYPE
 *   PHOT_APERTURES PHOT_AUTOPARAMS SATUR_LEVEL MAG_ZEROPOINT GAIN
 *   BACK_SIZE BACK_FILTERSIZE BACK_FILTTHRESH BACK_TYPE BACK_VALUE
 *   CHECKIMAGE_TYPE (NONE, SEGMENTATION, BACKGROUND, BACKGROUND_RMS, -BACKGROUND, FILTERED; a list,
 *   one CHECKIMAGE_NAME per type) CHECKIMAGE_NAME VERBOSE_TYPE
 *   WEIGHT_TYPE (NONE, MAP_VAR, MAP_RMS, MAP_WEIGHT, BACKGROUND) WEIGHT_IMAGE
 *   STARNNW_NAME SEEING_FWHM PIXEL_SCALE (CLASS_STAR)
 *   BACKPHOTO_TYPE (GLOBAL, LOCAL) BACKPHOTO_THICK
 * Multi-extension files: every image extension is a frame of one batched
 * extraction; catalogue rows carry EXT_NUMBER.
 * Other keywords of the reference are accepted and ignored.
 */
#include <ctype.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <time.h>

#include "sexgpu.h"

#define MAXLINE 4096

typedef struct {
    char catalog_name[1024], catalog_type[64], parameters_name[1024], filter_name[1024];
    char check_type[64], check_name[1024], verbose[32], weight_image[1024], nnw_name[1024];
    int nnw_given;
    sexgpu_config cfg;
    float mask[1024];
} prefs_t;

static void die(const char *msg, const char *arg)
{
    fprintf(stderr, "sex: %s%s\n", msg, arg ? arg : "");
    exit(EXIT_FAILURE);
}

static char *trim(char *s)
{
    char *e;
    while (*s && isspace((unsigned char)*s)) s++;
    e = s + strlen(s);
    while (e > s && isspace((unsigned char)e[-1])) *--e = 0;
    return s;
}

static int yes(const char *v) { return v[0] == 'Y' || v[0] == 'y' || v[0] == 'T' || v[0] == 't' || v[0] == '1'; }

/* one KEY value pair (src/prefs.c:66-305 semantics for the keys we use) */
static void setpref(prefs_t *p, const char *key, char *val)
{
    sexgpu_config *c = &p->cfg;
    char *comma;
    if ((comma = strchr(val, '#'))) *comma = 0;
    val = trim(val);
    if (!strcasecmp(key, "CATALOG_NAME")) snprintf(p->catalog_name, sizeof p->catalog_name, "%s", val);
    else if (!strcasecmp(key, "CATALOG_TYPE")) snprintf(p->catalog_type, sizeof p->catalog_type, "%s", val);
    else if (!strcasecmp(key, "PARAMETERS_NAME")) snprintf(p->parameters_name, sizeof p->parameters_name, "%s", val);
    else if (!strcasecmp(key, "FILTER_NAME")) snprintf(p->filter_name, sizeof p->filter_name, "%s", val);
    else if (!strcasecmp(key, "CHECKIMAGE_TYPE")) snprintf(p->check_type, sizeof p->check_type, "%s", val);
    else if (!strcasecmp(key, "CHECKIMAGE_NAME")) snprintf(p->check_name, sizeof p->check_name, "%s", val);
    else if (!strcasecmp(key, "VERBOSE_TYPE")) snprintf(p->verbose, sizeof p->verbose, "%s", val);
    else if (!strcasecmp(key, "DETECT_MINAREA")) c->detect_minarea = atoi(val);
    else if (!strcasecmp(key, "DETECT_THRESH")) c->detect_thresh = atof(val);
    else if (!strcasecmp(key, "ANALYSIS_THRESH")) c->analysis_thresh = atof(val);
    else if (!strcasecmp(key, "THRESH_TYPE")) c->thresh_type = !strncasecmp(val, "ABSOLUTE", 8);
    else if (!strcasecmp(key, "FILTER")) c->filter_flag = yes(val);
    else if (!strcasecmp(key, "DEBLEND_NTHRESH")) c->deblend_nthresh = atoi(val);
    else if (!strcasecmp(key, "DEBLEND_MINCONT")) c->deblend_mincont = atof(val);
    else if (!strcasecmp(key, "CLEAN")) c->clean_flag = yes(val);
    else if (!strcasecmp(key, "CLEAN_PARAM")) c->clean_param = atof(val);
    else if (!strcasecmp(key, "MASK_TYPE"))
        c->mask_type = !strncasecmp(val, "NONE", 4) ? 0 : !strncasecmp(val, "BLANK", 5) ? 1 : 2;
    else if (!strcasecmp(key, "PHOT_APERTURES")) {
        /* one diameter, or a list: the FLUX_APER columns become vectors */
        char *tok, *save = NULL;
        c->naper = 0;
        for (tok = strtok_r(val, ", \t", &save); tok && c->naper < SEXGPU_MAXAPER; tok = strtok_r(NULL, ", \t", &save))
            c->phot_apertures[c->naper++] = atof(tok);
        if (c->naper > 0) c->phot_aperture = c->phot_apertures[0];
        if (c->naper == 1) c->naper = 0;
    }
    else if (!strcasecmp(key, "PHOT_AUTOPARAMS")) {
        c->phot_autoparams[0] = atof(val);
        if ((comma = strchr(val, ','))) c->phot_autoparams[1] = atof(comma + 1);
    } else if (!strcasecmp(key, "SATUR_LEVEL")) c->satur_level = atof(val);
    else if (!strcasecmp(key, "MAG_ZEROPOINT")) c->mag_zeropoint = atof(val);
    else if (!strcasecmp(key, "GAIN")) c->gain = atof(val);
    else if (!strcasecmp(key, "BACK_SIZE")) c->back_size = atoi(val);
    else if (!strcasecmp(key, "BACK_FILTERSIZE")) c->back_filtersize = atoi(val);
    else if (!strcasecmp(key, "BACK_FILTTHRESH")) c->back_filtthresh = atof(val);
    else if (!strcasecmp(key, "BACK_TYPE")) c->back_type = !strncasecmp(val, "MANUAL", 6);
    else if (!strcasecmp(key, "BACK_VALUE")) c->back_value = atof(val);
    else if (!strcasecmp(key, "WEIGHT_TYPE"))
        c->weight_type = !strncasecmp(val, "MAP_VAR", 7)      ? 1
                         : !strncasecmp(val, "MAP_RMS", 7)    ? 2
                         : !strncasecmp(val, "MAP_WEIGHT", 10) ? 3
                         : !strncasecmp(val, "BACKGROUND", 10) ? 4
                                                               : 0;
    else if (!strcasecmp(key, "WEIGHT_IMAGE")) snprintf(p->weight_image, sizeof p->weight_image, "%s", val);
    else if (!strcasecmp(key, "SEEING_FWHM")) c->seeing_fwhm = atof(val);
    else if (!strcasecmp(key, "PIXEL_SCALE")) c->pixel_scale = atof(val);
    else if (!strcasecmp(key, "BACKPHOTO_TYPE")) c->back_photo_type = !strncasecmp(val, "LOCAL", 5);
    else if (!strcasecmp(key, "BACKPHOTO_THICK")) c->back_photo_thick = atoi(val);
    else if (!strcasecmp(key, "STARNNW_NAME")) {
        snprintf(p->nnw_name, sizeof p->nnw_name, "%s", val);
        p->nnw_given = 1;
    }
}

static void readprefs(prefs_t *p, const char *path)
{
    char line[MAXLINE], *key, *val;
    FILE *f = fopen(path, "r");
    if (!f) die("cannot open configuration file ", path);
    while (fgets(line, sizeof line, f)) {
        key = trim(line);
        if (!*key || *key == '#') continue;
        val = key;
        while (*val && !isspace((unsigned char)*val)) val++;
        if (*val) *val++ = 0;
        setpref(p, key, val);
    }
    fclose(f);
}

/* ---------------------------------------------------------------- FITS --- */
static double card_num(const char *hdr, int ncards, const char *key, double def, int *found)
{
    char k[9];
    int i;
    snprintf(k, sizeof k, "%-8s", key);
    for (i = 0; i < ncards; i++)
        if (!strncmp(hdr + 80 * i, k, 8) && hdr[80 * i + 8] == '=') {
            if (found) *found = 1;
            return atof(hdr + 80 * i + 10);
        }
    if (found) *found = 0;
    return def;
}

/* primary image of a FITS file as float (src/fits/fitsbody.c:195 read_body:
 * BITPIX 8/16/32/-32/-64, BSCALE/BZERO) */
/* the FITS data block of the primary HDU as stored, and its format */
static unsigned char *read_fits_raw(const char *path, int *w, int *h, sexgpu_fits_format *fmt)
{
    FILE *f = fopen(path, "rb");
    char *hdr = NULL;
    int ncards = 0, end = 0, naxis, i, found;
    size_t bytes;
    unsigned char *raw;
    if (!f) die("cannot open image ", path);
    while (!end) {
        hdr = (char *)realloc(hdr, (size_t)(ncards + 36) * 80);
        if (fread(hdr + (size_t)ncards * 80, 80, 36, f) != 36) die("truncated FITS header in ", path);
        for (i = 0; i < 36; i++)
            if (!strncmp(hdr + (size_t)(ncards + i) * 80, "END     ", 8)) end = 1;
        ncards += 36;
    }
    fmt->bitpix = (int)card_num(hdr, ncards, "BITPIX", 0, &found);
    naxis = (int)card_num(hdr, ncards, "NAXIS", 0, &found);
    *w = (int)card_num(hdr, ncards, "NAXIS1", 0, &found);
    *h = (int)card_num(hdr, ncards, "NAXIS2", 0, &found);
    fmt->bscale = card_num(hdr, ncards, "BSCALE", 1.0, &found);
    fmt->bzero = card_num(hdr, ncards, "BZERO", 0.0, &found);
    fmt->blank = (int64_t)card_num(hdr, ncards, "BLANK", 0.0, &found);
    fmt->has_blank = found && fmt->bitpix > 0;
    free(hdr);
    if (naxis < 2 || *w <= 0 || *h <= 0) die("not a 2-D image: ", path);
    if (fmt->bitpix != 8 && fmt->bitpix != 16 && fmt->bitpix != 32 && fmt->bitpix != -32 && fmt->bitpix != -64)
        die("unsupported BITPIX in ", path);
    bytes = (size_t)*w * *h * (size_t)(abs(fmt->bitpix) / 8);
    raw = (unsigned char *)malloc(bytes);
    if (fread(raw, 1, bytes, f) != bytes) die("truncated FITS data in ", path);
    fclose(f);
    return raw;
}

/* Every image HDU of a file (primary or XTENSION = 'IMAGE', NAXIS >= 2; the
 * first plane of a cube), as stored: a multi-extension file gives one frame
 * per CCD, as makeit() walks the extensions (src/makeit.c:164-228). */
typedef struct {
    int w, h;
    sexgpu_fits_format fmt;
    unsigned char *raw;
} fits_image;

static int card_has(const char *hdr, int ncards, const char *key, const char *text)
{
    char k[9];
    snprintf(k, sizeof k, "%-8s", key);
    for (int i = 0; i < ncards; i++)
        if (!strncmp(hdr + (size_t)i * 80, k, 8)) {
            char c[81];
            memcpy(c, hdr + (size_t)i * 80, 80);
            c[80] = 0;
            return strstr(c + 8, text) != NULL;
        }
    return 0;
}

static int read_fits_images(const char *path, fits_image **out)
{
    FILE *f = fopen(path, "rb");
    int nim = 0, cap = 0;
    *out = NULL;
    if (!f) die("cannot open image ", path);
    for (int hdu = 0;; hdu++) {
        char *hdr = NULL;
        int ncards = 0, end = 0, found, i;
        while (!end) {
            hdr = (char *)realloc(hdr, (size_t)(ncards + 36) * 80);
            if (fread(hdr + (size_t)ncards * 80, 80, 36, f) != 36) {
                free(hdr);
                if (hdu == 0) die("truncated FITS header in ", path);
                fclose(f);
                return nim;
            }
            for (i = 0; i < 36; i++)
                if (!strncmp(hdr + (size_t)(ncards + i) * 80, "END     ", 8)) end = 1;
            ncards += 36;
        }
        const int bitpix = (int)card_num(hdr, ncards, "BITPIX", 0, &found);
        const int naxis = (int)card_num(hdr, ncards, "NAXIS", 0, &found);
        size_t npix = naxis > 0 ? 1 : 0;
        int dims[8] = {0};
        for (i = 0; i < naxis && i < 8; i++) {
            char key[16];
            snprintf(key, sizeof key, "NAXIS%d", i + 1);
            dims[i] = (int)card_num(hdr, ncards, key, 0, &found);
            npix *= (size_t)(dims[i] > 0 ? dims[i] : 0);
        }
        const long pcount = (long)card_num(hdr, ncards, "PCOUNT", 0, &found);
        const long gcount = (long)card_num(hdr, ncards, "GCOUNT", 1, &found);
        const size_t bytes = (size_t)(abs(bitpix) / 8) * (size_t)gcount * (npix + (size_t)pcount);
        const int image = (hdu == 0 || card_has(hdr, ncards, "XTENSION", "IMAGE")) && naxis >= 2 && dims[0] > 0 &&
                          dims[1] > 0;
        if (image) {
            fits_image im;
            im.w = dims[0];
            im.h = dims[1];
            im.fmt.bitpix = bitpix;
            im.fmt.bscale = card_num(hdr, ncards, "BSCALE", 1.0, &found);
            im.fmt.bzero = card_num(hdr, ncards, "BZERO", 0.0, &found);
            im.fmt.blank = (int64_t)card_num(hdr, ncards, "BLANK", 0.0, &found);
            im.fmt.has_blank = found && bitpix > 0;
            if (bitpix != 8 && bitpix != 16 && bitpix != 32 && bitpix != -32 && bitpix != -64)
                die("unsupported BITPIX in ", path);
            const size_t plane = (size_t)im.w * im.h * (size_t)(abs(bitpix) / 8);
            im.raw = (unsigned char *)malloc(plane);
            if (fread(im.raw, 1, plane, f) != plane) die("truncated FITS data in ", path);
            if (bytes > plane) fseek(f, (long)(bytes - plane), SEEK_CUR);
            if (nim == cap) *out = (fits_image *)realloc(*out, sizeof(fits_image) * (size_t)(cap = cap ? 2 * cap : 4));
            (*out)[nim++] = im;
        } else if (bytes)
            fseek(f, (long)bytes, SEEK_CUR);
        if (bytes % 2880) fseek(f, (long)(2880 - bytes % 2880), SEEK_CUR);
        free(hdr);
    }
}

/* the float frame of a data block, converted as src/fits/fitsbody.c:195
 * (read_body) converts it, the same arithmetic sexgpu_extract_fits does on
 * the device */
static float *fits_to_float(const unsigned char *raw, const sexgpu_fits_format *fmt, size_t n)
{
    const float bs = (float)fmt->bscale, bz = (float)fmt->bzero;
    const int bp = fmt->bitpix, bpp = abs(bp) / 8;
    float *img = (float *)malloc(n * sizeof(float));
    for (size_t k = 0; k < n; k++) {
        const unsigned char *q = raw + k * (size_t)bpp;
        float v;
        if (bp == 8) {
            v = (fmt->has_blank && q[0] == (unsigned char)fmt->blank) ? -1e30f : q[0] * bs + bz;
        } else if (bp == 16) {
            const short s = (short)((q[0] << 8) | q[1]);
            v = (fmt->has_blank && s == (short)fmt->blank) ? -1e30f : s * bs + bz;
        } else if (bp == 32) {
            const int s = (int)(((uint32_t)q[0] << 24) | ((uint32_t)q[1] << 16) | ((uint32_t)q[2] << 8) | q[3]);
            v = (fmt->has_blank && s == (int)fmt->blank) ? -1e30f : s * bs + bz;
        } else if (bp == -32) {
            const uint32_t u = ((uint32_t)q[0] << 24) | ((uint32_t)q[1] << 16) | ((uint32_t)q[2] << 8) | q[3];
            float fv;
            memcpy(&fv, &u, 4);
            v = (u & 0x7f800000u) == 0x7f800000u ? -1e30f : fv * bs + bz;
        } else {
            uint64_t u = 0;
            double dv;
            for (int b = 0; b < 8; b++) u = (u << 8) | q[b];
            memcpy(&dv, &u, 8);
            v = ((u >> 32) & 0x7ff00000u) == 0x7ff00000u ? -1e30f : (float)(dv * bs + bz);
        }
        img[k] = v;
    }
    return img;
}

static float *read_fits(const char *path, int *w, int *h)
{
    sexgpu_fits_format fmt;
    unsigned char *raw = read_fits_raw(path, w, h, &fmt);
    float *img = fits_to_float(raw, &fmt, (size_t)*w * *h);
    free(raw);
    return img;
}

static void write_card(FILE *f, const char *card)
{
    char buf[81];
    memset(buf, ' ', 80);
    buf[80] = 0;
    memcpy(buf, card, strlen(card) < 80 ? strlen(card) : 80);
    fwrite(buf, 1, 80, f);
}

/* check image: BITPIX 32 (segmentation) or -32 (maps) */
static void write_fits(const char *path, const void *data, int w, int h, int bitpix)
{
    FILE *f = fopen(path, "wb");
    char card[81];
    size_t n = (size_t)w * h, k;
    int ncard = 0;
    if (!f) die("cannot write ", path);
    write_card(f, "SIMPLE  =                    T"); ncard++;
    snprintf(card, sizeof card, "BITPIX  = %20d", bitpix); write_card(f, card); ncard++;
    write_card(f, "NAXIS   =                    2"); ncard++;
    snprintf(card, sizeof card, "NAXIS1  = %20d", w); write_card(f, card); ncard++;
    snprintf(card, sizeof card, "NAXIS2  = %20d", h); write_card(f, card); ncard++;
    write_card(f, "END"); ncard++;
    for (; ncard % 36; ncard++) write_card(f, "");
    for (k = 0; k < n; k++) {
        uint32_t u;
        unsigned char b[4];
        memcpy(&u, (const char *)data + 4 * k, 4);
        b[0] = u >> 24; b[1] = u >> 16; b[2] = u >> 8; b[3] = u;
        fwrite(b, 1, 4, f);
    }
    for (k = (n * 4) % 2880; k && k < 2880; k++) fputc(0, f);
    fclose(f);
}

/* ------------------------------------------------------------ catalogue --- */
typedef struct {
    const char *name, *fmt, *unit, *comment;
} col_t;

static const col_t COLS[] = {
    {"NUMBER", "%10d", "", "Running object number"},
    {"X_IMAGE", "%11.4f", "pixel", "Object position along x"},
    {"Y_IMAGE", "%11.4f", "pixel", "Object position along y"},
    {"XMIN_IMAGE", "%10d", "pixel", "Minimum x-coordinate among detected pixels"},
    {"YMIN_IMAGE", "%10d", "pixel", "Minimum y-coordinate among detected pixels"},
    {"XMAX_IMAGE", "%10d", "pixel", "Maximum x-coordinate among detected pixels"},
    {"YMAX_IMAGE", "%10d", "pixel", "Maximum y-coordinate among detected pixels"},
    {"ISOAREA_IMAGE", "%9d", "pixel**2", "Isophotal area above Analysis threshold"},
    {"FLUX_ISO", "%12.7g", "count", "Isophotal flux"},
    {"FLUXERR_ISO", "%12.7g", "count", "RMS error for isophotal flux"},
    {"MAG_ISO", "%8.4f", "mag", "Isophotal magnitude"},
    {"MAGERR_ISO", "%8.4f", "mag", "RMS error for isophotal magnitude"},
    {"FLUX_ISOCOR", "%12.7g", "count", "Corrected isophotal flux"},
    {"FLUXERR_ISOCOR", "%12.7g", "count", "RMS error for corrected isophotal flux"},
    {"FLUX_APER", "%12.7g", "count", "Flux vector within fixed circular aperture(s)"},
    {"FLUXERR_APER", "%12.7g", "count", "RMS error vector for aperture flux(es)"},
    {"MAG_APER", "%8.4f", "mag", "Fixed aperture magnitude vector"},
    {"MAGERR_APER", "%8.4f", "mag", "RMS error vector for fixed aperture mag."},
    {"FLUX_AUTO", "%12.7g", "count", "Flux within a Kron-like elliptical aperture"},
    {"FLUXERR_AUTO", "%12.7g", "count", "RMS error for AUTO flux"},
    {"MAG_AUTO", "%8.4f", "mag", "Kron-like elliptical aperture magnitude"},
    {"MAGERR_AUTO", "%8.4f", "mag", "RMS error for AUTO magnitude"},
    {"KRON_RADIUS", "%5.2f", "", "Kron apertures in units of A or B"},
    {"BACKGROUND", "%12.7g", "count", "Background at centroid position"},
    {"THRESHOLD", "%12.7g", "count", "Detection threshold above background"},
    {"FLUX_MAX", "%12.7g", "count", "Peak flux above background"},
    {"X2_IMAGE", "%15.10e", "pixel**2", "Variance along x"},
    {"Y2_IMAGE", "%15.10e", "pixel**2", "Variance along y"},
    {"XY_IMAGE", "%15.10e", "pixel**2", "Covariance between x and y"},
    {"ERRX2_IMAGE", "%15.10e", "pixel**2", "Variance of position along x"},
    {"ERRY2_IMAGE", "%15.10e", "pixel**2", "Variance of position along y"},
    {"ERRXY_IMAGE", "%15.10e", "pixel**2", "Covariance of position between x and y"},
    {"CXX_IMAGE", "%12.7g", "pixel**(-2)", "Cxx object ellipse parameter"},
    {"CYY_IMAGE", "%12.7g", "pixel**(-2)", "Cyy object ellipse parameter"},
    {"CXY_IMAGE", "%12.7g", "pixel**(-2)", "Cxy object ellipse parameter"},
    {"A_IMAGE", "%9.3f", "pixel", "Profile RMS along major axis"},
    {"B_IMAGE", "%9.3f", "pixel", "Profile RMS along minor axis"},
    {"THETA_IMAGE", "%5.1f", "deg", "Position angle (CCW/x)"},
    {"ELONGATION", "%8.3f", "", "A_IMAGE/B_IMAGE"},
    {"ELLIPTICITY", "%8.3f", "", "1 - B_IMAGE/A_IMAGE"},
    {"FWHM_IMAGE", "%8.2f", "pixel", "FWHM assuming a gaussian core"},
    {"FLAGS", "%3d", "", "Extraction flags"},
    {"XPEAK_IMAGE", "%10d", "pixel", "x-coordinate of the brightest pixel"},
    {"YPEAK_IMAGE", "%10d", "pixel", "y-coordinate of the brightest pixel"},
    {"CLASS_STAR", "%6.3f", "", "S/G classifier output"},
    {"EXT_NUMBER", "%3d", "", "FITS extension number"},
    {NULL, NULL, NULL, NULL}};

static int g_ext = 1;  /* extension of the rows being written (EXT_NUMBER) */
/* every aperture of the rows being written (rows x g_naper x 4: flux, error,
   mag, mag error), when PHOT_APERTURES has several diameters */
static const float *g_aper;
static int g_naper = 1;

/* values a column holds per row: the aperture columns are vectors */
static int col_width(int c) { return (c >= 14 && c <= 17 && g_aper) ? g_naper : 1; }

static void print_col(FILE *f, int c, const sexgpu_object *o, int row)
{
    const char *fmt = COLS[c].fmt;
    if (col_width(c) > 1) {
        for (int k = 0; k < g_naper; k++) {
            if (k) fputc(' ', f);
            fprintf(f, fmt, g_aper[((size_t)row * g_naper + k) * 4 + (c - 14)]);
        }
        return;
    }
    switch (c) {
    case 0: fprintf(f, fmt, o->number); break;
    case 1: fprintf(f, fmt, o->mx + 1.0); break;
    case 2: fprintf(f, fmt, o->my + 1.0); break;
    case 3: fprintf(f, fmt, o->xmin + 1); break;
    case 4: fprintf(f, fmt, o->ymin + 1); break;
    case 5: fprintf(f, fmt, o->xmax + 1); break;
    case 6: fprintf(f, fmt, o->ymax + 1); break;
    case 7: fprintf(f, fmt, o->npix); break;
    case 8: fprintf(f, fmt, o->flux_iso); break;
    case 9: fprintf(f, fmt, o->fluxerr_iso); break;
    case 10: fprintf(f, fmt, o->mag_iso); break;
    case 11: fprintf(f, fmt, o->magerr_iso); break;
    case 12: fprintf(f, fmt, o->flux_isocor); break;
    case 13: fprintf(f, fmt, o->fluxerr_isocor); break;
    case 14: fprintf(f, fmt, o->flux_aper); break;
    case 15: fprintf(f, fmt, o->fluxerr_aper); break;
    case 16: fprintf(f, fmt, o->mag_aper); break;
    case 17: fprintf(f, fmt, o->magerr_aper); break;
    case 18: fprintf(f, fmt, o->flux_auto); break;
    case 19: fprintf(f, fmt, o->fluxerr_auto); break;
    case 20: fprintf(f, fmt, o->mag_auto); break;
    case 21: fprintf(f, fmt, o->magerr_auto); break;
    case 22: fprintf(f, fmt, o->kronfactor); break;
    case 23: fprintf(f, fmt, o->bkg); break;
    case 24: fprintf(f, fmt, o->thresh); break;
    case 25: fprintf(f, fmt, o->peak); break;
    case 26: fprintf(f, fmt, o->mx2); break;
    case 27: fprintf(f, fmt, o->my2); break;
    case 28: fprintf(f, fmt, o->mxy); break;
    case 29: fprintf(f, fmt, o->poserr_mx2); break;
    case 30: fprintf(f, fmt, o->poserr_my2); break;
    case 31: fprintf(f, fmt, o->poserr_mxy); break;
    case 32: fprintf(f, fmt, o->cxx); break;
    case 33: fprintf(f, fmt, o->cyy); break;
    case 34: fprintf(f, fmt, o->cxy); break;
    case 35: fprintf(f, fmt, o->a); break;
    case 36: fprintf(f, fmt, o->b); break;
    case 37: fprintf(f, fmt, o->theta); break;
    case 38: fprintf(f, fmt, o->elong); break;
    case 39: fprintf(f, fmt, o->ellip); break;
    case 40: fprintf(f, fmt, o->fwhm); break;
    case 41: fprintf(f, fmt, o->flags); break;
    case 42: fprintf(f, fmt, o->peakx); break;
    case 43: fprintf(f, fmt, o->peaky); break;
    case 44: fprintf(f, fmt, o->class_star); break;
    case 45: fprintf(f, fmt, g_ext); break;
    }
}

/* the 31 columns of src/scan.c:331-406 (printobj); world coordinates and
 * CLASS_STAR are written as 0, as the reference does for ALPHA/DELTA */
static void printobj(FILE *f, const sexgpu_object *o)
{
    fprintf(f, "%10d %11.7f %+11.7f %10.3f %10.3f %12.7g %12.7g %8.4f %8.4f %12.7g %12.7g %12.7g %12.7g "
               "%8.4f %8.4f %12.7g %12.7g %8.4f %8.4f %5.1f %15.10e %15.10e %15.10e %3d %8.3f %8.3f %5.2f "
               "%12.7g %5.2f %12.7g %8.2f\n",
            o->number, 0.0, 0.0, (float)(o->mx + 1.0), (float)(o->my + 1.0), o->flux_iso, o->fluxerr_iso,
            o->mag_iso, o->magerr_iso, o->flux_isocor, o->fluxerr_isocor, o->flux_aper, o->fluxerr_aper,
            o->mag_aper, o->magerr_aper, o->flux_auto, o->fluxerr_auto, o->mag_auto, o->magerr_auto, o->theta,
            o->poserr_mx2, o->poserr_my2, o->poserr_mxy, o->flags, o->elong, o->ellip, o->class_star, o->peak,
            o->kronfactor, o->bkg, o->fwhm);
}

/* ------------------------------------------------------------ FITS_LDAC --- */
/* binary type of a column: J int32, D double (second moments), E float */
static char col_type(int c)
{
    const char *fmt = COLS[c].fmt;
    return fmt[strlen(fmt) - 1] == 'd' ? 'J' : !strcmp(fmt, "%15.10e") ? 'D' : 'E';
}

static double col_value(int c, const sexgpu_object *o)
{
    switch (c) {
    case 0: return o->number;
    case 1: return o->mx + 1.0;
    case 2: return o->my + 1.0;
    case 3: return o->xmin + 1;
    case 4: return o->ymin + 1;
    case 5: return o->xmax + 1;
    case 6: return o->ymax + 1;
    case 7: return o->npix;
    case 8: return o->flux_iso;
    case 9: return o->fluxerr_iso;
    case 10: return o->mag_iso;
    case 11: return o->magerr_iso;
    case 12: return o->flux_isocor;
    case 13: return o->fluxerr_isocor;
    case 14: return o->flux_aper;
    case 15: return o->fluxerr_aper;
    case 16: return o->mag_aper;
    case 17: return o->magerr_aper;
    case 18: return o->flux_auto;
    case 19: return o->fluxerr_auto;
    case 20: return o->mag_auto;
    case 21: return o->magerr_auto;
    case 22: return o->kronfactor;
    case 23: return o->bkg;
    case 24: return o->thresh;
    case 25: return o->peak;
    case 26: return o->mx2;
    case 27: return o->my2;
    case 28: return o->mxy;
    case 29: return o->poserr_mx2;
    case 30: return o->poserr_my2;
    case 31: return o->poserr_mxy;
    case 32: return o->cxx;
    case 33: return o->cyy;
    case 34: return o->cxy;
    case 35: return o->a;
    case 36: return o->b;
    case 37: return o->theta;
    case 38: return o->elong;
    case 39: return o->ellip;
    case 40: return o->fwhm;
    case 41: return o->flags;
    case 42: return o->peakx;
    case 43: return o->peaky;
    case 44: return o->class_star;
    case 45: return g_ext;
    }
    return 0.0;
}

static void put_be(FILE *f, const void *v, int n)
{
    const unsigned char *b = (const unsigned char *)v;
    for (int i = n - 1; i >= 0; i--) fputc(b[i], f);
}

static void pad_block(FILE *f, long n, int fill)
{
    for (long k = n % 2880; k && k < 2880; k++) fputc(fill, f);
}

static void card_str(FILE *f, const char *key, const char *val)
{
    char card[81];
    snprintf(card, sizeof card, "%-8s= '%-8s'", key, val);
    write_card(f, card);
}

static void card_int(FILE *f, const char *key, long v)
{
    char card[81];
    snprintf(card, sizeof card, "%-8s= %20ld", key, v);
    write_card(f, card);
}

/* FITS_LDAC catalogue (the layout of SExtractor's LDAC output): an empty
 * primary HDU, LDAC_IMHEAD (the image header as one character cell) and
 * LDAC_OBJECTS (one row per object, the .param columns, big-endian) */
static FILE *ldac_open(const char *path)
{
    FILE *f = fopen(path, "wb");
    int ncard;
    if (!f) die("cannot write ", path);
    write_card(f, "SIMPLE  =                    T");
    write_card(f, "BITPIX  =                    8");
    write_card(f, "NAXIS   =                    0");
    write_card(f, "EXTEND  =                    T");
    write_card(f, "END");
    for (ncard = 5; ncard % 36; ncard++) write_card(f, "");
    return f;
}

/* one image's LDAC_IMHEAD and LDAC_OBJECTS tables (one pair per extension) */
static void ldac_write_ext(FILE *f, const sexgpu_object *objs, int n, const int *sel, int ns, int w, int h)
{
    char card[81], hdr[6 * 80 + 1], form[32];
    int k, ncard = 0, rowbytes = 0, nhdr = 6;
    /* LDAC_IMHEAD */
    memset(hdr, ' ', sizeof hdr - 1);
    hdr[sizeof hdr - 1] = 0;
    snprintf(card, sizeof card, "%-8s= %20s", "SIMPLE", "T"); memcpy(hdr, card, strlen(card));
    snprintf(card, sizeof card, "%-8s= %20d", "BITPIX", -32); memcpy(hdr + 80, card, strlen(card));
    snprintf(card, sizeof card, "%-8s= %20d", "NAXIS", 2); memcpy(hdr + 160, card, strlen(card));
    snprintf(card, sizeof card, "%-8s= %20d", "NAXIS1", w); memcpy(hdr + 240, card, strlen(card));
    snprintf(card, sizeof card, "%-8s= %20d", "NAXIS2", h); memcpy(hdr + 320, card, strlen(card));
    memcpy(hdr + 400, "END", 3);
    ncard = 0;
    card_str(f, "XTENSION", "BINTABLE"); ncard++;
    card_int(f, "BITPIX", 8); ncard++;
    card_int(f, "NAXIS", 2); ncard++;
    card_int(f, "NAXIS1", 80 * nhdr); ncard++;
    card_int(f, "NAXIS2", 1); ncard++;
    card_int(f, "PCOUNT", 0); ncard++;
    card_int(f, "GCOUNT", 1); ncard++;
    card_int(f, "TFIELDS", 1); ncard++;
    card_str(f, "TTYPE1", "Field Header Card"); ncard++;
    snprintf(form, sizeof form, "%dA", 80 * nhdr);
    card_str(f, "TFORM1", form); ncard++;
    snprintf(form, sizeof form, "(80, %d)", nhdr);
    card_str(f, "TDIM1", form); ncard++;
    card_str(f, "EXTNAME", "LDAC_IMHEAD"); ncard++;
    write_card(f, "END"); ncard++;
    for (; ncard % 36; ncard++) write_card(f, "");
    fwrite(hdr, 1, 80 * nhdr, f);
    pad_block(f, 80 * nhdr, 0);
    /* LDAC_OBJECTS */
    for (k = 0; k < ns; k++) rowbytes += (col_type(sel[k]) == 'D' ? 8 : 4) * col_width(sel[k]);
    ncard = 0;
    card_str(f, "XTENSION", "BINTABLE"); ncard++;
    card_int(f, "BITPIX", 8); ncard++;
    card_int(f, "NAXIS", 2); ncard++;
    card_int(f, "NAXIS1", rowbytes); ncard++;
    card_int(f, "NAXIS2", n); ncard++;
    card_int(f, "PCOUNT", 0); ncard++;
    card_int(f, "GCOUNT", 1); ncard++;
    card_int(f, "TFIELDS", ns); ncard++;
    for (k = 0; k < ns; k++) {
        char key[16];
        snprintf(key, sizeof key, "TTYPE%d", k + 1);
        card_str(f, key, COLS[sel[k]].name); ncard++;
        snprintf(key, sizeof key, "TFORM%d", k + 1);
        snprintf(form, sizeof form, "%d%c", col_width(sel[k]), col_type(sel[k]));
        card_str(f, key, form); ncard++;
        if (*COLS[sel[k]].unit) {
            snprintf(key, sizeof key, "TUNIT%d", k + 1);
            card_str(f, key, COLS[sel[k]].unit); ncard++;
        }
    }
    card_str(f, "EXTNAME", "LDAC_OBJECTS"); ncard++;
    write_card(f, "END"); ncard++;
    for (; ncard % 36; ncard++) write_card(f, "");
    for (int i = 0; i < n; i++)
        for (k = 0; k < ns; k++) {
            double v = col_value(sel[k], &objs[i]);
            char t = col_type(sel[k]);
            if (col_width(sel[k]) > 1) {
                for (int a = 0; a < g_naper; a++) {
                    float fv = g_aper[((size_t)i * g_naper + a) * 4 + (sel[k] - 14)];
                    put_be(f, &fv, 4);
                }
                continue;
            }
            if (t == 'J') {
                int32_t iv = (int32_t)v;
                put_be(f, &iv, 4);
            } else if (t == 'D') {
                put_be(f, &v, 8);
            } else {
                float fv = (float)v;
                put_be(f, &fv, 4);
            }
        }
    pad_block(f, (long)rowbytes * n, 0);
}

static int read_params(const char *path, int *sel, int maxsel)
{
    char line[MAXLINE];
    int n = 0;
    FILE *f = fopen(path, "r");
    if (!f) return 0;
    while (fgets(line, sizeof line, f) && n < maxsel) {
        char *s = trim(line), *par;
        if (!*s || *s == '#') continue;
        if ((par = strchr(s, '('))) *par = 0;
        for (int c = 0; COLS[c].name; c++)
            if (!strcasecmp(COLS[c].name, s)) {
                sel[n++] = c;
                break;
            }
    }
    fclose(f);
    return n;
}

/* ASCII / ASCII_HEAD rows of one image (the .param columns, or the
 * reference's default row when there is no .param file) */
static void write_ascii(FILE *cat, const prefs_t *p, const sexgpu_object *objs, int n, int head)
{
    int sel[64], ns = read_params(p->parameters_name, sel, 64), i, k;
    if (ns == 0) {
        for (i = 0; i < n; i++) printobj(cat, &objs[i]);
        return;
    }
    if (head && !strcasecmp(p->catalog_type, "ASCII_HEAD"))
        for (k = 0, i = 1; k < ns; i += col_width(sel[k]), k++)
            fprintf(cat, "#%4d %-22s %-58s [%s]\n", i, COLS[sel[k]].name, COLS[sel[k]].comment, COLS[sel[k]].unit);
    for (i = 0; i < n; i++) {
        for (k = 0; k < ns; k++) {
            if (k) fputc(' ', cat);
            print_col(cat, sel[k], &objs[i], i);
        }
        fputc('\n', cat);
    }
}

/* A multi-extension file: every extension is a frame of one batched
 * extraction (sexgpu_extract_batch: frames of uneven sizes on concurrent
 * streams); NUMBER restarts in every extension and EXT_NUMBER tells them
 * apart; FITS_LDAC gets one table pair per extension. */
static int run_mef(const prefs_t *p, sexgpu_ctx *ctx, fits_image *ims, int nim)
{
    sexgpu_batch_frame *fr = (sexgpu_batch_frame *)calloc((size_t)nim, sizeof(sexgpu_batch_frame));
    int k, rc, tot = 0;
    if (strcasecmp(p->check_type, "NONE") || p->cfg.weight_type || p->cfg.naper > 1)
        die("check images, weight maps and several PHOT_APERTURES need a single-image FITS file", NULL);
    for (k = 0; k < nim; k++) {
        const size_t npix = (size_t)ims[k].w * ims[k].h;
        const int cap = (int)(npix / (size_t)(p->cfg.detect_minarea > 0 ? p->cfg.detect_minarea : 1) / 2 + 16);
        fr[k].img = fits_to_float(ims[k].raw, &ims[k].fmt, npix);
        fr[k].w = ims[k].w;
        fr[k].h = ims[k].h;
        fr[k].cfg = &p->cfg;
        fr[k].objs = (sexgpu_object *)malloc(sizeof(sexgpu_object) * (size_t)cap);
        fr[k].max_objects = cap;
    }
    rc = sexgpu_extract_batch(ctx, fr, nim, 4);
    if (rc != SEXGPU_OK) {
        fprintf(stderr, "sex: extraction failed (%d): %s\n", rc, sexgpu_last_error(ctx));
        exit(EXIT_FAILURE);
    }
    if (strcasecmp(p->catalog_type, "NONE")) {
        if (!strcasecmp(p->catalog_type, "FITS_LDAC")) {
            int sel[64], ns = read_params(p->parameters_name, sel, 64);
            FILE *f = ldac_open(p->catalog_name);
            if (ns == 0)
                for (ns = 0; COLS[ns].name; ns++) sel[ns] = ns;
            for (k = 0; k < nim; k++) {
                g_ext = k + 1;
                ldac_write_ext(f, fr[k].objs, fr[k].nobj, sel, ns, fr[k].w, fr[k].h);
            }
            fclose(f);
        } else {
            FILE *cat = !strcmp(p->catalog_name, "STDOUT") ? stdout : fopen(p->catalog_name, "w");
            if (!cat) die("cannot write ", p->catalog_name);
            for (k = 0; k < nim; k++) {
                g_ext = k + 1;
                write_ascii(cat, p, fr[k].objs, fr[k].nobj, k == 0);
            }
            if (cat != stdout) fclose(cat);
        }
    }
    for (k = 0; k < nim; k++) {
        tot += fr[k].nobj;
        free((void *)fr[k].img);
        free(fr[k].objs);
    }
    free(fr);
    return tot;
}

int main(int argc, char **argv)
{
    prefs_t p;
    const char *image = NULL, *conf = "default.sex";
    int i, w, h, n = 0, rc, mw, mh, nim;
    fits_image *ims;
    float *img = NULL, *wmap = NULL;
    unsigned char *raw;
    sexgpu_fits_format fmt;
    sexgpu_object *objs;
    int32_t *seg = NULL;
    float *sub = NULL, *cd = NULL;
    sexgpu_summary s;
    sexgpu_ctx *ctx;
    clock_t t0 = clock();

    memset(&p, 0, sizeof p);
    sexgpu_default_config(&p.cfg);
    strcpy(p.catalog_name, "test.cat");
    strcpy(p.catalog_type, "ASCII_HEAD");
    strcpy(p.parameters_name, "default.param");
    strcpy(p.filter_name, "default.conv");
    strcpy(p.nnw_name, "default.nnw");
    strcpy(p.check_type, "NONE");
    strcpy(p.check_name, "check.fits");
    /* src/main.c:65-121: configuration file first, then -KEY value overrides */
    for (i = 1; i < argc; i++)
        if (!strcmp(argv[i], "-c") && i + 1 < argc) conf = argv[++i];
        else if (argv[i][0] == '-' && i + 1 < argc) i++;
        else if (!image) image = argv[i];
    if (!image) {
        fprintf(stderr, "usage: sex image.fits [-c file.sex] [-KEYWORD value ...]\n");
        return EXIT_FAILURE;
    }
    {
        FILE *f = fopen(conf, "r");
        if (f) {
            fclose(f);
            readprefs(&p, conf);
        } else if (strcmp(conf, "default.sex"))
            die("cannot open configuration file ", conf);
    }
    for (i = 1; i < argc; i++)
        if (!strcmp(argv[i], "-c")) i++;
        else if (argv[i][0] == '-' && i + 1 < argc) {
            char val[MAXLINE];
            snprintf(val, sizeof val, "%s", argv[i + 1]);
            setpref(&p, argv[i] + 1, val);
            i++;
        }
    if (p.cfg.filter_flag) {
        if (sexgpu_getconv(p.filter_name, p.mask, 1024, &mw, &mh) < 0) die("cannot read filter ", p.filter_name);
        p.cfg.conv = p.mask;
        p.cfg.conv_w = mw;
        p.cfg.conv_h = mh;
    }
    nim = read_fits_images(image, &ims);
    if (nim == 0) die("no image in ", image);
    raw = ims[0].raw;
    fmt = ims[0].fmt;
    w = ims[0].w;
    h = ims[0].h;
    if (p.cfg.weight_type >= 1 && p.cfg.weight_type <= 3 && nim == 1) {
        int ww, wh;
        if (!*p.weight_image) die("WEIGHT_IMAGE missing", NULL);
        wmap = read_fits(p.weight_image, &ww, &wh);
        if (ww != w || wh != h) die("measured frame and weight map have different sizes: ", p.weight_image);
        /* read_fits marks NaN as -1e30; for a weight map that is unusable */
        for (size_t k = 0; k < (size_t)w * h; k++)
            if (wmap[k] <= -1e30f) wmap[k] = p.cfg.weight_type == 3 ? 0.0f : 1e30f;
    }
    if ((rc = sexgpu_create(&ctx, 0)) != SEXGPU_OK) die("no usable CUDA device", NULL);
    {
        /* CLASS_STAR: the network of STARNNW_NAME (default.nnw when present) */
        sexgpu_nnw net;
        if (sexgpu_read_nnw(p.nnw_name, &net) == SEXGPU_OK)
            sexgpu_set_nnw(ctx, &net);
        else if (p.nnw_given)
            die("cannot read the star/galaxy network ", p.nnw_name);
    }
    if (nim > 1) {
        n = run_mef(&p, ctx, ims, nim);
        if (strcasecmp(p.verbose, "QUIET"))
            fprintf(stderr, "Extensions: %d / sextracted %d\n> All done (in %.2f s)\n", nim, n,
                    (double)(clock() - t0) / CLOCKS_PER_SEC);
        sexgpu_destroy(ctx);
        for (i = 0; i < nim; i++) free(ims[i].raw);
        free(ims);
        return EXIT_SUCCESS;
    }
    objs = (sexgpu_object *)malloc(sizeof(sexgpu_object) * 1024);
    if (strcasecmp(p.check_type, "NONE")) {
        seg = (int32_t *)malloc(sizeof(int32_t) * (size_t)w * h);
        sub = (float *)malloc(sizeof(float) * (size_t)w * h);
        cd = (float *)malloc(sizeof(float) * (size_t)w * h);
    }
    /* the data block goes to the device as stored and is converted there */
    rc = sexgpu_extract_fits(ctx, raw, &fmt, wmap, w, h, &p.cfg, objs, 1024, &n, seg, sub, cd, &s);
    if (rc == SEXGPU_ERR_CAPACITY) {
        objs = (sexgpu_object *)realloc(objs, sizeof(sexgpu_object) * (size_t)(n + 1));
        rc = sexgpu_copy_results(ctx, objs, n, &n, NULL, NULL, NULL);
    }
    if (rc != SEXGPU_OK) {
        fprintf(stderr, "sex: extraction failed (%d): %s\n", rc, sexgpu_last_error(ctx));
        return EXIT_FAILURE;
    }
    if (p.cfg.naper > 1) {
        /* the aperture vectors of the rows (src/photom.c:36, one call per
           diameter in the reference's own CPU code) */
        float *ap = (float *)malloc(sizeof(float) * 4 * (size_t)(n + 1) * p.cfg.naper);
        if (!ap || sexgpu_copy_apertures(ctx, ap, n, NULL, &g_naper) != SEXGPU_OK)
            die("apertures: ", sexgpu_last_error(ctx));
        g_aper = ap;
    }
    if (strcasecmp(p.catalog_type, "NONE")) {
        FILE *cat = !strcmp(p.catalog_name, "STDOUT") ? stdout : fopen(p.catalog_name, "w");
        if (!cat) die("cannot write ", p.catalog_name);
        if (!strcasecmp(p.catalog_type, "ASCII_HEAD") || !strcasecmp(p.catalog_type, "ASCII")) {
            write_ascii(cat, &p, objs, n, 1);
        } else if (!strcasecmp(p.catalog_type, "FITS_LDAC")) {
            int sel[64], ns = read_params(p.parameters_name, sel, 64);
            FILE *f;
            if (cat != stdout) fclose(cat);
            cat = stdout;
            if (ns == 0)
                for (ns = 0; COLS[ns].name; ns++) sel[ns] = ns;
            f = ldac_open(p.catalog_name);
            ldac_write_ext(f, objs, n, sel, ns, w, h);
            fclose(f);
        } else
            for (i = 0; i < n; i++) printobj(cat, &objs[i]);
        if (cat != stdout) fclose(cat);
    }
    if (seg) {
        /* CHECKIMAGE_TYPE and CHECKIMAGE_NAME are lists, paired in order
           (src/prefs.c: one check image per type) */
        char types[sizeof p.check_type], names[sizeof p.check_name], *ts = NULL, *ns = NULL, *t, *nm;
        float *map = NULL;
        snprintf(types, sizeof types, "%s", p.check_type);
        snprintf(names, sizeof names, "%s", p.check_name);
        for (t = strtok_r(types, ", \t", &ts), nm = strtok_r(names, ", \t", &ns); t;
             t = strtok_r(NULL, ", \t", &ts), nm = strtok_r(NULL, ", \t", &ns)) {
            if (!nm) die("CHECKIMAGE_NAME has fewer names than CHECKIMAGE_TYPE has types", NULL);
            if (!strcasecmp(t, "SEGMENTATION")) write_fits(nm, seg, w, h, 32);
            else if (!strcasecmp(t, "-BACKGROUND")) write_fits(nm, sub, w, h, -32);
            else if (!strcasecmp(t, "FILTERED")) write_fits(nm, cd, w, h, -32);
            else if (!strcasecmp(t, "BACKGROUND_RMS") || !strcasecmp(t, "BACKGROUND")) {
                /* src/check.c:221 (the rms map) and src/readimage.c:114 (the
                   background subtracted from every pixel), made on the device */
                int r;
                if (!map && !(map = (float *)malloc(sizeof(float) * (size_t)w * h))) die("out of memory", NULL);
                r = !strcasecmp(t, "BACKGROUND") ? sexgpu_background_map(ctx, map) : sexgpu_background_rms(ctx, map);
                if (r != SEXGPU_OK) die("background map: ", sexgpu_last_error(ctx));
                write_fits(nm, map, w, h, -32);
            } else if (strcasecmp(t, "NONE"))
                die("unsupported CHECKIMAGE_TYPE ", t);
        }
        free(map);
    }
    if (strcasecmp(p.verbose, "QUIET"))
        fprintf(stderr, "Background: %g RMS: %g / Threshold: %g\nObjects: detected %d / sextracted %d\n"
                        "> All done (in %.2f s)\n",
                s.backmean, s.backsig, s.dthresh, s.ndetected, n, (double)(clock() - t0) / CLOCKS_PER_SEC);
    sexgpu_destroy(ctx);
    free(img);
    free(raw);
    free(ims);
    free(wmap);
    free(objs);
    free(seg);
    free(sub);
    free(cd);
    return EXIT_SUCCESS;
}
