/* scan_like.c -- test harness: drives libsexgpu_compat.so with the call
 * sequence of the reference's host code, makeback() (src/back.c:104-110,
 * relative thresholds :171, :190) then scanimage() (src/scan.c:78-157), on a
 * raw float32 frame, and writes the records scanimage() would print, in its
 * order and with its NUMBER, plus the background-subtracted frame that
 * clear_device() returns.
 *
 * usage: scan_like frame.f32 W H mask.f32 MASKW out_rows.bin out_sub.f32
 *        BACK_SIZE BACK_FILTERSIZE BACK_FILTTHRESH DETECT_THRESH ANALYSIS_THRESH
 *        MINAREA NTHRESH MINCONT CLEAN CLEAN_PARAM GAIN SATUR [NNW SEEING_FWHM PIXSCALE]
 */
#include <stdio.h>
#include <stdlib.h>

#include "sexgpu_compat.h"

static void *slurp(const char *path, size_t bytes) {
    FILE *f = fopen(path, "rb");
    void *p = malloc(bytes);
    if (!f || !p || fread(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(2);
    }
    fclose(f);
    return p;
}

int main(int argc, char **argv) {
    if (argc != 20 && argc != 23) {
        fprintf(stderr, "usage: see the header of scan_like.c\n");
        return 2;
    }
    int w = atoi(argv[2]), h = atoi(argv[3]), mw = atoi(argv[5]);
    float *img = (float *)slurp(argv[1], (size_t)w * h * 4);
    float *mask = (float *)slurp(argv[4], (size_t)mw * mw * 4);
    int back_size = atoi(argv[8]), nbackf = atoi(argv[9]);
    double fthresh = atof(argv[10]), dthr = atof(argv[11]), athr = atof(argv[12]);
    int minarea = atoi(argv[13]), nthresh = atoi(argv[14]);
    double mincont = atof(argv[15]);
    int clean = atoi(argv[16]);
    double clean_param = atof(argv[17]), gain = atof(argv[18]), satur = atof(argv[19]);
    int deb_maxarea = minarea < 3 ? minarea : 3; /* src/prefs.c:463 */

    /* makeit(): the star/galaxy network when a .nnw file is given (argv[20]) */
    if (argc > 20) {
        sexgpu_nnw net;
        if (sexgpu_read_nnw(argv[20], &net) != SEXGPU_OK) return 3;
        sexgpu_compat_set_nnw(&net, atof(argv[21]));
    }

    /* makeback() */
    float backmean = 0.0f, backsig = 0.0f;
    init_device(w, h, img);
    back_estimate(back_size, (float)fthresh, &backmean, &backsig, nbackf, nbackf, 0);
    float dthresh = dthr * backsig, thresh = athr * backsig;

    /* scanimage() */
    size_t nobj = 0, npix = 0;
    init_detection();
    cudaFilter(mask, (unsigned)mw);
    run_detection(dthresh, thresh, minarea, &nobj, &npix);
    init_deblend(dthresh, nthresh, nobj, npix);
    int numdetected = parcel_out(dthresh, nthresh, deb_maxarea, nobj, npix, mincont);
    clear_deblend(nthresh);
    analyse_gpu(0.0, 0, 0, 0.0f, backsig, gain, 0.0, thresh, dthresh, satur, 0, 0, 0, minarea, clean, 0, 0, 0,
                back_size, back_size, w, numdetected);
    int *master = (int *)malloc((size_t)(numdetected + 1) * sizeof(int));
    run_clean(master, clean_param, 3000, numdetected);
    sexgpu_outobj *objlist = (sexgpu_outobj *)malloc((size_t)(numdetected + 1) * sizeof(sexgpu_outobj));
    endobject_gpu(NULL, NULL, NULL, objlist, NULL, 0, h, w, h, backsig, thresh, satur, argc > 22 ? atof(argv[22]) : 1.0,
                  0.0, gain, numdetected);
    clear_detection();
    clear_device(img);

    FILE *fo = fopen(argv[6], "wb"), *fs = fopen(argv[7], "wb");
    if (!fo || !fs) return 3;
    int number = 0;
    for (int i = 0; i < numdetected; i++)
        if (master[i] == -1) {
            objlist[i].number = number++;
            fwrite(&objlist[i], sizeof(sexgpu_outobj), 1, fo);
        }
    fwrite(img, 4, (size_t)w * h, fs);
    fclose(fo);
    fclose(fs);
    printf("detected %d sextracted %d raw %zu pixels %zu backmean %.9g backsig %.9g\n", numdetected, number, nobj,
           npix, backmean, backsig);
    return 0;
}
