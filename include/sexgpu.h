/*
 * sexgpu.h -- C ABI of libsexgpu, the B200 (sm_100a) implementation of
 * SExtractor's per-field extraction path (background -> detection filter ->
 * thresholding/CCL -> multi-threshold deblending -> CLEAN -> isophotal
 * analysis, photometry and FLAGS -> catalogue).
 *
 * Every entry point returns an int status (SEXGPU_OK or a negative code) and
 * never exits the process.  All arguments are plain pointers and sizes.
 *
 * Reference interfaces replaced (baoxuezhao/GPU-SExtractor):
 *   sexgpu_background   <- makeback()            src/back.c:43, with
 *                          back_estimate()       src/cuda/cudaback.h:5
 *   sexgpu_filter       <- cudaFilter()          src/cuda/cudafilter.h:11
 *   sexgpu_extract      <- scanimage()           src/scan.c:65, i.e. the call
 *                          sequence init_device  src/cuda/cudainit.h:11,
 *                          run_detection         src/cuda/cudadetection.h:15,
 *                          init_deblend/parcel_out src/cuda/cudadeblend.h:11,16,
 *                          analyse_gpu           src/cuda/cudaanalyse.h:13,
 *                          run_clean             src/cuda/cudaclean.h:4,
 *                          endobject_gpu         src/cuda/cudaanalyse.h:39,
 *                          clear_device          src/cuda/cudainit.h:12
 *   sexgpu_getconv      <- getconv()             src/filter.c:101
 */
#ifndef SEXGPU_H
#define SEXGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SEXGPU_OK              0
#define SEXGPU_ERR_ARG        -1   /* bad argument (sizes, config values) */
#define SEXGPU_ERR_CUDA       -2   /* CUDA runtime error */
#define SEXGPU_ERR_NOMEM      -3   /* device allocation failed */
#define SEXGPU_ERR_RANGE      -4   /* an exact sum exceeded its dynamic range */
#define SEXGPU_ERR_CAPACITY   -5   /* caller buffer too small (count returned) */
#define SEXGPU_ERR_NODEVICE   -6   /* no usable CUDA device */
#define SEXGPU_ERR_THRESH     -7   /* zero or negative threshold (src/back.c:196) */
#define SEXGPU_ERR_LOOP       -8   /* a bounded device loop hit its iteration cap */
#define SEXGPU_ERR_NOALLOC_LIMIT -9 /* frame beyond the fixed scratch of sexgpu_background_noalloc */
#define SEXGPU_ERR_LOAD      -10   /* a tile load did not complete in time: destroy the context */
#define SEXGPU_ERR_MISMATCH  -11   /* results differed between execution parameters (a defect) */

#define SEXGPU_NISO 8
#define SEXGPU_MAXAPER 16   /* PHOT_APERTURES diameters per extraction */

/* Extraction settings; names follow the .sex keywords (src/preflist.h). */
typedef struct {
    int     back_size;          /* BACK_SIZE (square meshes) */
    int     back_filtersize;    /* BACK_FILTERSIZE (square window) */
    double  back_filtthresh;    /* BACK_FILTTHRESH */
    int     back_type;          /* BACK_TYPE: 0 AUTO, 1 MANUAL */
    double  back_value;         /* BACK_VALUE */
    int     thresh_type;        /* THRESH_TYPE: 0 RELATIVE, 1 ABSOLUTE */
    double  detect_thresh;      /* DETECT_THRESH */
    double  analysis_thresh;    /* ANALYSIS_THRESH */
    int     filter_flag;        /* FILTER */
    int     conv_w, conv_h;     /* normalised mask size (<= 31 x 31) */
    const float *conv;          /* normalised mask, row-major (host memory) */
    int     detect_minarea;     /* DETECT_MINAREA */
    int     deblend_nthresh;    /* DEBLEND_NTHRESH (1..64) */
    double  deblend_mincont;    /* DEBLEND_MINCONT */
    int     clean_flag;         /* CLEAN */
    double  clean_param;        /* CLEAN_PARAM */
    double  satur_level;        /* SATUR_LEVEL */
    double  gain;               /* GAIN */
    double  mag_zeropoint;      /* MAG_ZEROPOINT */
    double  phot_aperture;      /* PHOT_APERTURES (one diameter) */
    double  phot_autoparams[2]; /* PHOT_AUTOPARAMS */
    int     mask_type;          /* MASK_TYPE: 0 NONE, 1 BLANK, 2 CORRECT */
    int     weight_type;        /* WEIGHT_TYPE: 0 NONE, 1 MAP_VAR, 2 MAP_RMS, 3 MAP_WEIGHT,
                                   4 BACKGROUND (variance from the background rms map, no map given) */
    int     numbering;          /* 0 completion order, 1 first-pixel order */
    double  seeing_fwhm;        /* SEEING_FWHM (arcsec): CLASS_STAR input */
    double  pixel_scale;        /* PIXEL_SCALE (arcsec/pixel); <= 0 means 1 (no WCS here) */
    int     back_photo_type;    /* BACKPHOTO_TYPE: 0 GLOBAL, 1 LOCAL (annulus mode per object) */
    int     back_photo_thick;   /* BACKPHOTO_THICK: LOCAL annulus thickness, 1..256 pixels */
    /* PHOT_APERTURES with several diameters (the reference allows one,
       src/define.h:50): naper of phot_apertures[]; 0 means phot_aperture
       alone.  The catalogue row carries the first aperture; all of them are
       read with sexgpu_copy_apertures. */
    int     naper;
    double  phot_apertures[SEXGPU_MAXAPER];
} sexgpu_config;

/* One catalogue row (0-based pixel coordinates unless stated). */
typedef struct {
    int32_t number;             /* NUMBER, 1-based */
    int32_t root;               /* raw (pre-deblending) object, first-pixel order */
    int32_t level;              /* deblending level of the branch */
    int32_t fdnpix, dnpix;
    int32_t npix;               /* ISOAREA_IMAGE */
    int32_t xmin, xmax, ymin, ymax;
    int32_t peakx, peaky;       /* 1-based */
    int32_t flags;              /* FLAGS */
    int32_t iso[SEXGPU_NISO];   /* ISO0..ISO7 */
    float   fdflux, dflux, flux, fluxerr, fdpeak, dpeak, peak;
    double  mx, my, mx2, my2, mxy;
    float   a, b, theta, abcor, cxx, cyy, cxy;
    float   class_star;         /* CLASS_STAR (0 when no network is set) */
    double  poserr_mx2, poserr_my2, poserr_mxy;
    float   bkg, thresh, dthresh, mthresh, fwhm;
    float   flux_iso, fluxerr_iso, mag_iso, magerr_iso;
    float   flux_isocor, fluxerr_isocor;
    float   flux_aper, fluxerr_aper, mag_aper, magerr_aper;
    float   kronfactor, flux_auto, fluxerr_auto, mag_auto, magerr_auto;
    float   elong, ellip, polar;
} sexgpu_object;

typedef struct {
    int     nbackx, nbacky;
    float   backmean, backsig;  /* global background median and rms */
    float   dthresh, thresh;    /* detection / analysis thresholds in ADU */
    int64_t npix_above;         /* pixels with filtered value >= dthresh */
    int32_t nraw;               /* connected components >= DETECT_MINAREA */
    int64_t nraw_pix;           /* pixels in those components */
    int32_t ndetected;          /* objects after deblending */
    int32_t nobj;               /* catalogue rows after CLEAN */
    int64_t level_pix;          /* sum over raw-object pixels of the highest
                                   deblending level each pixel reaches */
    float   sigfac;             /* weight-map scale factor (1 without a map) */
    int32_t pad;
} sexgpu_summary;

typedef struct sexgpu_ctx sexgpu_ctx;

/* Context on CUDA device `device`.  Device buffers grow on demand and are
 * kept for later calls. */
int sexgpu_create(sexgpu_ctx **ctx, int device);
int sexgpu_destroy(sexgpu_ctx *ctx);
/* Run later work on this cudaStream_t (NULL: the context's own stream). */
int sexgpu_set_stream(sexgpu_ctx *ctx, void *stream);

/* Whole extraction of one host frame (w*h float32, row-major).  var (w*h)
 * is the weight map of cfg->weight_type (variance, rms or weight values) and
 * must be NULL exactly when weight_type is NONE.  With a weight map, pixels of
 * unusable weight (variance or rms >= 1e30, weight <= 0, NaN) are blank, the
 * map is calibrated to the frame's noise (MAP_VAR, MAP_WEIGHT: scale factor
 * summary.sigfac, the median over the meshes of rms / sqrt(mean relative
 * variance)), relative thresholds are taken against the local rms, each
 * object's thresholds are its pixels' smallest, and the flux errors add the
 * pixels' variances.  Writes up to
 * max_objects catalogue rows to objs (host) and their count to *nobj; if the
 * catalogue is longer, *nobj holds its length and SEXGPU_ERR_CAPACITY is
 * returned.  segmap (w*h int32 host, may be NULL) receives NUMBER per pixel,
 * 0 for sky.  sub/cd (w*h float host, may be NULL) receive the background-
 * subtracted and the filtered frame. */
int sexgpu_extract(sexgpu_ctx *ctx, const float *img, const float *var, int w, int h,
                   const sexgpu_config *cfg, sexgpu_object *objs, int max_objects,
                   int *nobj, int32_t *segmap, float *sub, float *cd, sexgpu_summary *sum);

/* FITS pixel data as stored in the file (src/fits/fitsbody.c:195 read_body) */
typedef struct {
    int32_t bitpix;             /* BITPIX: 8, 16, 32, -32, -64 */
    int32_t has_blank;          /* a BLANK keyword is present (integer BITPIX) */
    int64_t blank;              /* BLANK */
    double  bscale, bzero;      /* BSCALE, BZERO */
} sexgpu_fits_format;

/* Same as sexgpu_extract for a frame given as the FITS data block itself
 * (w*h pixels of |BITPIX|/8 big-endian bytes): the block crosses to the
 * device at its stored size and is converted there as read_body does it
 * (value * BSCALE + BZERO in float, with BSCALE and BZERO rounded to float;
 * BITPIX -64 in double, rounded once; BLANK and non-finite values become
 * -1e30, blank). */
int sexgpu_extract_fits(sexgpu_ctx *ctx, const void *data, const sexgpu_fits_format *fmt, const float *var, int w,
                        int h, const sexgpu_config *cfg, sexgpu_object *objs, int max_objects, int *nobj,
                        int32_t *segmap, float *sub, float *cd, sexgpu_summary *sum);

/* Same, for a frame already in device memory (d_img, d_var are device
 * pointers; d_img is not modified).  Results stay on the device; read them
 * with sexgpu_copy_results. */
int sexgpu_extract_device(sexgpu_ctx *ctx, const float *d_img, const float *d_var, int w, int h,
                          const sexgpu_config *cfg, sexgpu_summary *sum);

/* Copy the results of the last extraction to host memory (any pointer may
 * be NULL). */
int sexgpu_copy_results(sexgpu_ctx *ctx, sexgpu_object *objs, int max_objects, int *nobj,
                        int32_t *segmap, float *sub, float *cd);

/* The background rms map of the last extraction (src/back.c:938
 * backrmsline; the BACKGROUND_RMS check image, src/check.c:221): w*h host
 * floats, the filtered sigma mesh map through the background's splines. */
int sexgpu_background_rms(sexgpu_ctx *ctx, float *rms);

/* The background map of the last extraction (src/back.c:790 subbackline's
 * backline; the BACKGROUND check image, src/readimage.c:114): w*h host
 * floats, the value subtracted from every pixel (backmean everywhere for an
 * absolute background). */
int sexgpu_background_map(sexgpu_ctx *ctx, float *back);

/* Background only (makeback + subbackline): img (host, w*h) is replaced by
 * the background-subtracted frame; back/sigma (host, nbackx*nbacky, may be
 * NULL) receive the filtered mesh maps. */
int sexgpu_background(sexgpu_ctx *ctx, float *img, int w, int h, const sexgpu_config *cfg,
                      float *back, float *sigma, sexgpu_summary *sum);

/* Detection filter only: cd = mask (x) sub with a zero-padded frame. */
int sexgpu_filter(sexgpu_ctx *ctx, const float *sub, int w, int h, const float *mask,
                  int mw, int mh, float *cd);

/* Read and normalise a .conv file (src/filter.c:101).  Returns the number
 * of elements (mw*mh) or a negative status. */
int sexgpu_getconv(const char *path, float *mask, int maxn, int *mw, int *mh);

/* Fill cfg with the defaults of the reference's default.sex. */
void sexgpu_default_config(sexgpu_config *cfg);

/* Star/galaxy classifier (CLASS_STAR): a feed-forward network read from a
 * SExtractor .nnw file (src/neurro.c getnnw; brainstruct, src/types.h:930).
 * w[l][i][j] weighs neuron i of layer l into neuron j of layer l + 1. */
#define SEXGPU_NNW_LAYERS 3
#define SEXGPU_NNW_NEURONS 10
typedef struct {
    int32_t nlayers;                                   /* input, hidden..., output (2..3) */
    int32_t nn[SEXGPU_NNW_LAYERS];                     /* neurons per layer (<= 10) */
    double  inbias[SEXGPU_NNW_NEURONS], inscale[SEXGPU_NNW_NEURONS];
    double  outbias[SEXGPU_NNW_NEURONS], outscale[SEXGPU_NNW_NEURONS];
    double  w[SEXGPU_NNW_LAYERS - 1][SEXGPU_NNW_NEURONS][SEXGPU_NNW_NEURONS];
    double  b[SEXGPU_NNW_LAYERS - 1][SEXGPU_NNW_NEURONS];
} sexgpu_nnw;
/* Parse a .nnw file; SEXGPU_ERR_ARG if it is not one or exceeds the limits. */
int sexgpu_read_nnw(const char *path, sexgpu_nnw *net);
/* Network of this context's later extractions (and its batch workers');
 * NULL switches CLASS_STAR off (0 in every row).  With a network, CLASS_STAR
 * is computed per object from its isophotal areas, FLUX_MAX, analysis
 * threshold, SEEING_FWHM and PIXEL_SCALE (src/cuda/cudaanalyse.cu:2901-2920). */
int sexgpu_set_nnw(sexgpu_ctx *ctx, const sexgpu_nnw *net);

/* Background mesh grid of a w x h frame and BACK_SIZE back_size
 * (src/field.c:124-135): bw = min(back_size, w), bh = min(back_size, h),
 * nbackx = (w - 1) / bw + 1, nbacky = (h - 1) / bh + 1.  Host only. */
int sexgpu_background_meshes(int w, int h, int back_size, int *nbackx, int *nbacky);

/* Background estimation and subtraction that allocates no device memory.
 *
 * No counterpart in the reference.  For callers that cannot call cudaMalloc or
 * cudaFree (a pipeline living inside another framework's memory pool, a
 * process with a device-memory budget fixed at start-up, a real-time loop that
 * must not allocate or trigger the synchronisation an allocation can cause):
 * the caller owns all buffers, the library's working memory is a fixed device
 * array of about 13.2 MB that every GPU loading this library holds until the
 * process exits.
 *
 * d_img (w*h floats) is the frame and d_sub (w*h) receives the background-
 * subtracted frame; d_back and d_sigma receive the filtered mesh maps,
 * nbackx*nbacky floats each (sexgpu_background_meshes gives the counts);
 * mesh_capacity is the number of floats each of them holds, and a capacity
 * below nbackx*nbacky returns SEXGPU_ERR_ARG before anything is written.  All
 * four are device pointers.  stream is a cudaStream_t (NULL: the default
 * stream).  sum (host, may be NULL) receives the global background, its rms
 * and the thresholds, after which the call has synchronised the stream.
 * Results equal those of sexgpu_background.
 *
 * Limits: w, h <= 16384, nbackx*nbacky <= 16384, h*nbackx <= 1048576;
 * larger frames return SEXGPU_ERR_NOALLOC_LIMIT.  The first call on a device
 * looks up the array's device address (make that first call before any
 * stream capture).  All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
int sexgpu_background_noalloc(const float *d_img, float *d_sub, int w, int h, const sexgpu_config *cfg,
                              float *d_back, float *d_sigma, int mesh_capacity, sexgpu_summary *sum, void *stream);

/* One frame of a batch: inputs, the caller's catalogue buffer, and outputs. */
typedef struct {
    const float *img;            /* host frame, w*h float32, row-major */
    const float *wmap;           /* host weight map of cfg->weight_type, or NULL */
    int32_t w, h;
    const sexgpu_config *cfg;    /* this frame's settings */
    sexgpu_object *objs;         /* host catalogue buffer (may be NULL) */
    int32_t max_objects;
    int32_t nobj;                /* out: catalogue length */
    int32_t status;              /* out: SEXGPU_OK or this frame's error */
    int32_t pad;
    sexgpu_summary summary;      /* out */
} sexgpu_batch_frame;

/* Extraction of many frames of any sizes and settings (the batched form of
 * scanimage(); no counterpart in the reference, which handles one frame per
 * process).  The frames are taken largest first by `workers` device streams
 * of this context's device (0: 8, or what sexgpu_autotune_batch chose), each
 * with its own buffers (with "graph", each frame kind stays with one worker,
 * which keeps its graph), so that the
 * stages of different frames overlap on the GPU.  Every frame's results are
 * exactly those of sexgpu_extract on that frame.  Returns SEXGPU_OK if every
 * frame succeeded, else the status of the first failed frame (each frame's
 * own status is in frames[i].status).  Not for use on the same context from
 * two threads at once. */
int sexgpu_extract_batch(sexgpu_ctx *ctx, sexgpu_batch_frame *frames, int nframes, int workers);

/* Frame streaming, for pipelines that extract frame after frame: the upload
 * of the next frame overlaps the extraction of the current one.
 * sexgpu_stream_submit queues a host frame (and weight map, or NULL) and
 * starts its upload on a copy stream of the context; it returns without
 * waiting.  sexgpu_stream_next extracts the oldest queued frame with cfg and
 * returns its catalogue as sexgpu_extract does (no maps).  At most two frames
 * are queued (SEXGPU_ERR_CAPACITY beyond).  A queued frame's host memory
 * must stay unchanged until sexgpu_stream_next has returned its catalogue.
 * The uploads overlap only from page-locked host memory; pageable frames are
 * copied before sexgpu_stream_submit returns. */
int sexgpu_stream_submit(sexgpu_ctx *ctx, const float *img, const float *var, int w, int h);
int sexgpu_stream_next(sexgpu_ctx *ctx, const sexgpu_config *cfg, sexgpu_object *objs, int max_objects,
                       int *nobj, sexgpu_summary *sum);

/* One timed candidate of the autotuners. */
typedef struct {
    char    param[24];          /* execution parameter (see sexgpu_set_param) */
    int32_t value;
    float   ms;                 /* best time of the timed runs: per frame, or per batch */
} sexgpu_tune_entry;

/* Autotuner of the execution parameters, which never change results.  Times
 * the extraction of one device-resident frame (arguments as for
 * sexgpu_extract_device) on this context with "graph" 0 and 1, then, with the
 * faster, "kron_warp_max" 1024, 2048, ..., 32768: each candidate after its
 * warm-up runs (a graph learns and captures), best of reps runs timed with
 * CUDA events on the context's stream.  The fastest value of each parameter
 * stays set on the context.  Every candidate's catalogue rows are compared
 * with the first candidate's, byte for byte: SEXGPU_ERR_MISMATCH if they
 * differ.  Up to max_entries candidates go to entries (may be NULL); returns
 * the number of candidates timed, or an error code. */
int sexgpu_autotune(sexgpu_ctx *ctx, const float *d_img, const float *d_wmap, int w, int h,
                    const sexgpu_config *cfg, int reps, sexgpu_tune_entry *entries, int max_entries);

/* Autotuner of the batched form: times sexgpu_extract_batch on these frames
 * (host wall clock, best of reps, after one warm-up batch per candidate) with
 * 4, 8, 12 and 16 workers, then "batch_grid_div" 1, 2 and 4, then (with
 * "graph" set) "batch_one_launch" 0 and 1, and keeps the fastest as this
 * context's defaults (the worker count of a batch called with workers = 0).  The frames' catalogues are compared with the first
 * candidate's (SEXGPU_ERR_MISMATCH if they differ); they hold the last run's
 * results on return.  Returns the number of candidates timed, or an error. */
int sexgpu_autotune_batch(sexgpu_ctx *ctx, sexgpu_batch_frame *frames, int nframes, int reps,
                          sexgpu_tune_entry *entries, int max_entries);

/* Aperture photometry of every aperture of the last extraction (FLUX_APER,
 * FLUXERR_APER, MAG_APER, MAGERR_APER as vectors), in catalogue order: out
 * receives rows x naper x 4 floats (flux, error, magnitude, magnitude
 * error) for up to max_rows rows; *nrows and *naper (may be NULL) receive
 * the catalogue length and the number of apertures.  SEXGPU_ERR_CAPACITY
 * when the catalogue is longer than max_rows (nothing is copied). */
int sexgpu_copy_apertures(sexgpu_ctx *ctx, float *out, int max_rows, int *nrows, int *naper);

/* Last CUDA error string of this context (empty if none). */
const char *sexgpu_last_error(sexgpu_ctx *ctx);

/* Timed kernel launches of the last extraction, per stage: number of
 * launches of this library's kernels and event-timed milliseconds.  stages
 * is filled with up to max entries; returns the number of stages. */
typedef struct {
    char    name[24];
    int32_t launches;
    float   ms;
} sexgpu_stage;
int sexgpu_stage_times(sexgpu_ctx *ctx, sexgpu_stage *stages, int max);

/* Execution parameters of this context (and of its batch workers); results
 * do not depend on them.  "kron_warp_max": AUTO-photometry boxes of more
 * pixels than this are summed by whole thread blocks instead of one warp
 * (default 8192, >= 1).  "batch_grid_div": the persistent grids of
 * sexgpu_extract_batch's workers use 1/n of the resident capacity each
 * (default 1).  "batch_sync": 1 (default) makes the batch workers wait for
 * their streams on blocking events, which leaves the host cores to the other
 * workers and keeps batch times steady; 0 spins.  "loop_cap": n > 0 caps
 * every union-find walk, union retry and CLEAN chain walk of the following
 * extractions at n steps (a walk that runs out returns SEXGPU_ERR_LOOP and the
 * context stays usable); 0 (default) keeps the built-in caps, which no valid
 * frame reaches -- it exists to test the error path.  "batch_workers": the
 * worker count of a batch called with workers = 0 (1..64, default 8).
 * "batch_one_launch": with "graph", 1 runs a batch repeated after
 * one whose every frame replayed a graph (same frame sizes, settings and
 * order; new pixel values allowed) as a single launch of a batch graph: the
 * workers' chains of upload, frame graph and result copies side by side.
 * Frames in page-locked host memory are uploaded from where they are, others
 * through the batch's pinned buffer.  0 (default) keeps one graph launch per
 * frame on the worker streams, which overlaps each frame's upload with the
 * other workers' kernels.
 * "graph": 1 extracts
 * through captured CUDA graphs (default 0).  The first frame of a kind (frame
 * size, configuration, detection mask, input buffers and the parameters
 * above) runs as without the parameter and sets capacities a quarter above its
 * counts; the next one runs sized by those capacities, with every count kept
 * on the device, and is captured; each later one is a single graph launch
 * and one wait.  A frame whose counts exceed the capacities is extracted again
 * without the graph and the capacities grow.  The catalogue is the same in
 * every case; per-stage times are not kept for graph frames.  Returns
 * SEXGPU_ERR_ARG for an unknown name or value. */
int sexgpu_set_param(sexgpu_ctx *ctx, const char *name, int value);

/* How the last extraction of this context ran: *replayed 1 when it was a
 * captured graph launch, *kernels the kernel launches of that graph (0
 * otherwise), *kinds the frame kinds this context holds graphs for.  Any
 * pointer may be NULL. */
int sexgpu_graph_stats(sexgpu_ctx *ctx, int *replayed, int *kernels, int *kinds);

#ifdef __cplusplus
}
#endif
#endif
