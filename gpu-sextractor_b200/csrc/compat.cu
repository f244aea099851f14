// compat.cu -- the reference's thirteen CUDA entry points (include/sexgpu_compat.h)
// on the staged pipeline of sexgpu.cu.  Built into libsexgpu_compat.so only
// (compat_lib.cu), so that libsexgpu.so exports no generic names.
#include <cstdio>
#include <cstdlib>

#include "sexgpu_compat.h"

namespace {

struct CompatState {
    sexgpu_ctx *ctx = nullptr;
    int device = 0;
    int w = 0, h = 0;
    sexgpu_config cfg;
    bool cfg_init = false;
    std::vector<float> mask;
    int mask_w = 0;
    int nobj = 0;
    void (*handler)(const char *) = nullptr;
    bool have_nnw = false;
    sexgpu_nnw nnw;
};

CompatState &cs() {
    static CompatState s;
    if (!s.cfg_init) {
        sexgpu_default_config(&s.cfg);
        s.cfg_init = true;
    }
    return s;
}

void compat_fail(const char *what, int rc) {
    CompatState &s = cs();
    char msg[512];
    const char *detail = s.ctx ? sexgpu_last_error(s.ctx) : "";
    snprintf(msg, sizeof(msg), "%s failed (status %d%s%s)", what, rc, detail && *detail ? ": " : "",
             detail ? detail : "");
    if (s.handler) {
        s.handler(msg);
        return;
    }
    fprintf(stderr, "*Error*: %s\n", msg);
    exit(EXIT_FAILURE);
}

// false (after reporting) when the call sequence is broken
bool compat_ready(const char *what, int stage) {
    CompatState &s = cs();
    if (!s.ctx || s.ctx->ps.stage != stage) {
        compat_fail(what, SEXGPU_ERR_ARG);
        return false;
    }
    return true;
}

__global__ void k_compat_thresholds(FrameScalars *sc, float dthresh, float thresh) {
    sc->dthresh = dthresh;
    sc->thresh = thresh;
    sc->e0cd = fexpo(dthresh);
}

// one record per object, in object index order
__global__ void k_compat_rows(ObjBufs O, int n, sexgpu_outobj *rows) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= n) return;
    sexgpu_outobj q;
    memset(&q, 0, sizeof(q));
    q.number = 0;
    q.alpha2000 = 0.0;
    q.delta2000 = 0.0;
    q.sposx = (float)(O.mx[o] + 1.0);
    q.sposy = (float)(O.my[o] + 1.0);
    q.flux_iso = O.flux[o];
    q.fluxerr_iso = O.fluxerr_iso[o];
    q.mag_iso = O.mag_iso[o];
    q.magerr_iso = O.magerr_iso[o];
    q.flux_isocor = O.flux_isocor[o];
    q.fluxerr_isocor = O.fluxerr_isocor[o];
    q.flux_aper[0] = O.flux_aper[o];
    q.fluxerr_aper[0] = O.fluxerr_aper[o];
    q.mag_aper[0] = O.mag_aper[o];
    q.magerr_aper[0] = O.magerr_aper[o];
    q.flux_auto = O.flux_auto[o];
    q.fluxerr_auto = O.fluxerr_auto[o];
    q.mag_auto = O.mag_auto[o];
    q.magerr_auto = O.magerr_auto[o];
    q.theta = O.theta[o];
    q.poserr_mx2 = O.pmx2[o];
    q.poserr_my2 = O.pmy2[o];
    q.poserr_mxy = O.pmxy[o];
    q.flag = (short)O.flags[o];
    q.elong = O.a[o] / O.b[o];
    q.ellip = 1 - O.b[o] / O.a[o];
    q.sprob = O.sprob ? O.sprob[o] : 0.0f;
    q.peak = O.peak[o];
    q.kronfactor = O.kron[o];
    q.bkg = O.bkg[o];
    q.fwhm = O.fwhm[o];
    memcpy(rows + o, &q, sizeof(q));  // padding bytes too
}

}  // namespace

extern "C" {

void sexgpu_compat_configure(double mag_zeropoint, double phot_aperture, double autoparam0, double autoparam1,
                             int mask_type, double back_value) {
    CompatState &s = cs();
    s.cfg.mag_zeropoint = mag_zeropoint;
    s.cfg.phot_aperture = phot_aperture;
    s.cfg.phot_autoparams[0] = autoparam0;
    s.cfg.phot_autoparams[1] = autoparam1;
    s.cfg.mask_type = mask_type;
    s.cfg.back_value = back_value;
}

void sexgpu_compat_set_device(int device) { cs().device = device; }

void sexgpu_compat_set_nnw(const sexgpu_nnw *net, double seeing_fwhm) {
    CompatState &s = cs();
    s.have_nnw = net != nullptr;
    if (net) s.nnw = *net;
    if (seeing_fwhm > 0.0) s.cfg.seeing_fwhm = seeing_fwhm;
    if (s.ctx) {
        const int rc = sexgpu_set_nnw(s.ctx, s.have_nnw ? &s.nnw : nullptr);
        if (rc) compat_fail("sexgpu_compat_set_nnw", rc);
    }
}

void sexgpu_compat_set_error_handler(void (*handler)(const char *msg)) { cs().handler = handler; }

void init_device(int width, int height, float *img) {
    CompatState &s = cs();
    int rc;
    if (!s.ctx && (rc = sexgpu_create(&s.ctx, s.device)) != SEXGPU_OK) {
        s.ctx = nullptr;
        compat_fail("init_device", rc);
        return;
    }
    if (s.have_nnw && (rc = sexgpu_set_nnw(s.ctx, &s.nnw)) != SEXGPU_OK) {
        compat_fail("init_device (CLASS_STAR network)", rc);
        return;
    }
    if (!img || width <= 0 || height <= 0) {
        compat_fail("init_device", SEXGPU_ERR_ARG);
        return;
    }
    sexgpu_ctx *ctx = s.ctx;
    cudaSetDevice(ctx->device);
    s.w = width;
    s.h = height;
    ctx->ps.stage = 0;
    const size_t n = (size_t)width * height;
    rc = ensure(ctx, ctx->img, n * 4);
    if (rc == SEXGPU_OK && cudaMemcpyAsync(ctx->img.p, img, n * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        rc = SEXGPU_ERR_CUDA;
    if (rc) compat_fail("init_device", rc);
}

void back_estimate(int back_size, float backfthresh, float *backmean, float *backsig, int nbackfx, int nbackfy,
                   int backtype) {
    CompatState &s = cs();
    if (!s.ctx || s.w <= 0) {
        compat_fail("back_estimate", SEXGPU_ERR_ARG);
        return;
    }
    if (nbackfx != nbackfy) {
        compat_fail("back_estimate (BACK_FILTERSIZE must be square)", SEXGPU_ERR_ARG);
        return;
    }
    s.cfg.back_size = back_size;
    s.cfg.back_filtersize = nbackfx;
    s.cfg.back_filtthresh = backfthresh;
    s.cfg.back_type = backtype == 1;  // BACK_ABSOLUTE (src/types.h:37)
    s.cfg.filter_flag = 0;            // the mask comes with cudaFilter
    s.cfg.conv = nullptr;
    s.cfg.conv_w = s.cfg.conv_h = 0;
    sexgpu_ctx *ctx = s.ctx;
    int rc = pipe_begin(ctx, P<float>(ctx->img), nullptr, s.w, s.h, &s.cfg);
    if (!rc) rc = read_scalars(ctx);
    if (rc) {
        compat_fail("back_estimate", rc);
        return;
    }
    if (backmean) *backmean = ctx->hsc.backmean;
    if (backsig) *backsig = ctx->hsc.backsig;
}

void cudaFilter(float *mask, unsigned int mask_width) {
    CompatState &s = cs();
    if (!mask || mask_width == 0 || mask_width > SX_MAXCONV) {
        compat_fail("cudaFilter", SEXGPU_ERR_ARG);
        return;
    }
    s.mask.assign(mask, mask + (size_t)mask_width * mask_width);
    s.mask_w = (int)mask_width;
}

void init_detection(void) {}

void run_detection(float dthresh, float thresh, int minarea, size_t *numValidObj, size_t *numValidPix) {
    CompatState &s = cs();
    if (!compat_ready("run_detection", 1)) return;
    sexgpu_ctx *ctx = s.ctx;
    if (dthresh <= 0.0f || thresh <= 0.0f || minarea < 1) {
        compat_fail("run_detection (zero or negative threshold)", SEXGPU_ERR_THRESH);
        return;
    }
    FrameParams &Pm = ctx->ps.Pm;
    Pm.minarea = minarea;
    Pm.debminarea = minarea < SX_MAXDEBAREA ? minarea : SX_MAXDEBAREA;
    if (s.mask_w > 0) {
        Pm.filter_flag = 1;
        Pm.conv_w = Pm.conv_h = s.mask_w;
    } else {
        Pm.filter_flag = 0;
        Pm.conv_w = Pm.conv_h = 1;
    }
    int rc = load_mask(ctx, s.mask_w > 0 ? s.mask.data() : nullptr, s.mask_w, s.mask_w);
    if (rc) {
        compat_fail("run_detection", rc);
        return;
    }
    k_compat_thresholds<<<1, 1, 0, ctx->stream>>>(P<FrameScalars>(ctx->sc), dthresh, thresh);
    rc = pipe_detect(ctx);
    if (rc) {
        compat_fail("run_detection", rc);
        return;
    }
    if (numValidObj) *numValidObj = (size_t)ctx->ps.nroots;
    if (numValidPix) *numValidPix = (size_t)ctx->ps.nrootpix;
}

void clear_detection(void) {}

void init_deblend(float basethresh, int nthresh, size_t numValidObj, size_t numValidPix) {
    (void)basethresh;
    (void)numValidObj;
    (void)numValidPix;
    if (nthresh < 1 || nthresh > 64) compat_fail("init_deblend (DEBLEND_NTHRESH out of 1..64)", SEXGPU_ERR_ARG);
}

int parcel_out(float basethresh, int nthresh, int deb_minarea, size_t numValidObj, size_t numValidPix,
               double deblend_mincont) {
    CompatState &s = cs();
    (void)basethresh;
    (void)numValidObj;
    (void)numValidPix;
    if (!compat_ready("parcel_out", 2)) return 0;
    if (nthresh < 1 || nthresh > 64 || deb_minarea < 1) {
        compat_fail("parcel_out", SEXGPU_ERR_ARG);
        return 0;
    }
    sexgpu_ctx *ctx = s.ctx;
    FrameParams &Pm = ctx->ps.Pm;
    Pm.nthresh = nthresh;
    Pm.debminarea = deb_minarea;
    Pm.mincont = deblend_mincont;
    int rc = pipe_deblend(ctx);
    if (rc) {
        compat_fail("parcel_out", rc);
        return 0;
    }
    s.nobj = ctx->ps.nobj;
    return s.nobj;
}

void clear_deblend(int nthresh) { (void)nthresh; }

void analyse_gpu(double flagobj_poserr_mx2, int flagobj_peakx, int flagobj_iso_0, float flagobj_fwhm, float backsig,
                 double gain, double ngamma, float thresh, float dthresh, double satur_level, int plistexist_var,
                 int plistoff_var, int prefs_weightgain_flag, int prefs_ext_minarea, int prefs_clean_flag,
                 int detect_type, int nbackx, int nbacky, int backw, int backh, int width, int numobj) {
    CompatState &s = cs();
    (void)flagobj_poserr_mx2, (void)flagobj_peakx, (void)flagobj_iso_0, (void)flagobj_fwhm, (void)backsig;
    (void)ngamma, (void)thresh, (void)dthresh, (void)plistexist_var, (void)plistoff_var;
    (void)prefs_weightgain_flag, (void)detect_type, (void)nbackx, (void)nbacky, (void)backw, (void)backh, (void)width;
    if (!compat_ready("analyse_gpu", 3)) return;
    if (numobj != s.nobj) {
        compat_fail("analyse_gpu (object count differs from parcel_out)", SEXGPU_ERR_ARG);
        return;
    }
    FrameParams &Pm = s.ctx->ps.Pm;
    Pm.gain = gain;
    Pm.satur_level = satur_level;
    Pm.minarea = prefs_ext_minarea;
    Pm.clean_flag = prefs_clean_flag;
    int rc = pipe_analyse(s.ctx);
    if (rc) compat_fail("analyse_gpu", rc);
}

int run_clean(int *masterIndex, double clean_param, int clean_stacksize, int numobj) {
    CompatState &s = cs();
    (void)clean_stacksize;
    if (!compat_ready("run_clean", 4)) return 0;
    if (numobj != s.nobj) {
        compat_fail("run_clean (object count differs from parcel_out)", SEXGPU_ERR_ARG);
        return 0;
    }
    sexgpu_ctx *ctx = s.ctx;
    ctx->ps.Pm.clean_param = clean_param;
    int rc = pipe_clean(ctx);
    if (!rc && masterIndex && numobj > 0)
        rc = cudaMemcpyAsync(masterIndex, ctx->O.fmaster, (size_t)numobj * 4, cudaMemcpyDeviceToHost, ctx->stream) ==
                     cudaSuccess
                 ? SEXGPU_OK
                 : SEXGPU_ERR_CUDA;
    if (!rc) rc = cudaStreamSynchronize(ctx->stream) == cudaSuccess ? SEXGPU_OK : SEXGPU_ERR_CUDA;
    if (rc) {
        compat_fail("run_clean", rc);
        return 0;
    }
    int kept = 0;
    if (masterIndex)
        for (int i = 0; i < numobj; i++) kept += masterIndex[i] < 0;
    return kept;
}

void endobject_gpu(void *prefs, void *brain, void *flagobj2, sexgpu_outobj *outobj, void *wcs, int fymin, int fymax,
                   int width, int height, float backsig, float thresh, double satur, double pixscale, double ngamma,
                   double gain, int numobj) {
    CompatState &s = cs();
    (void)prefs, (void)brain, (void)flagobj2, (void)wcs, (void)fymin, (void)fymax, (void)backsig, (void)thresh;
    (void)ngamma;
    if (!compat_ready("endobject_gpu", 5)) return;
    if (numobj != s.nobj || width != s.w || height != s.h) {
        compat_fail("endobject_gpu (object count or frame size differs)", SEXGPU_ERR_ARG);
        return;
    }
    sexgpu_ctx *ctx = s.ctx;
    FrameParams &Pm = ctx->ps.Pm;
    Pm.satur_level = satur;
    Pm.gain = gain;
    Pm.mag_zeropoint = s.cfg.mag_zeropoint;
    Pm.aperture = s.cfg.phot_aperture;
    Pm.autoparam0 = s.cfg.phot_autoparams[0];
    Pm.autoparam1 = s.cfg.phot_autoparams[1];
    Pm.mask_type = s.cfg.mask_type;
    Pm.numbering = 1;
    Pm.seeing = s.cfg.seeing_fwhm;
    Pm.pixscale = pixscale > 0.0 ? pixscale : 1.0;
    int rc = pipe_end(ctx);
    if (!rc && numobj > 0) {
        rc = ensure(ctx, ctx->rows, (size_t)numobj * sizeof(sexgpu_outobj));
        if (!rc) {
            k_compat_rows<<<grid1(numobj, 128), 128, 0, ctx->stream>>>(ctx->O, numobj, P<sexgpu_outobj>(ctx->rows));
            if (outobj &&
                cudaMemcpyAsync(outobj, ctx->rows.p, (size_t)numobj * sizeof(sexgpu_outobj), cudaMemcpyDeviceToHost,
                                ctx->stream) != cudaSuccess)
                rc = SEXGPU_ERR_CUDA;
            if (!rc && cudaStreamSynchronize(ctx->stream) != cudaSuccess) rc = SEXGPU_ERR_CUDA;
        }
    }
    if (rc) compat_fail("endobject_gpu", rc);
}

void clear_device(float *img) {
    CompatState &s = cs();
    if (!s.ctx || s.ctx->ps.stage < 2 || !img) {
        compat_fail("clear_device", SEXGPU_ERR_ARG);
        return;
    }
    sexgpu_ctx *ctx = s.ctx;
    const size_t n = (size_t)s.w * s.h;
    if (cudaMemcpyAsync(img, ctx->sub.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        compat_fail("clear_device", SEXGPU_ERR_CUDA);
}

}  // extern "C"
