// sexgpu.cu -- libsexgpu: context, extraction pipeline and the C ABI of
// include/sexgpu.h.  Built as one translation unit with the stage files.
//
// The pipeline is the reference's scanimage() sequence (src/scan.c:65-163):
// background (makeback), filter + threshold, connected components, deblending
// (init_deblend/parcel_out), analysis (analyse_gpu), CLEAN (run_clean),
// photometry/FLAGS (endobject_gpu), catalogue.  All stages run on one CUDA
// stream (the deblending forks two more).  In the plain form the host reads
// back the counts between stages to size the launches; in the capacity form
// the launches are sized by capacities learned from an earlier frame, the
// counts stay on the device, and the whole frame is one CUDA graph.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <atomic>
#include <string>
#include <thread>
#include <mutex>
#include <chrono>
#include <vector>

#include "sexgpu.h"
#include "common.cuh"
#include "kernels.cuh"
#include "prim.cuh"

#include "prim.cu"
#include "k_back.cu"
#include "k_detect.cu"
#include "k_roots.cu"
#include "k_deblend.cu"
#include "k_deblend_local.cu"
#include "k_analyse.cu"
#include "k_post.cu"
#include "k_fits.cu"

using namespace sx;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

struct StageRec {
    const char *name;
    int launches;
    cudaEvent_t ev;
};

}  // namespace

namespace {
struct PipeState {
    FrameParams Pm;
    int w = 0, h = 0;
    const float *d_img = nullptr;
    const float *wvar = nullptr;  // calibrated variance map (weight map given), else null
    int nroots = 0, nrootpix = 0, nobj = 0, ns = 0;
    int stage = 0;  // last completed: 1 background ... 6 catalogue
    // capacity form: launches sized by these capacities, counts read on the
    // device only (k_gate stands in for the host checks between stages)
    bool capf = false;
    int cap_roots = 0, cap_rootpix = 0, cap_obj = 0;
    // while the stages are captured: device memory already holding the
    // frame's constants (column tables, then the mask: 8 w + 4 SX_MAXCONV^2
    // bytes), so that the graph has no host-to-device copies, which would
    // queue behind a concurrent frame upload on the copy engine
    unsigned char *cst = nullptr;
    BackBufs B;
    RootBufs R;
    DebArgs A;
};
}  // namespace

namespace sx {
thread_local int sx_grid_div = 1;
}

// A captured frame: the graph of the capacity form for one frame geometry,
// configuration, detection mask and input buffers.
struct GraphEntry {
    FrameParams Pm;
    std::vector<float> mask;
    const float *d_img = nullptr, *d_wmap = nullptr;
    const sexgpu_nnw *nnw = nullptr;
    int kron_warp_max = 0, grid_div = 1;
    int cap_roots = 0, cap_rootpix = 0, cap_obj = 0;  // 0: not learned yet
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;   // the captured graph (child node of a batch graph)
    unsigned long long id = 0;     // unique within the context
    unsigned char *cst = nullptr;  // device copy of the frame's constants (PipeState::cst)
    PipeState ps;                  // host state of the captured frame, restored on replay
    ObjBufs O;
    unsigned long long gen = 0;  // allocation generation the graph's pointers belong to
    bool no_graph = false;       // capture failed: the capacity form runs uncaptured
    int kernels = 0;             // kernel nodes of the graph
    unsigned long long used = 0;
};

// One-launch form of a batch (sexgpu_extract_batch with graphs): per worker
// a chain of its frames, each the upload of the frame into the worker's
// input buffer, the frame kind's captured graph as a child graph, and copies
// of its catalogue rows and scalars into per-frame areas; the chains side by
// side in one graph, ended by one copy of every frame's scalars to the host.
struct BatchGraph {
    std::vector<unsigned long long> sig;            // per frame: kind, size, weight map, worker
    std::vector<unsigned long long> epochs, gens;   // per worker at build time
    std::vector<std::vector<int>> lists;            // per worker: its frames in order
    std::vector<size_t> in_off, row_off;            // per frame: pinned input offset, first row
    std::vector<int> cap;                           // per frame: rows the area holds
    std::vector<FrameParams> pm;                    // per frame
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;                    // kept: its upload nodes are re-pointed per launch
    std::vector<cudaGraphNode_t> up_img, up_wmap;   // per frame: upload nodes (weight map: null if none)
    std::vector<void *> dst_img, dst_wmap;          // per frame: the worker's input buffers
    unsigned char *in_host = nullptr;               // pinned frames and weight maps
    size_t in_bytes = 0;
    void *rows_dev = nullptr, *sc_dev = nullptr;
    FrameScalars *sc_host = nullptr;                // pinned
    unsigned char *rows_host = nullptr;             // pinned
    size_t rows_total = 0;
    int kernels = 0;
};

struct sexgpu_ctx {
    int device = 0;
    int batch_grid_div = 1;  // persistent-grid divisor of batch workers
    int batch_sync = 1;      // batch workers wait on blocking events (1) or spin (0)
    int sync_block = 0;      // this context waits on a blocking event instead of spinning
    cudaEvent_t ev_block = nullptr;
    PipeState ps;
    cudaStream_t stream = nullptr;
    cudaStream_t side[DL_SIDE] = {};  // fork/join helpers of the deblending
    cudaEvent_t ev_fork = nullptr, ev_join[DL_SIDE] = {};
    bool own_stream = false;
    std::vector<DevBuf *> bufs;
    std::string err;
    // frame-size buffers
    DevBuf img, sub, cd, lab, cnt, flag, pos, alloc, seg, pos2idx, var, imgm, wvar, wratio;
    // frame streaming (sexgpu_stream_*): two input slots uploaded on a copy stream
    DevBuf qimg[2], qvar[2];
    int qw[2] = {0, 0}, qh[2] = {0, 0};
    bool qhasvar[2] = {false, false};
    int qhead = 0, qcount = 0;
    cudaStream_t qstream = nullptr;
    cudaEvent_t qev[2] = {nullptr, nullptr};
    // scan / sort scratch
    DevBuf scan_tmp, keys, vals, kalt, valt;
    // background
    DevBuf ms, back, sigma, back2, back3, sigma3, dback, bu, rownode, rowdnode, rowu, colk, coldx;
    // roots
    DevBuf rsize, roff, rfirst, rymax, rlastx, rfdpeak, rfdflux, rnkept, robjbase, rdthr, rathr, rlists, rcounts;
    // deblend scratch
    DevBuf dpar, dlev, dsz, dorder, drl0, drl1, dnid0, dnid1, dacc, nr0, nr1, nf0, nf1, ns0, ns1, nc0, nc1, na0, na1,
        dkept, down, dkl, dkidx, dpint, objkey, rpix, darena, drec;
    // objects
    DevBuf o_i[20], o_f[32], o_d[10], o_iso, o_sortkey, amp, alpha, cellhead, cellnext, vkey, vval, vkalt, vvalt,
        skeys, svals, skalt, svalt, rows;
    DevBuf kitem[2], kchunk[2], kpart[2];  // queued Kron boxes
    DevBuf o_sprob;                        // CLASS_STAR per object
    DevBuf o_raw, o_xraw, o_eraw;          // robust preanalysis / examineiso / photometry scratch per object
    DevBuf o_dbkg, o_lstat;                // BACKPHOTO_TYPE LOCAL: annulus mode, annulus statistics
    DevBuf o_aper, aperrows;               // every aperture per object; per catalogue row
    bool cfg_local = false;                // the current extraction uses LOCAL photometry background
    DevBuf fitsraw;                        // FITS data block as stored (sexgpu_extract_fits)
    DevBuf rmsd, rmsnode, rmsdnode, rmsu, rmsmap;  // background rms map (sexgpu_background_rms)
    DevBuf dnnw;                           // this context's copy of the CLASS_STAR network
    const sexgpu_nnw *nnw_dev = nullptr;   // network used (this context's or, for a batch worker, its owner's)
    int kron_warp_max = KR_WARP_MAX;
    int loop_cap = 0;  // "loop_cap" parameter: cap on device walks, for failure tests (0: built-in caps)
    int graph_mode = 0;                  // "graph" parameter: extract through captured graphs
    unsigned long long gen = 0;          // bumped by every device allocation (graphs hold pointers)
    std::vector<GraphEntry> graphs;      // captured frames, least recently used evicted
    unsigned long long graph_clock = 0;
    unsigned long long graph_epoch = 0;  // bumped whenever a graph is captured or dropped
    unsigned long long last_entry = 0;   // id of the graph entry of the last extraction (0: none)
    BatchGraph *bgraph = nullptr;        // one-launch form of the last batch (sexgpu_extract_batch)
    FrameScalars *hsc_pin = nullptr;     // pinned copy of the frame scalars (capacity form)
    int last_graph = 0;                  // the last extraction replayed a graph
    int last_kernels = 0;                // kernel launches of the last extraction
    DevBuf sc;
    FrameScalars hsc;
    ObjBufs O;
    std::vector<int> colk_h;
    std::vector<float> coldx_h;
    int last_w = 0, last_h = 0, last_nobj = 0, last_ns = 0;
    std::vector<StageRec> stages;
    cudaEvent_t ev0 = nullptr;
    std::vector<float> stage_ms;
    std::vector<std::string> stage_names;
    std::vector<int> stage_launches;
    std::vector<sexgpu_ctx *> workers;  // contexts of sexgpu_extract_batch
    std::vector<unsigned long long> batch_kinds;  // frame kinds a batch worker has extracted
    int batch_workers = 8;  // workers of a batch called with workers = 0 (sexgpu_autotune_batch)
    int batch_one_launch = 0;  // with graphs, a repeated batch is one launch of a batch graph
    // buffers outgrown during a batch: freed when the batch ends, because
    // cudaFree waits for the whole device and would stall the other workers
    bool defer_free = false;
    std::vector<void *> graveyard, host_graveyard;
    void *stage_host = nullptr;         // pinned staging of a batch worker's frames
    size_t stage_bytes = 0;
    void *rows_host = nullptr;          // pinned staging of a batch worker's catalogue rows
    size_t rows_bytes = 0;
    DevBuf dmask;                       // detection mask of the current extraction
    std::vector<float> hmask;
    ConvMask cmask{nullptr, nullptr, 1, 1};
};

namespace {

int set_err(sexgpu_ctx *c, cudaError_t e, const char *what) {
    c->err = std::string(what) + ": " + cudaGetErrorString(e);
    return SEXGPU_ERR_CUDA;
}

#define CK(call)                                               \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return set_err(ctx, _e, #call); \
    } while (0)

int ensure(sexgpu_ctx *ctx, DevBuf &b, size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (b.bytes >= bytes) return SEXGPU_OK;
    if (b.p) {
        if (ctx->defer_free)
            ctx->graveyard.push_back(b.p);
        else
            cudaFree(b.p);
    }
    b.p = nullptr;
    b.bytes = 0;
    size_t want = bytes + bytes / 8;
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        ctx->err = "device allocation failed";
        return SEXGPU_ERR_NOMEM;
    }
    b.bytes = want;
    ctx->gen++;
    return SEXGPU_OK;
}

#define EN(buf, bytes)                                 \
    do {                                               \
        int _r = ensure(ctx, ctx->buf, (size_t)(bytes)); \
        if (_r) return _r;                             \
    } while (0)

template <class T> T *P(DevBuf &b) { return (T *)b.p; }

// stage timing (plain form only: a graph has no per-stage events)
void stage_begin(sexgpu_ctx *ctx) {
    ctx->stage_names.clear();
    ctx->stage_launches.clear();
    ctx->stage_ms.clear();
    if (ctx->ps.capf) return;  // (no event calls while the stages may be captured)
    for (auto &s : ctx->stages) cudaEventDestroy(s.ev);
    ctx->stages.clear();
    if (!ctx->ev0) cudaEventCreate(&ctx->ev0);
    cudaEventRecord(ctx->ev0, ctx->stream);
}

void stage_mark(sexgpu_ctx *ctx, const char *name, int launches) {
    if (ctx->ps.capf) return;
    StageRec s;
    s.name = name;
    s.launches = launches;
    cudaEventCreate(&s.ev);
    cudaEventRecord(s.ev, ctx->stream);
    ctx->stages.push_back(s);
}

void stage_collect(sexgpu_ctx *ctx) {
    ctx->stage_ms.clear();
    ctx->stage_names.clear();
    ctx->stage_launches.clear();
    cudaEvent_t prev = ctx->ev0;
    for (auto &s : ctx->stages) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, prev, s.ev);
        ctx->stage_ms.push_back(ms);
        ctx->stage_names.push_back(s.name);
        ctx->stage_launches.push_back(s.launches);
        prev = s.ev;
    }
}

// x-interpolation table of src/back.c:863-899 (segment index and dx of
// every column), the same float arithmetic as the reference's loop
void column_table(int width, int nbx, int backw, std::vector<int> &colk, std::vector<float> &coldx) {
    colk.assign(width, 0);
    coldx.assign(width, 0.f);
    if (nbx <= 1) return;
    int nx = backw, changepoint = nx / 2, x = 0, i = 0, k = 0;
    float xstep = 1.0 / nx;
    float dx = (xstep - 1) / 2;
    float dx0 = ((nx + 1) % 2) * xstep / 2;
    for (int j = 0; j < width; j++, i++, dx += xstep) {
        if (i == changepoint && x > 0 && x < nbx - 1) {
            k++;
            dx = dx0;
        }
        colk[j] = k;
        coldx[j] = dx;
        if (i == nx) {
            x++;
            i = 0;
        }
    }
}

int check_config(const sexgpu_config *cfg, int w, int h) {
    if (!cfg || w <= 0 || h <= 0) return SEXGPU_ERR_ARG;
    if ((long long)w * h >= (1ll << 31)) return SEXGPU_ERR_ARG;
    if (cfg->back_size < 1 || cfg->back_filtersize < 1 || cfg->back_filtersize > 11) return SEXGPU_ERR_ARG;
    if (cfg->filter_flag && (!cfg->conv || cfg->conv_w < 1 || cfg->conv_h < 1 || cfg->conv_w > SX_MAXCONV ||
                             cfg->conv_h > SX_MAXCONV))
        return SEXGPU_ERR_ARG;
    if (cfg->detect_minarea < 1 || cfg->deblend_nthresh < 1 || cfg->deblend_nthresh > 64) return SEXGPU_ERR_ARG;
    if (cfg->weight_type < 0 || cfg->weight_type > 4) return SEXGPU_ERR_ARG;
    if (!(cfg->seeing_fwhm > 0.0)) return SEXGPU_ERR_ARG;
    if (cfg->back_photo_type < 0 || cfg->back_photo_type > 1) return SEXGPU_ERR_ARG;
    if (cfg->back_photo_type == 1 && (cfg->back_photo_thick < 1 || cfg->back_photo_thick > 256)) return SEXGPU_ERR_ARG;
    if (cfg->naper < 0 || cfg->naper > SEXGPU_MAXAPER) return SEXGPU_ERR_ARG;
    for (int k = 0; k < cfg->naper; k++)
        if (!(cfg->phot_apertures[k] > 0.0)) return SEXGPU_ERR_ARG;
    return SEXGPU_OK;
}

void make_params(const sexgpu_config *cfg, int w, int h, FrameParams &P) {
    memset(&P, 0, sizeof(P));
    P.w = w;
    P.h = h;
    P.bw = cfg->back_size < w ? cfg->back_size : w;
    P.bh = cfg->back_size < h ? cfg->back_size : h;
    P.nbx = (w - 1) / P.bw + 1;
    P.nby = (h - 1) / P.bh + 1;
    P.nfx = P.nbx > 1 ? cfg->back_filtersize : 1;
    P.nfy = P.nby > 1 ? cfg->back_filtersize : 1;
    P.fthresh = (float)cfg->back_filtthresh;
    P.back_type = cfg->back_type;
    P.back_value = (float)cfg->back_value;
    P.thresh_type = cfg->thresh_type;
    P.detect_thresh = cfg->detect_thresh;
    P.analysis_thresh = cfg->analysis_thresh;
    P.filter_flag = cfg->filter_flag;
    P.conv_w = cfg->conv_w;
    P.conv_h = cfg->conv_h;
    P.minarea = cfg->detect_minarea;
    P.debminarea = cfg->detect_minarea < SX_MAXDEBAREA ? cfg->detect_minarea : SX_MAXDEBAREA;
    P.nthresh = cfg->deblend_nthresh;
    P.mincont = cfg->deblend_mincont;
    P.clean_flag = cfg->clean_flag;
    P.clean_param = cfg->clean_param;
    P.satur_level = cfg->satur_level;
    P.gain = cfg->gain;
    P.mag_zeropoint = cfg->mag_zeropoint;
    P.naper = cfg->naper > 0 ? cfg->naper : 1;
    for (int k = 0; k < SEXGPU_MAXAPER; k++)
        P.apertures[k] = k < cfg->naper ? cfg->phot_apertures[k] : cfg->phot_aperture;
    P.aperture = P.apertures[0];
    P.autoparam0 = cfg->phot_autoparams[0];
    P.autoparam1 = cfg->phot_autoparams[1];
    P.mask_type = cfg->mask_type;
    P.numbering = cfg->numbering;
    P.wtype = cfg->weight_type;
    P.wthr = cfg->weight_type != 0 && cfg->thresh_type != 1;
    P.seeing = cfg->seeing_fwhm;
    P.pixscale = cfg->pixel_scale > 0.0 ? cfg->pixel_scale : 1.0;
    P.bp_local = cfg->back_photo_type == 1;
    P.bp_thick = cfg->back_photo_thick;
    P.loop_cap = 0;
}

__global__ void k_init_scalars(FrameScalars *sc) {
    FrameScalars z;
    memset(&z, 0, sizeof(z));
    z.e0sub = 1000;
    z.sigfac = 1.0f;
    *sc = z;
}

// Capacity form: the checks the plain form makes on the host between stages.
// An error so far, a zero or negative threshold (check_thr) or a count beyond
// the capacity the launches were sized for sets the counts the later stages
// read to 0, and the nl deblending list lengths at lists, so that the rest of
// the frame does nothing; the status tells the host afterwards.
__global__ void k_gate(FrameScalars *sc, int check_thr, int cap_roots, int cap_rootpix, int cap_obj, int *lists,
                       int nl) {
    int st = sc->status;
    if (check_thr && (sc->dthresh <= 0.0f || sc->thresh <= 0.0f)) st |= SX_ST_THRESH;
    if (sc->nroots > cap_roots || sc->nrootpix > cap_rootpix || sc->nobj > cap_obj) st |= SX_ST_CAPACITY;
    sc->status = st;
    if (st & SX_ST_STOP) {
        sc->nroots = sc->nrootpix = sc->nobj = sc->nsurv = 0;
        for (int k = 0; k < nl; k++) lists[k] = 0;
    }
}

// Waits for the work queued on st: a spinning wait (the runtime's default
// with few host threads), or, for a batch worker told so, a blocking event
// wait that leaves the host core to the other workers.
cudaError_t stream_wait(sexgpu_ctx *ctx, cudaStream_t st) {
    if (!ctx->sync_block) return cudaStreamSynchronize(st);
    if (!ctx->ev_block) {
        cudaError_t e = cudaEventCreateWithFlags(&ctx->ev_block, cudaEventBlockingSync | cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    cudaError_t e = cudaEventRecord(ctx->ev_block, st);
    return e == cudaSuccess ? cudaEventSynchronize(ctx->ev_block) : e;
}

int read_scalars(sexgpu_ctx *ctx) {
    CK(cudaMemcpyAsync(&ctx->hsc, ctx->sc.p, sizeof(FrameScalars), cudaMemcpyDeviceToHost, ctx->stream));
    CK(stream_wait(ctx, ctx->stream));
    if (ctx->hsc.status & SX_ST_LOAD) {
        ctx->err = "a tile load did not complete in time; destroy this context";
        return SEXGPU_ERR_LOAD;
    }
    if (ctx->hsc.status & SX_ST_LOOP) {
        ctx->err = "device loop iteration cap reached";
        return SEXGPU_ERR_LOOP;
    }
    if (ctx->hsc.status & SX_ST_RANGE) {
        ctx->err = "exact sum out of range";
        return SEXGPU_ERR_RANGE;
    }
    return SEXGPU_OK;
}

// the detection mask of this context's next extraction (host and device copy)
int load_mask(sexgpu_ctx *ctx, const float *mask, int mw, int mh) {
    static const float one = 1.0f;
    if (!mask) {
        mask = &one;
        mw = mh = 1;
    }
    ctx->hmask.assign(mask, mask + (size_t)mw * mh);
    EN(dmask, sizeof(float) * SX_MAXCONV * SX_MAXCONV);
    if (ctx->ps.cst) {  // being captured: the graph's device copy
        ctx->cmask.dev = reinterpret_cast<const float *>(ctx->ps.cst + (size_t)8 * ctx->ps.w);
    } else {
        CK(cudaMemcpyAsync(ctx->dmask.p, ctx->hmask.data(), sizeof(float) * mw * mh, cudaMemcpyHostToDevice,
                           ctx->stream));
        ctx->cmask.dev = P<float>(ctx->dmask);
    }
    ctx->cmask.host = ctx->hmask.data();
    ctx->cmask.mw = mw;
    ctx->cmask.mh = mh;
    return SEXGPU_OK;
}

int alloc_objects(sexgpu_ctx *ctx, int nobj) {
    size_t n = (size_t)nobj + 1;
    int *ip[20];
    float *fp[32];
    double *dp[10];
    for (int i = 0; i < 20; i++) {
        EN(o_i[i], n * sizeof(int));
        ip[i] = P<int>(ctx->o_i[i]);
    }
    for (int i = 0; i < 32; i++) {
        EN(o_f[i], n * sizeof(float));
        fp[i] = P<float>(ctx->o_f[i]);
    }
    for (int i = 0; i < 10; i++) {
        EN(o_d[i], n * sizeof(double));
        dp[i] = P<double>(ctx->o_d[i]);
    }
    EN(o_iso, n * SX_NISO_ * sizeof(int));
    ObjBufs &O = ctx->O;
    O.root = ip[0];
    O.level = ip[1];
    O.n = ip[2];
    O.off = ip[3];
    O.xmin = ip[4];
    O.xmax = ip[5];
    O.ymin = ip[6];
    O.ymax = ip[7];
    O.dnpix = ip[8];
    O.flags = ip[9];
    O.singu = ip[10];
    O.npix = ip[11];
    O.peakx = ip[12];
    O.peaky = ip[13];
    O.master = ip[14];
    O.fmaster = ip[15];
    O.number = ip[16];
    O.fdnpix = ip[17];
    O.fdflux = fp[0];
    O.dflux = fp[1];
    O.fdpeak = fp[2];
    O.dpeak = fp[3];
    O.node_dthresh = fp[4];
    O.a = fp[5];
    O.b = fp[6];
    O.theta = fp[7];
    O.abcor = fp[8];
    O.cxx = fp[9];
    O.cyy = fp[10];
    O.cxy = fp[11];
    O.flux = fp[12];
    O.fluxerr = fp[13];
    O.peak = fp[14];
    O.bkg = fp[15];
    O.mthresh = fp[16];
    O.fwhm = fp[17];
    O.flux_isocor = fp[18];
    O.fluxerr_isocor = fp[19];
    O.flux_aper = fp[20];
    O.fluxerr_aper = fp[21];
    O.mag_aper = fp[22];
    O.magerr_aper = fp[23];
    O.kron = fp[24];
    O.flux_auto = fp[25];
    O.fluxerr_auto = fp[26];
    O.mag_auto = fp[27];
    O.magerr_auto = fp[28];
    O.mag_iso = fp[29];
    O.dthr = fp[30];
    O.athr = fp[31];
    O.mx = dp[0];
    O.my = dp[1];
    O.mx2 = dp[2];
    O.my2 = dp[3];
    O.mxy = dp[4];
    O.pmx2 = dp[5];
    O.pmy2 = dp[6];
    O.pmxy = dp[7];
    O.iso = P<int>(ctx->o_iso);
    EN(o_d[8], n * sizeof(float));   // magerr_iso
    EN(o_d[9], n * sizeof(float));   // fluxerr_iso
    O.magerr_iso = P<float>(ctx->o_d[8]);
    EN(o_sprob, n * sizeof(float));
    O.sprob = ctx->nnw_dev ? P<float>(ctx->o_sprob) : nullptr;
    EN(o_dbkg, n * sizeof(float));
    EN(o_lstat, n * sizeof(MeshStat));
    const int naper = ctx->ps.Pm.naper > 1 ? ctx->ps.Pm.naper : 1;
    EN(o_aper, n * naper * sizeof(float4));
    O.aper = P<float4>(ctx->o_aper);
    O.dbkg = ctx->cfg_local ? P<float>(ctx->o_dbkg) : nullptr;
    O.lstat = P<MeshStat>(ctx->o_lstat);
    O.fluxerr_iso = P<float>(ctx->o_d[9]);
    return SEXGPU_OK;
}

unsigned grid1(long long n, int t) { return n > 0 ? (unsigned)((n + t - 1) / t) : 1u; }

// ---------------------------------------------------------------------------
// The pipeline in resumable stages: pipe_begin (buffers, background),
// pipe_detect (subtraction, filter, threshold, components, raw objects),
// pipe_deblend, pipe_analyse, pipe_clean, pipe_end (photometry, catalogue).
// State that crosses stages lives in ctx->ps; parameters a later stage reads
// (ps.Pm) may be changed between stages.
// ---------------------------------------------------------------------------
int pipe_begin(sexgpu_ctx *ctx, const float *d_img, const float *d_wmap, int w, int h, const sexgpu_config *cfg) {
    int rc = check_config(cfg, w, h);
    // MAP_VAR, MAP_RMS, MAP_WEIGHT need a weight map; NONE and BACKGROUND take none
    if (!rc && (cfg->weight_type >= 1 && cfg->weight_type <= 3) != (d_wmap != nullptr)) rc = SEXGPU_ERR_ARG;
    if (rc) {
        ctx->err = "invalid configuration or frame size";
        return rc;
    }
    cudaStream_t st = ctx->stream;
    PipeState &ps = ctx->ps;
    ps.stage = 0;
    FrameParams &Pm = ps.Pm;
    make_params(cfg, w, h, Pm);
    Pm.loop_cap = ctx->loop_cap;
    ps.w = w;
    ps.h = h;
    ps.d_img = d_img;
    const long long N = (long long)w * h;
    const int nb = Pm.nbx * Pm.nby;
    // ---- buffers sized by the frame
    EN(sub, N * 4);
    EN(cd, N * 4);
    EN(lab, N * 4);
    EN(cnt, N * 4);
    EN(flag, N * 4);
    EN(pos, std::max(N, 4 * ((N + SCAN_TILE - 1) / SCAN_TILE) + 4) * 4);  // or the four tile arrays of the root scans
    EN(alloc, N * 4);
    EN(pos2idx, N * 4);
    EN(keys, N * 4);
    EN(vals, N * 4);
    EN(kalt, N * 4);
    EN(valt, N * 4);
    EN(rpix, N * 4);
    EN(objkey, N * 4);
    EN(scan_tmp, (std::max(scan_temp_ints(N), radix_temp_ints(N)) + 64) * 4);
    EN(ms, nb * sizeof(MeshStat));
    EN(back, nb * 4);
    EN(sigma, nb * 4);
    EN(back2, nb * 4);
    EN(back3, nb * 4);
    EN(sigma3, nb * 4);
    EN(dback, nb * 4);
    EN(bu, (size_t)nb * 4 + 64);
    EN(rownode, (size_t)h * Pm.nbx * 4);
    EN(rowdnode, (size_t)h * Pm.nbx * 4);
    EN(rowu, (size_t)h * Pm.nbx * 4);
    EN(colk, w * 4);
    EN(coldx, w * 4);
    EN(sc, sizeof(FrameScalars));
    BackBufs &B = ps.B;
    B.ms = P<MeshStat>(ctx->ms);
    B.back = P<float>(ctx->back);
    B.sigma = P<float>(ctx->sigma);
    B.back2 = P<float>(ctx->back2);
    B.back3 = P<float>(ctx->back3);
    B.sigma3 = P<float>(ctx->sigma3);
    B.dback = P<float>(ctx->dback);
    B.u = P<float>(ctx->bu);
    B.rownode = P<float>(ctx->rownode);
    B.rowdnode = P<float>(ctx->rowdnode);
    B.rowu = P<float>(ctx->rowu);
    B.colk = P<int>(ctx->colk);
    B.coldx = P<float>(ctx->coldx);
    FrameScalars *d_sc = P<FrameScalars>(ctx->sc);
    int *tmp = P<int>(ctx->scan_tmp);

    if (ps.cst) {  // being captured: the graph's device copy
        B.colk = reinterpret_cast<int *>(ps.cst);
        B.coldx = reinterpret_cast<float *>(ps.cst + (size_t)w * 4);
    } else {
        column_table(w, Pm.nbx, Pm.bw, ctx->colk_h, ctx->coldx_h);
        CK(cudaMemcpyAsync(B.colk, ctx->colk_h.data(), w * 4, cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(B.coldx, ctx->coldx_h.data(), w * 4, cudaMemcpyHostToDevice, st));
    }
    rc = load_mask(ctx, cfg->filter_flag ? cfg->conv : nullptr, cfg->conv_w, cfg->conv_h);
    if (rc) return rc;

    stage_begin(ctx);
    int nl = 0;
    k_init_scalars<<<1, 1, 0, st>>>(d_sc);
    ps.wvar = nullptr;
    if (d_wmap) {
        // pixels of unusable weight are blank for the background and the detection
        EN(imgm, N * 4);
        EN(wvar, N * 4);
        EN(wratio, (size_t)nb * 4);
        launch_weight_mask(d_img, d_wmap, Pm.wtype, P<float>(ctx->imgm), N, st);
        d_img = ps.d_img = P<float>(ctx->imgm);
        nl += 1;
    }
    launch_background(B, d_img, Pm, d_sc, st, nl);
    if (d_wmap) {
        launch_weight_var(B, d_wmap, Pm, P<float>(ctx->wratio), P<float>(ctx->wvar), d_sc, st);
        ps.wvar = P<float>(ctx->wvar);
        nl += Pm.wtype != 2 ? 3 : 1;
    } else if (Pm.wtype == 4) {
        // WEIGHT_TYPE BACKGROUND: the variance of every pixel is the square of
        // the background rms map (the sigma mesh map through the background's
        // splines, as BACKGROUND_RMS)
        const int nbm = Pm.nbx * Pm.nby;
        EN(wvar, N * 4);
        EN(rmsd, (size_t)nbm * 4);
        EN(rmsu, std::max((size_t)nbm * 4 + 64, (size_t)h * Pm.nbx * 4));
        EN(rmsnode, (size_t)h * Pm.nbx * 4);
        EN(rmsdnode, (size_t)h * Pm.nbx * 4);
        k_back_spline<<<(Pm.nbx + 127) / 128, 128, 0, st>>>(B.sigma3, P<float>(ctx->rmsd), P<float>(ctx->rmsu), Pm.nbx,
                                                            Pm.nby);
        k_row_nodes<<<(h + 127) / 128, 128, 0, st>>>(B.sigma3, P<float>(ctx->rmsd), Pm.nbx, Pm.nby, Pm.bh, h,
                                                     P<float>(ctx->rmsnode), P<float>(ctx->rmsdnode),
                                                     P<float>(ctx->rmsu));
        k_rms_map<<<grid1(N, 256), 256, 0, st>>>(P<float>(ctx->rmsnode), P<float>(ctx->rmsdnode), B.colk, B.coldx,
                                                Pm.nbx, w, N, P<float>(ctx->wvar), 1);
        ps.wvar = P<float>(ctx->wvar);
        nl += 3;
    }
    stage_mark(ctx, "background", nl + 1);
    ps.stage = 1;
    return SEXGPU_OK;
}

int pipe_detect(sexgpu_ctx *ctx) {
    PipeState &ps = ctx->ps;
    if (ps.stage != 1) return SEXGPU_ERR_ARG;
    cudaStream_t st = ctx->stream;
    const FrameParams &Pm = ps.Pm;
    const int w = ps.w, h = ps.h;
    const long long N = (long long)w * h;
    const float *d_img = ps.d_img;
    BackBufs &B = ps.B;
    FrameScalars *d_sc = P<FrameScalars>(ctx->sc);
    int *tmp = P<int>(ctx->scan_tmp);
    int rc = SEXGPU_OK, nl = 0;
    const bool tiled = launch_sub_filter(d_img, P<float>(ctx->sub), P<float>(ctx->cd), P<int>(ctx->lab), B, Pm, d_sc, ps.wvar,
                      ctx->cmask, st, nl);
    stage_mark(ctx, "sub_filter", nl);

    nl = 0;
    int *lab = P<int>(ctx->lab), *cnt = P<int>(ctx->cnt), *flag = P<int>(ctx->flag), *pos = P<int>(ctx->pos);
    CK(cudaMemsetAsync(cnt, 0, N * 4, st));
    launch_ccl(lab, cnt, Pm, d_sc, st, nl, tiled);  // labels to roots, component sizes at the roots
    stage_mark(ctx, "ccl", nl);

    // ---- raw objects
    // per-tile counts of roots and kept pixels, scanned into tile offsets
    // (pos holds the two count arrays and the two offset arrays)
    const int ntile = (int)((N + SCAN_TILE - 1) / SCAN_TILE);
    int *troots = pos, *tkept = pos + ntile, *troff = pos + 2 * ntile, *tkoff = pos + 3 * ntile;
    k_root_tile_counts<<<ntile, SCAN_THREADS, 0, st>>>(lab, cnt, N, Pm.minarea, troots, tkept);
    exclusive_scan(troots, troff, ntile, &d_sc->nroots, tmp, st);
    exclusive_scan(tkept, tkoff, ntile, nullptr, tmp, st);
    // roots (the capacity in the capacity form) and the length of the root
    // arrays: in the capacity form, the most roots the frame can hold (each
    // has minarea pixels), since they are numbered before the gate checks
    int nroots, rlen;
    if (ps.capf) {
        nroots = ps.cap_roots;
        rlen = (int)(N / std::max(Pm.minarea, 1));
        k_gate<<<1, 1, 0, st>>>(d_sc, 1, ps.cap_roots, ps.cap_rootpix, ps.cap_obj, nullptr, 0);
    } else {
        rc = read_scalars(ctx);
        if (rc) return rc;
        if (ctx->hsc.dthresh <= 0.0f || ctx->hsc.thresh <= 0.0f) {
            ctx->err = "zero or negative threshold";
            return SEXGPU_ERR_THRESH;
        }
        nroots = rlen = ctx->hsc.nroots;
    }
    ps.nroots = nroots;
    const int *nroots_dev = ps.capf ? &d_sc->nroots : nullptr;
    EN(rsize, ((size_t)rlen + 1) * 4);
    EN(roff, ((size_t)rlen + 1) * 4);
    EN(rfirst, ((size_t)rlen + 1) * 4);
    EN(rymax, ((size_t)rlen + 1) * 4);
    EN(rlastx, ((size_t)rlen + 1) * 4);
    EN(rfdpeak, ((size_t)rlen + 1) * 4);
    EN(rfdflux, ((size_t)rlen + 1) * 4);
    EN(rnkept, ((size_t)rlen + 1) * 4);
    EN(robjbase, ((size_t)rlen + 1) * 4);
    EN(rdthr, ((size_t)rlen + 1) * 4);
    EN(rathr, ((size_t)rlen + 1) * 4);
    RootBufs &R = ps.R;
    R.size = P<int>(ctx->rsize);
    R.off = P<int>(ctx->roff);
    R.first = P<int>(ctx->rfirst);
    R.ymax = P<int>(ctx->rymax);
    R.lastx = P<int>(ctx->rlastx);
    R.fdpeak = P<float>(ctx->rfdpeak);
    R.fdflux = P<float>(ctx->rfdflux);
    R.nkept = P<int>(ctx->rnkept);
    R.objbase = P<int>(ctx->robjbase);
    R.dthresh = P<float>(ctx->rdthr);
    R.thresh = P<float>(ctx->rathr);
    k_root_number<<<ntile, SCAN_THREADS, 0, st>>>(lab, cnt, N, Pm.minarea, troff, flag, R.size, R.first);
    exclusive_scan(R.size, R.off, nroots, &d_sc->nrootpix, tmp, st, nroots_dev);
    unsigned *keys = P<unsigned>(ctx->keys), *vals = P<unsigned>(ctx->vals);
    int *pos2idx = P<int>(ctx->pos2idx);
    k_root_compact<<<ntile, SCAN_THREADS, 0, st>>>(lab, cnt, N, Pm.minarea, tkoff, flag, keys, vals,
                                                   P<int>(ctx->alloc), pos2idx);
    if (ps.wvar) {
        CK(cudaMemsetAsync(R.dthresh, 0x7f, (size_t)(nroots + 1) * 4, st));
        CK(cudaMemsetAsync(R.thresh, 0x7f, (size_t)(nroots + 1) * 4, st));
        k_root_thresholds<<<grid1(N, 256), 256, 0, st>>>(lab, cnt, flag, N, Pm.minarea, ps.wvar, Pm.wthr,
                                                         Pm.detect_thresh, Pm.analysis_thresh, d_sc,
                                                         (int *)R.dthresh, (int *)R.thresh);
    } else {
        k_root_thresholds_global<<<grid1(nroots, 256), 256, 0, st>>>(nroots, nroots_dev, d_sc, R.dthresh,
                                                                       R.thresh);
    }
    int nrootpix;
    if (ps.capf) {
        nrootpix = ps.cap_rootpix;
        k_gate<<<1, 1, 0, st>>>(d_sc, 0, ps.cap_roots, ps.cap_rootpix, ps.cap_obj, nullptr, 0);
    } else {
        rc = read_scalars(ctx);
        if (rc) return rc;
        nrootpix = ctx->hsc.nrootpix;
    }
    ps.nrootpix = nrootpix;
    const int *nrootpix_dev = ps.capf ? &d_sc->nrootpix : nullptr;
    // the sort's last pass writes the pixel lists (rpix) and each root
    // pixel's list index (pos2idx) directly
    unsigned *rpix = P<unsigned>(ctx->rpix);
    radix_sort_pairs(keys, vals, P<unsigned>(ctx->kalt), P<unsigned>(ctx->valt), nrootpix, bits_for(nroots), tmp, st,
                     nrootpix_dev, rpix, pos2idx);
    stage_mark(ctx, "roots", 4 + 2 * scan_launches(ntile) + scan_launches(nroots) +
                                 radix_launches(bits_for(nroots), nrootpix) + (nrootpix == 1 ? 1 : 0));
    ps.stage = 2;
    return SEXGPU_OK;
}

int pipe_deblend(sexgpu_ctx *ctx) {
    PipeState &ps = ctx->ps;
    if (ps.stage != 2) return SEXGPU_ERR_ARG;
    cudaStream_t st = ctx->stream;
    const FrameParams &Pm = ps.Pm;
    const int w = ps.w, h = ps.h, nroots = ps.nroots, nrootpix = ps.nrootpix;
    RootBufs &R = ps.R;
    FrameScalars *d_sc = P<FrameScalars>(ctx->sc);
    int *tmp = P<int>(ctx->scan_tmp);
    int *pos2idx = P<int>(ctx->pos2idx);
    unsigned *rpix = P<unsigned>(ctx->rpix);
    int rc = SEXGPU_OK;
    // ---- deblending
    size_t M = (size_t)nrootpix + 1;
    EN(dpar, M * 4);
    EN(dlev, M * 4);
    EN(dsz, M * 4);
    EN(dorder, M * 4);
    EN(drl0, M * 4);
    EN(drl1, M * 4);
    EN(dnid0, M * 4);
    EN(dnid1, M * 4);
    EN(dacc, M * 32);
    EN(nr0, M * 4);
    EN(nr1, M * 4);
    EN(nf0, M * 4);
    EN(nf1, M * 4);
    EN(ns0, M * 4);
    EN(ns1, M * 4);
    EN(nc0, M * 4);
    EN(nc1, M * 4);
    EN(na0, M * 4);
    EN(na1, M * 4);
    EN(dkept, M * 8);
    EN(down, M * 4);
    EN(dkl, M * 4);
    EN(dkidx, M * 4);
    EN(dpint, M * 8 * 4);
    EN(darena, M * DL_ARENA_BYTES);
    EN(drec, M * 4);
    DebArgs &A = ps.A;
    A.cd = P<float>(ctx->cd);
    A.sub = P<float>(ctx->sub);
    A.pos2idx = pos2idx;
    A.rpix = rpix;
    A.R = R;
    DebBufs &D = A.D;
    D.par = P<int>(ctx->dpar);
    D.lev = P<int>(ctx->dlev);
    D.sz = P<int>(ctx->dsz);
    D.order = P<int>(ctx->dorder);
    D.rl0 = P<int>(ctx->drl0);
    D.rl1 = P<int>(ctx->drl1);
    D.nid0 = P<int>(ctx->dnid0);
    D.nid1 = P<int>(ctx->dnid1);
    D.acc = P<unsigned long long>(ctx->dacc);
    D.nd_root0 = P<int>(ctx->nr0);
    D.nd_root1 = P<int>(ctx->nr1);
    D.nd_flag0 = P<int>(ctx->nf0);
    D.nd_flag1 = P<int>(ctx->nf1);
    D.nd_nson0 = P<int>(ctx->ns0);
    D.nd_nson1 = P<int>(ctx->ns1);
    D.nd_okc0 = P<int>(ctx->nc0);
    D.nd_okc1 = P<int>(ctx->nc1);
    D.nd_oka0 = P<int>(ctx->na0);
    D.nd_oka1 = P<int>(ctx->na1);
    D.kept = P<unsigned long long>(ctx->dkept);
    D.own = P<int>(ctx->down);
    D.kl = P<int>(ctx->dkl);
    D.kidx = P<int>(ctx->dkidx);
    D.pint = P<int>(ctx->dpint);
    D.arena = P<unsigned char>(ctx->darena);
    D.rec = P<int>(ctx->drec);
    A.sc = d_sc;
    A.alloc = P<int>(ctx->alloc);
    A.objkey = P<unsigned>(ctx->objkey);
    A.w = w;
    A.h = h;
    A.N = Pm.nthresh;
    A.debminarea = Pm.debminarea;
    A.mincont = Pm.mincont;
    A.loop_cap = Pm.loop_cap;
    A.wdiv = make_fastdiv((unsigned)w);
    EN(rlists, (size_t)(DL_NLISTS * (nroots + 1)) * 4);
    EN(rcounts, 5 * DL_NLISTS * 4);
    DebStreams S;
    S.main = st;
    for (int i = 0; i < DL_SIDE; i++) {
        S.side[i] = ctx->side[i];
        S.join[i] = ctx->ev_join[i];
    }
    S.fork = ctx->ev_fork;
    const int *nroots_dev = ps.capf ? &d_sc->nroots : nullptr;
    launch_deblend_split(R.size, nroots, nroots_dev, P<int>(ctx->rlists), P<int>(ctx->rcounts), P<unsigned>(ctx->keys),
                         P<unsigned>(ctx->vals), P<unsigned>(ctx->kalt), P<unsigned>(ctx->valt), tmp, st);
    launch_deblend_sweep(A, P<int>(ctx->rlists), P<int>(ctx->rcounts), nroots, S);
    exclusive_scan(R.nkept, R.objbase, nroots, &d_sc->nobj, tmp, st, nroots_dev);
    int nobj;
    if (ps.capf) {
        // a stop also empties the size-class lists, so that no branch is assigned
        nobj = ps.cap_obj;
        k_gate<<<1, 1, 0, st>>>(d_sc, 0, ps.cap_roots, ps.cap_rootpix, ps.cap_obj, P<int>(ctx->rcounts), DL_NLISTS);
    } else {
        rc = read_scalars(ctx);
        if (rc) return rc;
        nobj = ctx->hsc.nobj;
    }
    ps.nobj = nobj;
    ctx->cfg_local = Pm.bp_local != 0;
    rc = alloc_objects(ctx, nobj);
    if (rc) return rc;
    A.O = ctx->O;
    launch_deblend_assign(A, P<int>(ctx->rlists), P<int>(ctx->rcounts), nroots, S);
    stage_mark(ctx, "deblend", 16 + deblend_split_launches(nroots) + scan_launches(nroots));
    ps.stage = 3;
    return SEXGPU_OK;
}

int pipe_analyse(sexgpu_ctx *ctx) {
    PipeState &ps = ctx->ps;
    if (ps.stage != 3) return SEXGPU_ERR_ARG;
    cudaStream_t st = ctx->stream;
    const FrameParams &Pm = ps.Pm;
    const int w = ps.w, h = ps.h, nobj = ps.nobj;
    const DebArgs &A = ps.A;
    const BackBufs &B = ps.B;
    FrameScalars *d_sc = P<FrameScalars>(ctx->sc);
    int *tmp = P<int>(ctx->scan_tmp);
    unsigned *vals = P<unsigned>(ctx->vals);
    unsigned *rpix = P<unsigned>(ctx->rpix);
    // ---- object pixel lists (stable by object id: raster order inside)
    ObjBufs &O = ctx->O;
    const int *nobj_dev = ps.capf ? &d_sc->nobj : nullptr;
    exclusive_scan(O.n, O.off, nobj, nullptr, tmp, st, nobj_dev);
    // the deblending's size-class lists are free now: the list of the raw
    // objects too large for the one-warp partition goes there
    launch_obj_partition(rpix, A.objkey, ps.R, O.off, ps.nroots, ps.capf ? &d_sc->nroots : nullptr, vals,
                         P<int>(ctx->kalt), &d_sc->nbig, P<int>(ctx->rlists), st);
    AnaArgs AA;
    EN(o_raw, (size_t)(nobj + 1) * sizeof(RobustRaw));
    AA.raw = P<RobustRaw>(ctx->o_raw);
    EN(o_xraw, (size_t)(nobj + 1) * sizeof(ExamRaw));
    AA.xraw = P<ExamRaw>(ctx->o_xraw);
    AA.cd = A.cd;
    AA.sub = A.sub;
    AA.back = B.back3;
    AA.opix = vals;
    AA.O = O;
    AA.sc = d_sc;
    AA.w = w;
    AA.h = h;
    AA.nbx = Pm.nbx;
    AA.nby = Pm.nby;
    AA.bw = Pm.bw;
    AA.bh = Pm.bh;
    AA.nobj = nobj;
    AA.nobj_dev = nobj_dev;
    AA.minarea = Pm.minarea;
    AA.clean_flag = Pm.clean_flag;
    AA.gain = Pm.gain;
    AA.satur = Pm.satur_level;
    AA.wdiv = make_fastdiv((unsigned)w);
    AA.wvar = ps.wvar;
    AA.wthr = Pm.wthr;
    AA.afac = Pm.analysis_thresh;
    AA.bp_thick = Pm.bp_thick;
    launch_analyse(AA, st);
    stage_mark(ctx, "analyse", 6 + (Pm.bp_local ? 2 : 0) + scan_launches(nobj));
    ps.stage = 4;
    return SEXGPU_OK;
}

int pipe_clean(sexgpu_ctx *ctx) {
    PipeState &ps = ctx->ps;
    if (ps.stage != 4) return SEXGPU_ERR_ARG;
    cudaStream_t st = ctx->stream;
    const FrameParams &Pm = ps.Pm;
    const int w = ps.w, h = ps.h, nobj = ps.nobj;
    const DebArgs &A = ps.A;
    ObjBufs &O = ctx->O;
    FrameScalars *d_sc = P<FrameScalars>(ctx->sc);
    int *tmp = P<int>(ctx->scan_tmp);
    unsigned *vals = P<unsigned>(ctx->vals);
    int rc = SEXGPU_OK;
    // ---- CLEAN
    int nv = 0;
    int cl_launch = 0;
    if (Pm.clean_flag && nobj > 0) {
        int gx = (int)(w / CL_CELL) + 2, gy = (int)(h / CL_CELL) + 2, ncell = gx * gy;
        EN(cellhead, (size_t)(ncell + 1) * 4);   // cell counts, then starts
        EN(cellnext, (size_t)(ncell + 1) * 4);   // fill cursors
        EN(amp, (size_t)(nobj + 1) * sizeof(CleanObj));
        EN(vkey, (size_t)(nobj + 1) * 4);
        EN(vval, (size_t)(nobj + 1) * 4);
        EN(vkalt, (size_t)(nobj + 1) * 4);
        EN(vvalt, (size_t)(nobj + 1) * 4);
        int *cellcnt = P<int>(ctx->cellhead), *cellcur = P<int>(ctx->cellnext);
        CK(cudaMemsetAsync(cellcnt, 0, (size_t)(ncell + 1) * 4, st));
        CK(cudaMemsetAsync(cellcur, 0, (size_t)(ncell + 1) * 4, st));
        const int *nobj_dev = ps.capf ? &d_sc->nobj : nullptr;
        k_clean_count<<<grid1(nobj, 128), 128, 0, st>>>(O, nobj, nobj_dev, cellcnt, gx, gy);
        exclusive_scan(cellcnt, cellcnt, ncell + 1, nullptr, tmp, st);
        k_clean_pack<<<grid1(nobj, 128), 128, 0, st>>>(O, nobj, nobj_dev, Pm.clean_param, cellcnt, cellcur,
                                                       P<CleanObj>(ctx->amp), gx, gy);
        k_clean_pairs<<<(unsigned)nobj, CL_PAIR_WARPS * 32, 0, st>>>(P<CleanObj>(ctx->amp), nobj, nobj_dev,
                                                                      Pm.clean_param, cellcnt, O.master, gx, gy);
        CK(cudaMemsetAsync(&d_sc->nsurv, 0, 4, st));
        k_clean_chain<<<grid1(nobj, 256), 256, 0, st>>>(O, nobj, nobj_dev, P<unsigned>(ctx->vkey),
                                                        P<unsigned>(ctx->vval), &d_sc->nsurv, &d_sc->status,
                                                        Pm.loop_cap);
        if (ps.capf) {
            // the victim count stays on the device: the one-block sort takes
            // short lists, the radix sorts (counted by nvbig) long ones
            unsigned *vkey = P<unsigned>(ctx->vkey), *vval = P<unsigned>(ctx->vval);
            k_gate<<<1, 1, 0, st>>>(d_sc, 0, ps.cap_roots, ps.cap_rootpix, ps.cap_obj, nullptr, 0);
            k_victim_sort<<<1, 1024, 0, st>>>(vkey, vval, nobj, &d_sc->nsurv, &d_sc->nvbig);
            radix_sort_pairs(vval, vkey, P<unsigned>(ctx->vkalt), P<unsigned>(ctx->vvalt), nobj, bits_for(nobj), tmp,
                             st, &d_sc->nvbig);
            radix_sort_pairs(vkey, vval, P<unsigned>(ctx->vkalt), P<unsigned>(ctx->vvalt), nobj, bits_for(nobj), tmp,
                             st, &d_sc->nvbig);
            k_clean_merge<<<grid1(nobj, 128), 128, 0, st>>>(O, vkey, vval, nobj, &d_sc->nsurv);
            k_alloc_victims<<<nobj, 128, 0, st>>>(O, vals, A.alloc, nobj, nobj_dev);
            stage_mark(ctx, "clean", 0);
            ps.stage = 5;
            return SEXGPU_OK;
        }
        rc = read_scalars(ctx);
        if (rc) return rc;
        nv = ctx->hsc.nsurv;
        int sort_launches = 0;
        if (nv > 0 && nv <= CL_SORT_MAX) {
            k_victim_sort<<<1, 1024, 0, st>>>(P<unsigned>(ctx->vkey), P<unsigned>(ctx->vval), nv, nullptr, nullptr);
            sort_launches = 1;
        } else if (nv > 0) {
            radix_sort_pairs(P<unsigned>(ctx->vval), P<unsigned>(ctx->vkey), P<unsigned>(ctx->vkalt),
                             P<unsigned>(ctx->vvalt), nv, bits_for(nobj), tmp, st);  // victims by index
            radix_sort_pairs(P<unsigned>(ctx->vkey), P<unsigned>(ctx->vval), P<unsigned>(ctx->vkalt),
                             P<unsigned>(ctx->vvalt), nv, bits_for(nobj), tmp, st);  // then by master
            sort_launches = 2 * radix_launches(bits_for(nobj), nv);
        }
        if (nv > 0) {
            k_clean_merge<<<grid1(nv, 128), 128, 0, st>>>(O, P<unsigned>(ctx->vkey), P<unsigned>(ctx->vval), nv,
                                                          nullptr);
            k_alloc_victims<<<nobj, 128, 0, st>>>(O, vals, A.alloc, nobj, nullptr);
        }
        cl_launch = 6 + scan_launches(ncell + 1) + sort_launches;
    } else if (nobj > 0) {
        CK(cudaMemsetAsync(O.fmaster, 0xff, (size_t)nobj * 4, st));
    }
    stage_mark(ctx, "clean", cl_launch);
    ps.stage = 5;
    return SEXGPU_OK;
}

int pipe_end(sexgpu_ctx *ctx) {
    PipeState &ps = ctx->ps;
    if (ps.stage != 5) return SEXGPU_ERR_ARG;
    cudaStream_t st = ctx->stream;
    const FrameParams &Pm = ps.Pm;
    const int w = ps.w, h = ps.h, nobj = ps.nobj;
    const DebArgs &A = ps.A;
    const RootBufs &R = ps.R;
    ObjBufs &O = ctx->O;
    FrameScalars *d_sc = P<FrameScalars>(ctx->sc);
    int *tmp = P<int>(ctx->scan_tmp);
    int rc = SEXGPU_OK;
    // ---- photometry / FLAGS
    EndArgs E;
    EN(o_eraw, (size_t)(nobj + 1) * sizeof(EndRaw));
    E.raw = P<EndRaw>(ctx->o_eraw);
    E.sub = A.sub;
    E.alloc = A.alloc;
    E.O = O;
    E.sc = d_sc;
    E.w = w;
    E.h = h;
    E.n = nobj;
    const int *nobj_dev = ps.capf ? &d_sc->nobj : nullptr;
    E.n_dev = nobj_dev;
    E.mask_type = Pm.mask_type;
    E.aperture = Pm.aperture;
    E.naper = Pm.naper;
    for (int k = 0; k < SEXGPU_MAXAPER; k++) E.apertures[k] = Pm.apertures[k];
    E.autoparam0 = Pm.autoparam0;
    E.autoparam1 = Pm.autoparam1;
    E.gain = Pm.gain;
    E.zp = Pm.mag_zeropoint;
    E.satur = Pm.satur_level;
    E.wvar = ps.wvar;
    for (int p = 0; p < 2; p++) {
        EN(kitem[p], (size_t)KR_ITEMS * sizeof(KronItem));
        EN(kchunk[p], (size_t)KR_CHUNKS * sizeof(int));
        EN(kpart[p], (size_t)KR_CHUNKS * sizeof(KronAcc));
        E.K.item[p] = P<KronItem>(ctx->kitem[p]);
        E.K.chunk[p] = P<int>(ctx->kchunk[p]);
        E.K.part[p] = P<KronAcc>(ctx->kpart[p]);
    }
    E.K.icap = KR_ITEMS;
    E.K.ccap = KR_CHUNKS;
    E.K.warp_max = ctx->kron_warp_max;
    E.nnw = ctx->nnw_dev;
    E.seeing = Pm.seeing;
    E.pixscale = Pm.pixscale;
    int nl = 0;
    launch_endobject(E, nobj, st, nl);
    stage_mark(ctx, "endobject", nl);

    // ---- catalogue order
    EN(skeys, (size_t)(nobj + 1) * 4);
    EN(svals, (size_t)(nobj + 1) * 4);
    EN(skalt, (size_t)(nobj + 1) * 4);
    EN(svalt, (size_t)(nobj + 1) * 4);
    int *sflag = P<int>(ctx->cnt);  // free now
    CK(cudaMemsetAsync(O.number, 0, (size_t)(nobj + 1) * 4, st));
    k_surv_flags<<<grid1(nobj + 1, 256), 256, 0, st>>>(O, nobj, nobj_dev, sflag);
    exclusive_scan(sflag, sflag, nobj, &d_sc->nsurv, tmp, st, nobj_dev);
    int ns;
    if (ps.capf) {
        ns = nobj;
        k_gate<<<1, 1, 0, st>>>(d_sc, 0, ps.cap_roots, ps.cap_rootpix, ps.cap_obj, nullptr, 0);
    } else {
        rc = read_scalars(ctx);
        if (rc) return rc;
        ns = ctx->hsc.nsurv;
    }
    const int *ns_dev = ps.capf ? &d_sc->nsurv : nullptr;
    k_surv_compact<<<grid1(nobj + 1, 256), 256, 0, st>>>(O, R.ymax, R.lastx, sflag, nobj, nobj_dev, w, Pm.numbering,
                                                         P<unsigned>(ctx->skeys), P<unsigned>(ctx->svals));
    // completion keys are below w*h; first-pixel numbering has all keys 0
    // (the survivors are already in index order)
    const int cbits = Pm.numbering == 0 ? bits_for((long long)w * h - 1) : 0;
    radix_sort_pairs(P<unsigned>(ctx->skeys), P<unsigned>(ctx->svals), P<unsigned>(ctx->skalt),
                     P<unsigned>(ctx->svalt), ns, cbits, tmp, st, ns_dev);
    k_number<<<grid1(ns + 1, 256), 256, 0, st>>>(O, P<unsigned>(ctx->svals), ns, ns_dev);
    EN(rows, (size_t)(ns + 1) * sizeof(sexgpu_object));
    k_write_rows<<<grid1(ns + 1, 128), 128, 0, st>>>(O, P<unsigned>(ctx->svals), ns, ns_dev,
                                                     P<sexgpu_object>(ctx->rows));
    stage_mark(ctx, "catalog", 4 + scan_launches(nobj) + radix_launches(cbits, ns));
    CK(cudaGetLastError());
    if (ps.capf) {
        // the scalars come back with the frame; the host reads them after the
        // stream (or the graph) has finished
        CK(cudaMemcpyAsync(ctx->hsc_pin, d_sc, sizeof(FrameScalars), cudaMemcpyDeviceToHost, st));
        ps.ns = ns;
        ps.stage = 6;
        return SEXGPU_OK;
    }
    rc = read_scalars(ctx);
    if (rc) return rc;
    stage_collect(ctx);
    ctx->last_w = w;
    ctx->last_h = h;
    ctx->last_nobj = nobj;
    ctx->last_ns = ns;
    ps.ns = ns;
    ps.stage = 6;
    return SEXGPU_OK;
}

// the whole pipeline on a device-resident frame
int run_pipeline(sexgpu_ctx *ctx, const float *d_img, const float *d_wmap, int w, int h, const sexgpu_config *cfg) {
    int rc = pipe_begin(ctx, d_img, d_wmap, w, h, cfg);
    if (!rc) rc = pipe_detect(ctx);
    if (!rc) rc = pipe_deblend(ctx);
    if (!rc) rc = pipe_analyse(ctx);
    if (!rc) rc = pipe_clean(ctx);
    if (!rc) rc = pipe_end(ctx);
    return rc;
}

// ---------------------------------------------------------------------------
// Extraction through captured graphs ("graph" parameter).  A frame kind (the
// frame geometry, the configuration, the detection mask, the input buffers)
// is first extracted in the plain form, which gives its counts; capacities a
// quarter above them size the capacity form, which the next frame of that
// kind runs uncaptured (allocating what it needs) and then captures: from the
// frame after on, a frame is one cudaGraphLaunch and one wait for the
// scalars.  A frame whose counts exceed the capacities is extracted again in
// the plain form and the capacities grow.
// ---------------------------------------------------------------------------
constexpr int GRAPH_CACHE = 8;  // frame kinds kept per context

void free_batch_graph(sexgpu_ctx *ctx) {
    BatchGraph *b = ctx->bgraph;
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->in_host) cudaFreeHost(b->in_host);
    if (b->rows_dev) cudaFree(b->rows_dev);
    if (b->sc_dev) cudaFree(b->sc_dev);
    if (b->sc_host) cudaFreeHost(b->sc_host);
    if (b->rows_host) cudaFreeHost(b->rows_host);
    delete b;
    ctx->bgraph = nullptr;
}

// status of one frame from its scalars, as capacity_status: 1 when the frame
// must be extracted again without its graph
int scalars_status(const FrameScalars &sc) {
    const int s = sc.status;
    if (s & SX_ST_LOAD) return SEXGPU_ERR_LOAD;
    if (s & SX_ST_CAPACITY) return 1;
    if (s & SX_ST_LOOP) return SEXGPU_ERR_LOOP;
    if (s & SX_ST_RANGE) return SEXGPU_ERR_RANGE;
    if (s & SX_ST_THRESH) return SEXGPU_ERR_THRESH;
    return SEXGPU_OK;
}

void summary_from_scalars(const FrameScalars &sc, const FrameParams &P, sexgpu_summary *s) {
    memset(s, 0, sizeof(*s));
    s->nbackx = P.nbx;
    s->nbacky = P.nby;
    s->backmean = sc.backmean;
    s->backsig = sc.backsig;
    s->dthresh = sc.dthresh;
    s->thresh = sc.thresh;
    s->npix_above = sc.npix_above;
    s->nraw = sc.nroots;
    s->nraw_pix = sc.nrootpix;
    s->ndetected = sc.nobj;
    s->nobj = sc.nsurv;
    s->level_pix = (int64_t)sc.levpix;
    s->sigfac = sc.sigfac;
}

int cap_of(long long count, long long bound) {
    const long long c = count + count / 4 + 256;
    return (int)std::max(0ll, std::min(c, bound));
}

void learn_caps(const sexgpu_ctx *ctx, GraphEntry &e, long long N, int minarea) {
    e.cap_roots = std::max(e.cap_roots, cap_of(ctx->hsc.nroots, N / std::max(minarea, 1)));
    e.cap_rootpix = std::max(e.cap_rootpix, cap_of(ctx->hsc.nrootpix, N));
    e.cap_obj = std::max(e.cap_obj, cap_of(ctx->hsc.nobj, N));
}

void drop_graph(sexgpu_ctx *ctx, GraphEntry &e) {
    if (e.exec || e.graph) ctx->graph_epoch++;
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (e.graph) cudaGraphDestroy(e.graph);
    if (e.cst) cudaFree(e.cst);
    e.exec = nullptr;
    e.graph = nullptr;
    e.cst = nullptr;
}

// status of a capacity-form frame from its scalars: 1 when it must be
// extracted again in the plain form (a count beyond its capacity)
int capacity_status(sexgpu_ctx *ctx) {
    const int s = ctx->hsc.status;
    if (s & SX_ST_LOAD) {
        ctx->err = "a tile load did not complete in time; destroy this context";
        return SEXGPU_ERR_LOAD;
    }
    if (s & SX_ST_CAPACITY) return 1;
    if (s & SX_ST_LOOP) {
        ctx->err = "device loop iteration cap reached";
        return SEXGPU_ERR_LOOP;
    }
    if (s & SX_ST_RANGE) {
        ctx->err = "exact sum out of range";
        return SEXGPU_ERR_RANGE;
    }
    if (s & SX_ST_THRESH) {
        ctx->err = "zero or negative threshold";
        return SEXGPU_ERR_THRESH;
    }
    return SEXGPU_OK;
}

void set_caps(PipeState &ps, const GraphEntry &e) {
    ps.cap_roots = e.cap_roots;
    ps.cap_rootpix = e.cap_rootpix;
    ps.cap_obj = e.cap_obj;
}

// Captures the capacity form of the frame just extracted; a capture that
// fails leaves the frame kind to the uncaptured capacity form.
void capture_graph(sexgpu_ctx *ctx, GraphEntry &e, const float *d_img, const float *d_wmap, int w, int h,
                   const sexgpu_config *cfg) {
    PipeState &ps = ctx->ps;
    cudaStream_t st = ctx->stream;
    // the frame's constants into the entry's own device memory before the
    // capture; the graph reads them there
    if (!e.cst && cudaMalloc((void **)&e.cst, (size_t)8 * w + 4 * SX_MAXCONV * SX_MAXCONV) != cudaSuccess) {
        cudaGetLastError();
        e.cst = nullptr;
        e.no_graph = true;
        return;
    }
    {
        std::vector<int> ck;
        std::vector<float> cdx;
        column_table(w, e.Pm.nbx, e.Pm.bw, ck, cdx);
        const float *m = e.mask.data();
        const size_t mbytes = sizeof(float) * e.mask.size();
        if (cudaMemcpy(e.cst, ck.data(), (size_t)w * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(e.cst + (size_t)w * 4, cdx.data(), (size_t)w * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(e.cst + (size_t)8 * w, m, mbytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            e.no_graph = true;
            return;
        }
    }
    const unsigned long long gen0 = ctx->gen;
    cudaGraph_t g = nullptr;
    ps.capf = true;
    ps.cst = e.cst;
    set_caps(ps, e);
    int rc = SEXGPU_ERR_CUDA;
    cudaError_t ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
        rc = run_pipeline(ctx, d_img, d_wmap, w, h, cfg);
        ce = cudaStreamEndCapture(st, &g);
    }
    ps.capf = false;
    ps.cst = nullptr;
    if (ce == cudaSuccess && rc == SEXGPU_OK && g && ctx->gen == gen0) {
        size_t n = 0;
        if (cudaGraphGetNodes(g, nullptr, &n) == cudaSuccess) {
            std::vector<cudaGraphNode_t> nodes(n);
            cudaGraphGetNodes(g, nodes.data(), &n);
            e.kernels = 0;
            for (cudaGraphNode_t nd : nodes) {
                cudaGraphNodeType t;
                if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) e.kernels++;
            }
        }
        ce = cudaGraphInstantiate(&e.exec, g, 0);
        if (ce != cudaSuccess) e.exec = nullptr;
    }
    if (!e.exec) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        e.no_graph = true;
        return;
    }
    e.graph = g;
    ctx->graph_epoch++;
    e.gen = ctx->gen;
    e.ps = ps;
    e.O = ctx->O;
}

// host state after a capacity-form frame (the counts come from its scalars)
void finish_capacity(sexgpu_ctx *ctx, int w, int h) {
    PipeState &ps = ctx->ps;
    ps.nroots = ctx->hsc.nroots;
    ps.nrootpix = ctx->hsc.nrootpix;
    ps.nobj = ctx->hsc.nobj;
    ps.ns = ctx->hsc.nsurv;
    ps.stage = 6;
    ctx->last_w = w;
    ctx->last_h = h;
    ctx->last_nobj = ctx->hsc.nobj;
    ctx->last_ns = ctx->hsc.nsurv;
}

int run_graph(sexgpu_ctx *ctx, const float *d_img, const float *d_wmap, int w, int h, const sexgpu_config *cfg) {
    ctx->last_graph = 0;
    ctx->last_kernels = 0;
    ctx->last_entry = 0;
    if (check_config(cfg, w, h) || (cfg->weight_type >= 1 && cfg->weight_type <= 3) != (d_wmap != nullptr))
        return run_pipeline(ctx, d_img, d_wmap, w, h, cfg);  // reports the error
    FrameParams Pm;
    make_params(cfg, w, h, Pm);
    Pm.loop_cap = ctx->loop_cap;
    std::vector<float> mask(1, 1.0f);
    if (cfg->filter_flag) mask.assign(cfg->conv, cfg->conv + (size_t)cfg->conv_w * cfg->conv_h);
    GraphEntry *e = nullptr;
    for (GraphEntry &x : ctx->graphs)
        if (!memcmp(&x.Pm, &Pm, sizeof(Pm)) && x.mask == mask && x.d_img == d_img && x.d_wmap == d_wmap &&
            x.nnw == ctx->nnw_dev && x.kron_warp_max == ctx->kron_warp_max && x.grid_div == sx_grid_div) {
            e = &x;
            break;
        }
    if (!e) {
        if ((int)ctx->graphs.size() >= GRAPH_CACHE) {
            auto old = std::min_element(ctx->graphs.begin(), ctx->graphs.end(),
                                        [](const GraphEntry &a, const GraphEntry &b) { return a.used < b.used; });
            drop_graph(ctx, *old);
            ctx->graphs.erase(old);
        }
        ctx->graphs.emplace_back();
        e = &ctx->graphs.back();
        e->Pm = Pm;
        e->mask = mask;
        e->d_img = d_img;
        e->d_wmap = d_wmap;
        e->nnw = ctx->nnw_dev;
        e->kron_warp_max = ctx->kron_warp_max;
        e->grid_div = sx_grid_div;
        e->id = ++ctx->graph_clock;
    }
    e->used = ++ctx->graph_clock;
    ctx->last_entry = e->id;
    const long long N = (long long)w * h;
    if (!e->cap_obj) {  // a new frame kind: the plain form, and its counts
        int rc = run_pipeline(ctx, d_img, d_wmap, w, h, cfg);
        if (!rc) learn_caps(ctx, *e, N, Pm.minarea);
        return rc;
    }
    if (!ctx->hsc_pin) {
        if (cudaMallocHost((void **)&ctx->hsc_pin, sizeof(FrameScalars)) != cudaSuccess) {
            cudaGetLastError();
            ctx->hsc_pin = nullptr;
            ctx->err = "pinned host allocation failed";
            return SEXGPU_ERR_NOMEM;
        }
    }
    cudaStream_t st = ctx->stream;
    const bool replay = e->exec && e->gen == ctx->gen;
    int rc = SEXGPU_OK;
    if (replay) {
        ctx->ps = e->ps;
        ctx->O = e->O;
        ctx->cfg_local = Pm.bp_local != 0;
        ctx->hmask = mask;
        ctx->stage_ms.clear();
        ctx->stage_names.clear();
        ctx->stage_launches.clear();
        CK(cudaGraphLaunch(e->exec, st));
        ctx->last_graph = 1;
        ctx->last_kernels = e->kernels;
    } else {
        drop_graph(ctx, *e);
        ctx->ps.capf = true;
        set_caps(ctx->ps, *e);
        rc = run_pipeline(ctx, d_img, d_wmap, w, h, cfg);
        ctx->ps.capf = false;
        if (rc) return rc;
    }
    CK(stream_wait(ctx, st));
    ctx->hsc = *ctx->hsc_pin;
    rc = capacity_status(ctx);
    if (rc == 1) {  // counts beyond the capacities: plain form, larger capacities
        ctx->last_graph = 0;
        ctx->last_kernels = 0;
        drop_graph(ctx, *e);
        e->no_graph = false;
        rc = run_pipeline(ctx, d_img, d_wmap, w, h, cfg);
        if (!rc) learn_caps(ctx, *e, N, Pm.minarea);
        return rc;
    }
    if (rc) return rc;
    finish_capacity(ctx, w, h);
    if (!replay && !e->no_graph) {
        capture_graph(ctx, *e, d_img, d_wmap, w, h, cfg);
        finish_capacity(ctx, w, h);
    }
    return SEXGPU_OK;
}


void fill_summary(sexgpu_ctx *ctx, const FrameParams &P, sexgpu_summary *s) {
    if (!s) return;
    memset(s, 0, sizeof(*s));
    s->nbackx = P.nbx;
    s->nbacky = P.nby;
    s->backmean = ctx->hsc.backmean;
    s->backsig = ctx->hsc.backsig;
    s->dthresh = ctx->hsc.dthresh;
    s->thresh = ctx->hsc.thresh;
    s->npix_above = ctx->hsc.npix_above;
    s->nraw = ctx->hsc.nroots;
    s->nraw_pix = ctx->hsc.nrootpix;
    s->ndetected = ctx->last_nobj;
    s->nobj = ctx->last_ns;
    s->level_pix = (int64_t)ctx->hsc.levpix;
    s->sigfac = ctx->hsc.sigfac;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int sexgpu_create(sexgpu_ctx **out, int device) {
    if (!out) return SEXGPU_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0 || device < 0 || device >= n) {
        cudaGetLastError();
        return SEXGPU_ERR_NODEVICE;
    }
    if (cudaSetDevice(device) != cudaSuccess) return SEXGPU_ERR_NODEVICE;
    sexgpu_ctx *ctx = new sexgpu_ctx();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return SEXGPU_ERR_CUDA;
    }
    ctx->own_stream = true;
    bool ok = true;
    for (int i = 0; i < DL_SIDE; i++)
        ok = ok && cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&ctx->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
    if (!ok || cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess) {
        sexgpu_destroy(ctx);
        return SEXGPU_ERR_CUDA;
    }
    *out = ctx;
    return SEXGPU_OK;
}

static void free_buf(DevBuf &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
}

int sexgpu_destroy(sexgpu_ctx *ctx) {
    if (!ctx) return SEXGPU_ERR_ARG;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    DevBuf *all[] = {&ctx->img, &ctx->sub, &ctx->cd, &ctx->lab, &ctx->cnt, &ctx->flag, &ctx->pos, &ctx->alloc,
                     &ctx->seg, &ctx->pos2idx, &ctx->var, &ctx->scan_tmp, &ctx->keys, &ctx->vals, &ctx->kalt,
                     &ctx->valt, &ctx->ms, &ctx->back, &ctx->sigma, &ctx->back2, &ctx->back3, &ctx->sigma3,
                     &ctx->dback, &ctx->bu, &ctx->rownode, &ctx->rowdnode, &ctx->rowu, &ctx->colk, &ctx->coldx,
                     &ctx->rsize, &ctx->roff, &ctx->rfirst, &ctx->rymax, &ctx->rlastx, &ctx->rfdpeak,
                     &ctx->rfdflux, &ctx->rnkept, &ctx->robjbase, &ctx->rdthr, &ctx->rathr, &ctx->imgm, &ctx->wvar, &ctx->wratio, &ctx->rlists, &ctx->rcounts, &ctx->dpar, &ctx->dlev, &ctx->dsz, &ctx->dorder,
                     &ctx->drl0, &ctx->drl1, &ctx->dnid0, &ctx->dnid1, &ctx->dacc, &ctx->nr0, &ctx->nr1,
                     &ctx->nf0, &ctx->nf1, &ctx->ns0, &ctx->ns1, &ctx->nc0, &ctx->nc1, &ctx->na0, &ctx->na1,
                     &ctx->dkept, &ctx->down, &ctx->dkl, &ctx->dkidx, &ctx->dpint, &ctx->objkey,
                     &ctx->rpix, &ctx->darena, &ctx->drec, &ctx->o_iso, &ctx->o_sortkey, &ctx->amp, &ctx->alpha, &ctx->cellhead,
                     &ctx->cellnext, &ctx->vkey, &ctx->vval, &ctx->vkalt, &ctx->vvalt, &ctx->skeys, &ctx->svals,
                     &ctx->skalt, &ctx->svalt, &ctx->rows, &ctx->sc};
    for (DevBuf *b : all) free_buf(*b);
    for (auto &b : ctx->o_i) free_buf(b);
    for (auto &b : ctx->o_f) free_buf(b);
    for (auto &b : ctx->o_d) free_buf(b);
    for (int i = 0; i < 2; i++) {
        free_buf(ctx->kitem[i]);
        free_buf(ctx->kchunk[i]);
        free_buf(ctx->kpart[i]);
    }
    free_buf(ctx->o_sprob);
    free_buf(ctx->o_raw);
    free_buf(ctx->o_xraw);
    free_buf(ctx->o_eraw);
    free_buf(ctx->o_dbkg);
    free_buf(ctx->o_lstat);
    free_buf(ctx->o_aper);
    free_buf(ctx->aperrows);
    free_buf(ctx->fitsraw);
    free_buf(ctx->rmsd);
    free_buf(ctx->rmsnode);
    free_buf(ctx->rmsdnode);
    free_buf(ctx->rmsu);
    free_buf(ctx->rmsmap);
    free_buf(ctx->dnnw);
    free_buf(ctx->dmask);
    for (auto &s : ctx->stages) cudaEventDestroy(s.ev);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    for (int i = 0; i < DL_SIDE; i++) {
        if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
        if (ctx->ev_join[i]) cudaEventDestroy(ctx->ev_join[i]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_block) cudaEventDestroy(ctx->ev_block);
    free_batch_graph(ctx);
    for (GraphEntry &e : ctx->graphs) drop_graph(ctx, e);
    for (int i = 0; i < 2; i++) {
        free_buf(ctx->qimg[i]);
        free_buf(ctx->qvar[i]);
        if (ctx->qev[i]) cudaEventDestroy(ctx->qev[i]);
    }
    if (ctx->qstream) cudaStreamDestroy(ctx->qstream);
    ctx->graphs.clear();
    if (ctx->hsc_pin) cudaFreeHost(ctx->hsc_pin);
    for (sexgpu_ctx *w : ctx->workers) sexgpu_destroy(w);
    for (void *p : ctx->graveyard) cudaFree(p);
    for (void *p : ctx->host_graveyard) cudaFreeHost(p);
    if (ctx->stage_host) cudaFreeHost(ctx->stage_host);
    if (ctx->rows_host) cudaFreeHost(ctx->rows_host);
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return SEXGPU_OK;
}

int sexgpu_set_stream(sexgpu_ctx *ctx, void *stream) {
    if (!ctx) return SEXGPU_ERR_ARG;
    if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->own_stream = false;
    } else {
        cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        ctx->own_stream = true;
    }
    return SEXGPU_OK;
}

void sexgpu_default_config(sexgpu_config *c) {
    static const float pyramid[9] = {1 / 16.f, 2 / 16.f, 1 / 16.f, 2 / 16.f, 4 / 16.f, 2 / 16.f, 1 / 16.f, 2 / 16.f, 1 / 16.f};
    memset(c, 0, sizeof(*c));
    c->back_size = 64;
    c->back_filtersize = 3;
    c->back_filtthresh = 0.0;
    c->back_type = 0;
    c->thresh_type = 0;
    c->detect_thresh = 1.5;
    c->analysis_thresh = 1.5;
    c->filter_flag = 1;
    c->conv_w = c->conv_h = 3;
    c->conv = pyramid;
    c->detect_minarea = 5;
    c->deblend_nthresh = 32;
    c->deblend_mincont = 0.005;
    c->clean_flag = 1;
    c->clean_param = 1.0;
    c->satur_level = 50000.0;
    c->gain = 0.0;
    c->mag_zeropoint = 0.0;
    c->phot_aperture = 5.0;
    c->phot_autoparams[0] = 2.5;
    c->phot_autoparams[1] = 3.5;
    c->mask_type = 2;
    c->weight_type = 0;
    c->numbering = 0;
    c->seeing_fwhm = 1.2;
    c->pixel_scale = 0.0;
    c->back_photo_type = 0;
    c->back_photo_thick = 24;
}

const char *sexgpu_last_error(sexgpu_ctx *ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int sexgpu_extract_device(sexgpu_ctx *ctx, const float *d_img, const float *d_var, int w, int h,
                          const sexgpu_config *cfg, sexgpu_summary *sum) {
    if (!ctx || !d_img) return SEXGPU_ERR_ARG;
    cudaSetDevice(ctx->device);
    ctx->err.clear();
    int rc = ctx->graph_mode ? run_graph(ctx, d_img, d_var, w, h, cfg) : run_pipeline(ctx, d_img, d_var, w, h, cfg);
    if (rc == SEXGPU_OK && sum) {
        FrameParams Pm;
        make_params(cfg, w, h, Pm);
        fill_summary(ctx, Pm, sum);
    }
    return rc;
}

int sexgpu_copy_results(sexgpu_ctx *ctx, sexgpu_object *objs, int max_objects, int *nobj, int32_t *segmap,
                        float *sub, float *cd) {
    if (!ctx) return SEXGPU_ERR_ARG;
    cudaStream_t st = ctx->stream;
    long long N = (long long)ctx->last_w * ctx->last_h;
    int ns = ctx->last_ns, rc = SEXGPU_OK;
    if (nobj) *nobj = ns;
    if (objs) {
        int n = ns < max_objects ? ns : max_objects;
        if (ns > max_objects) rc = SEXGPU_ERR_CAPACITY;
        if (n > 0) CK(cudaMemcpyAsync(objs, ctx->rows.p, (size_t)n * sizeof(sexgpu_object), cudaMemcpyDeviceToHost, st));
    }
    if (segmap && N > 0) {
        EN(seg, N * 4);
        k_segmap<<<grid1(N, 256), 256, 0, st>>>(P<int>(ctx->alloc), ctx->O.number, P<int>(ctx->seg), N);
        CK(cudaMemcpyAsync(segmap, ctx->seg.p, N * 4, cudaMemcpyDeviceToHost, st));
    }
    if (sub && N > 0) CK(cudaMemcpyAsync(sub, ctx->sub.p, N * 4, cudaMemcpyDeviceToHost, st));
    if (cd && N > 0) CK(cudaMemcpyAsync(cd, ctx->cd.p, N * 4, cudaMemcpyDeviceToHost, st));
    CK(stream_wait(ctx, st));
    return rc;
}

int sexgpu_extract(sexgpu_ctx *ctx, const float *img, const float *var, int w, int h, const sexgpu_config *cfg,
                   sexgpu_object *objs, int max_objects, int *nobj, int32_t *segmap, float *sub, float *cd,
                   sexgpu_summary *sum) {
    if (!ctx || !img || w <= 0 || h <= 0) return SEXGPU_ERR_ARG;
    cudaSetDevice(ctx->device);
    long long N = (long long)w * h;
    EN(img, N * 4);
    CK(cudaMemcpyAsync(ctx->img.p, img, N * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (var) {
        EN(var, N * 4);
        CK(cudaMemcpyAsync(ctx->var.p, var, N * 4, cudaMemcpyHostToDevice, ctx->stream));
    }
    int rc = sexgpu_extract_device(ctx, P<float>(ctx->img), var ? P<float>(ctx->var) : nullptr, w, h, cfg, sum);
    if (rc) return rc;
    return sexgpu_copy_results(ctx, objs, max_objects, nobj, segmap, sub, cd);
}

int sexgpu_stream_submit(sexgpu_ctx *ctx, const float *img, const float *var, int w, int h) {
    if (!ctx || !img || w <= 0 || h <= 0 || (long long)w * h >= (1ll << 31)) return SEXGPU_ERR_ARG;
    if (ctx->qcount >= 2) {
        ctx->err = "two frames are queued already";
        return SEXGPU_ERR_CAPACITY;
    }
    cudaSetDevice(ctx->device);
    if (!ctx->qstream) {
        CK(cudaStreamCreateWithFlags(&ctx->qstream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; i++) CK(cudaEventCreateWithFlags(&ctx->qev[i], cudaEventDisableTiming));
    }
    const int slot = (ctx->qhead + ctx->qcount) & 1;
    const long long N = (long long)w * h;
    EN(qimg[slot], N * 4);
    CK(cudaMemcpyAsync(ctx->qimg[slot].p, img, N * 4, cudaMemcpyHostToDevice, ctx->qstream));
    if (var) {
        EN(qvar[slot], N * 4);
        CK(cudaMemcpyAsync(ctx->qvar[slot].p, var, N * 4, cudaMemcpyHostToDevice, ctx->qstream));
    }
    CK(cudaEventRecord(ctx->qev[slot], ctx->qstream));
    ctx->qw[slot] = w;
    ctx->qh[slot] = h;
    ctx->qhasvar[slot] = var != nullptr;
    ctx->qcount++;
    return SEXGPU_OK;
}

int sexgpu_stream_next(sexgpu_ctx *ctx, const sexgpu_config *cfg, sexgpu_object *objs, int max_objects, int *nobj,
                       sexgpu_summary *sum) {
    if (!ctx || !cfg) return SEXGPU_ERR_ARG;
    if (ctx->qcount == 0) {
        ctx->err = "no frame is queued";
        return SEXGPU_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    const int slot = ctx->qhead;
    ctx->qhead ^= 1;
    ctx->qcount--;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->qev[slot], 0));
    int rc = sexgpu_extract_device(ctx, P<float>(ctx->qimg[slot]),
                                   ctx->qhasvar[slot] ? P<float>(ctx->qvar[slot]) : nullptr, ctx->qw[slot],
                                   ctx->qh[slot], cfg, sum);
    if (rc) return rc;
    return sexgpu_copy_results(ctx, objs, max_objects, nobj, nullptr, nullptr, nullptr);
}

int sexgpu_extract_fits(sexgpu_ctx *ctx, const void *data, const sexgpu_fits_format *fmt, const float *var, int w,
                        int h, const sexgpu_config *cfg, sexgpu_object *objs, int max_objects, int *nobj,
                        int32_t *segmap, float *sub, float *cd, sexgpu_summary *sum) {
    if (!ctx || !data || !fmt || w <= 0 || h <= 0) return SEXGPU_ERR_ARG;
    const int bp = fmt->bitpix;
    if (bp != 8 && bp != 16 && bp != 32 && bp != -32 && bp != -64) {
        ctx->err = "unsupported BITPIX";
        return SEXGPU_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    const long long N = (long long)w * h;
    const size_t bytes = (size_t)N * (size_t)(bp < 0 ? -bp : bp) / 8;
    EN(fitsraw, bytes);
    EN(img, N * 4);
    CK(cudaMemcpyAsync(ctx->fitsraw.p, data, bytes, cudaMemcpyHostToDevice, ctx->stream));
    launch_fits_to_float(ctx->fitsraw.p, bp, fmt->bscale, fmt->bzero, fmt->has_blank, fmt->blank, P<float>(ctx->img),
                         N, ctx->stream);
    if (var) {
        EN(var, N * 4);
        CK(cudaMemcpyAsync(ctx->var.p, var, N * 4, cudaMemcpyHostToDevice, ctx->stream));
    }
    int rc = sexgpu_extract_device(ctx, P<float>(ctx->img), var ? P<float>(ctx->var) : nullptr, w, h, cfg, sum);
    if (rc) return rc;
    return sexgpu_copy_results(ctx, objs, max_objects, nobj, segmap, sub, cd);
}

int sexgpu_background_rms(sexgpu_ctx *ctx, float *rms) {
    if (!ctx || !rms) return SEXGPU_ERR_ARG;
    const PipeState &ps = ctx->ps;
    if (ps.stage < 1 || ps.Pm.w <= 0) {
        ctx->err = "no extraction to take the rms map of";
        return SEXGPU_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const FrameParams &Pm = ps.Pm;
    const int w = Pm.w, h = Pm.h, nb = Pm.nbx * Pm.nby;
    const long long N = (long long)w * h;
    EN(rmsd, (size_t)nb * 4);
    EN(rmsu, std::max((size_t)nb * 4 + 64, (size_t)h * Pm.nbx * 4));  // column spline, then row splines
    EN(rmsnode, (size_t)h * Pm.nbx * 4);
    EN(rmsdnode, (size_t)h * Pm.nbx * 4);
    EN(rmsmap, (size_t)N * 4);
    k_back_spline<<<(Pm.nbx + 127) / 128, 128, 0, st>>>(ps.B.sigma3, P<float>(ctx->rmsd), P<float>(ctx->rmsu), Pm.nbx,
                                                        Pm.nby);
    k_row_nodes<<<(h + 127) / 128, 128, 0, st>>>(ps.B.sigma3, P<float>(ctx->rmsd), Pm.nbx, Pm.nby, Pm.bh, h,
                                                 P<float>(ctx->rmsnode), P<float>(ctx->rmsdnode),
                                                 P<float>(ctx->rmsu));
    k_rms_map<<<grid1(N, 256), 256, 0, st>>>(P<float>(ctx->rmsnode), P<float>(ctx->rmsdnode), ps.B.colk, ps.B.coldx,
                                            Pm.nbx, w, N, P<float>(ctx->rmsmap), 0);
    CK(cudaMemcpyAsync(rms, ctx->rmsmap.p, (size_t)N * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SEXGPU_OK;
}

int sexgpu_copy_apertures(sexgpu_ctx *ctx, float *out, int max_rows, int *nrows, int *naper) {
    if (!ctx || (!out && max_rows > 0)) return SEXGPU_ERR_ARG;
    const PipeState &ps = ctx->ps;
    if (ps.stage != 6) {
        ctx->err = "no finished extraction";
        return SEXGPU_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    const int ns = ps.ns, na = ps.Pm.naper;
    if (nrows) *nrows = ns;
    if (naper) *naper = na;
    if (ns > max_rows) return SEXGPU_ERR_CAPACITY;
    if (ns == 0) return SEXGPU_OK;
    cudaStream_t st = ctx->stream;
    EN(aperrows, (size_t)ns * na * sizeof(float4));
    k_write_apers<<<grid1(ns, 128), 128, 0, st>>>(ctx->O, P<unsigned>(ctx->svals), ns, na,
                                                  P<float4>(ctx->aperrows));
    CK(cudaMemcpyAsync(out, ctx->aperrows.p, (size_t)ns * na * sizeof(float4), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SEXGPU_OK;
}

int sexgpu_background_map(sexgpu_ctx *ctx, float *back) {
    if (!ctx || !back) return SEXGPU_ERR_ARG;
    const PipeState &ps = ctx->ps;
    if (ps.stage < 1 || ps.Pm.w <= 0) {
        ctx->err = "no extraction to take the background map of";
        return SEXGPU_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const FrameParams &Pm = ps.Pm;
    const long long N = (long long)Pm.w * Pm.h;
    EN(rmsmap, (size_t)N * 4);
    k_back_map<<<grid1(N, 256), 256, 0, st>>>(ps.B, Pm.nbx, Pm.back_type, P<FrameScalars>(ctx->sc), Pm.w, N,
                                             P<float>(ctx->rmsmap));
    CK(cudaMemcpyAsync(back, ctx->rmsmap.p, (size_t)N * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SEXGPU_OK;
}

int sexgpu_background(sexgpu_ctx *ctx, float *img, int w, int h, const sexgpu_config *cfg, float *back,
                      float *sigma, sexgpu_summary *sum) {
    if (!ctx || !img || !cfg) return SEXGPU_ERR_ARG;
    int rc = check_config(cfg, w, h);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    FrameParams Pm;
    make_params(cfg, w, h, Pm);
    Pm.filter_flag = 0;
    long long N = (long long)w * h;
    int nb = Pm.nbx * Pm.nby;
    EN(img, N * 4);
    EN(sub, N * 4);
    EN(cd, N * 4);
    EN(lab, N * 4);
    EN(ms, nb * sizeof(MeshStat));
    EN(back, nb * 4);
    EN(sigma, nb * 4);
    EN(back2, nb * 4);
    EN(back3, nb * 4);
    EN(sigma3, nb * 4);
    EN(dback, nb * 4);
    EN(bu, (size_t)nb * 4 + 64);
    EN(rownode, (size_t)h * Pm.nbx * 4);
    EN(rowdnode, (size_t)h * Pm.nbx * 4);
    EN(rowu, (size_t)h * Pm.nbx * 4);
    EN(colk, w * 4);
    EN(coldx, w * 4);
    EN(sc, sizeof(FrameScalars));
    BackBufs B;
    B.ms = P<MeshStat>(ctx->ms);
    B.back = P<float>(ctx->back);
    B.sigma = P<float>(ctx->sigma);
    B.back2 = P<float>(ctx->back2);
    B.back3 = P<float>(ctx->back3);
    B.sigma3 = P<float>(ctx->sigma3);
    B.dback = P<float>(ctx->dback);
    B.u = P<float>(ctx->bu);
    B.rownode = P<float>(ctx->rownode);
    B.rowdnode = P<float>(ctx->rowdnode);
    B.rowu = P<float>(ctx->rowu);
    B.colk = P<int>(ctx->colk);
    B.coldx = P<float>(ctx->coldx);
    column_table(w, Pm.nbx, Pm.bw, ctx->colk_h, ctx->coldx_h);
    CK(cudaMemcpyAsync(B.colk, ctx->colk_h.data(), w * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(B.coldx, ctx->coldx_h.data(), w * 4, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(ctx->img.p, img, N * 4, cudaMemcpyHostToDevice, st));
    rc = load_mask(ctx, nullptr, 1, 1);
    if (rc) return rc;
    FrameScalars *d_sc = P<FrameScalars>(ctx->sc);
    int nl = 0;
    k_init_scalars<<<1, 1, 0, st>>>(d_sc);
    launch_background(B, P<float>(ctx->img), Pm, d_sc, st, nl);
    launch_sub_filter(P<float>(ctx->img), P<float>(ctx->sub), P<float>(ctx->cd), P<int>(ctx->lab), B, Pm, d_sc,
                      nullptr, ctx->cmask, st, nl);
    CK(cudaMemcpyAsync(img, ctx->sub.p, N * 4, cudaMemcpyDeviceToHost, st));
    if (back) CK(cudaMemcpyAsync(back, B.back3, nb * 4, cudaMemcpyDeviceToHost, st));
    if (sigma) CK(cudaMemcpyAsync(sigma, B.sigma3, nb * 4, cudaMemcpyDeviceToHost, st));
    rc = read_scalars(ctx);
    if (rc) return rc;
    if (sum) {
        ctx->last_nobj = ctx->last_ns = 0;
        fill_summary(ctx, Pm, sum);
    }
    return SEXGPU_OK;
}

int sexgpu_filter(sexgpu_ctx *ctx, const float *sub, int w, int h, const float *mask, int mw, int mh, float *cd) {
    if (!ctx || !sub || !mask || !cd || w <= 0 || h <= 0 || mw < 1 || mh < 1 || mw > SX_MAXCONV || mh > SX_MAXCONV)
        return SEXGPU_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    long long N = (long long)w * h;
    EN(img, N * 4);
    EN(sub, N * 4);
    EN(cd, N * 4);
    EN(lab, N * 4);
    EN(sc, sizeof(FrameScalars));
    EN(rownode, 16);
    EN(colk, 16);
    EN(coldx, 16);
    CK(cudaMemcpyAsync(ctx->img.p, sub, N * 4, cudaMemcpyHostToDevice, st));
    int rc = load_mask(ctx, mask, mw, mh);
    if (rc) return rc;
    FrameScalars z;
    memset(&z, 0, sizeof(z));
    z.backmean = 0.0f;
    z.dthresh = 1e30f;
    z.e0sub = 1000;
    CK(cudaMemcpyAsync(ctx->sc.p, &z, sizeof(z), cudaMemcpyHostToDevice, st));
    BackBufs B;
    memset(&B, 0, sizeof(B));
    B.rownode = P<float>(ctx->rownode);
    B.colk = P<int>(ctx->colk);
    B.coldx = P<float>(ctx->coldx);
    FrameParams Pm;
    memset(&Pm, 0, sizeof(Pm));
    Pm.w = w;
    Pm.h = h;
    Pm.nbx = 1;
    Pm.back_type = 1;
    Pm.filter_flag = 1;
    Pm.conv_w = mw;
    Pm.conv_h = mh;
    int nl = 0;
    launch_sub_filter(P<float>(ctx->img), P<float>(ctx->sub), P<float>(ctx->cd), P<int>(ctx->lab), B, Pm,
                      P<FrameScalars>(ctx->sc), nullptr, ctx->cmask, st, nl);
    CK(cudaMemcpyAsync(cd, ctx->cd.p, N * 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    return SEXGPU_OK;
}

// src/filter.c:101-185, restated: header line CONV [NORM|NONORM], rows of
// numbers ('#' starts a comment line), L1 normalisation (variance
// normalisation for zero-sum masks)
int sexgpu_getconv(const char *path, float *mask, int maxn, int *mw, int *mh) {
    if (!path || !mask || !mw || !mh) return SEXGPU_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return SEXGPU_ERR_ARG;
    char line[512];
    if (!fgets(line, sizeof(line), f) || strncmp(line, "CONV", 4)) {
        fclose(f);
        return SEXGPU_ERR_ARG;
    }
    int normflag = strstr(line, "NORM") ? (strstr(line, "NONORM") ? 0 : 1) : 1;
    int n = 0, width = 0;
    while (fgets(line, sizeof(line), f)) {
        int j = 0;
        char *save = nullptr;
        char *tok = strtok_r(line, " \t\n", &save);
        if (!tok || tok[0] == '#') continue;
        do {
            if (n >= maxn) {
                fclose(f);
                return SEXGPU_ERR_CAPACITY;
            }
            mask[n++] = (float)atof(tok);
            j++;
        } while ((tok = strtok_r(nullptr, " \t\n", &save)));
        if (j > width) width = j;
    }
    fclose(f);
    if (width < 1 || n % width) return SEXGPU_ERR_ARG;
    *mw = width;
    *mh = n / width;
    double sum = 0.0, var = 0.0;
    for (int j = 0; j < n; j++) {
        double pix = mask[j];
        sum += fabs(pix);
        var += pix * pix;
    }
    var = sqrt(var);
    if (normflag) {
        if (sum == 0.0) sum = var;
        for (int j = 0; j < n; j++) mask[j] /= sum;
    }
    return n;
}

// host memory that the device can copy from directly (page-locked)
static bool host_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// pinned host buffers of a batch worker grow with headroom; outgrown ones
// are freed after the batch
static bool batch_grow(sexgpu_ctx *wc, void *&buf, size_t &have, size_t need) {
    if (have >= need) return true;
    if (buf) wc->host_graveyard.push_back(buf);
    buf = nullptr;
    have = 0;
    const size_t want = need + need / 4;
    if (cudaHostAlloc(&buf, want, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    have = want;
    return true;
}

// One frame of a batch on worker wc.  The worker copies the frame (and
// weight map) into its own pinned buffer first and brings the catalogue rows
// back through another, so that the transfers of different workers are DMA
// transfers that proceed in parallel instead of queueing on the driver's
// pageable staging.
static void batch_one_frame(sexgpu_ctx *wc, sexgpu_batch_frame &f) {
    f.nobj = 0;
    if (!f.img || !f.cfg || f.w <= 0 || f.h <= 0 || f.max_objects < 0 || (f.max_objects > 0 && !f.objs)) {
        f.status = SEXGPU_ERR_ARG;
        return;
    }
    const size_t bytes = (size_t)f.w * f.h * sizeof(float);
    const float *src = f.img, *wsrc = f.wmap;
    if (host_pinned(f.img) && (!f.wmap || host_pinned(f.wmap))) {
        // already page-locked: uploaded from where it is
    } else if (batch_grow(wc, wc->stage_host, wc->stage_bytes, f.wmap ? 2 * bytes : bytes)) {
        memcpy(wc->stage_host, f.img, bytes);
        src = (const float *)wc->stage_host;
        if (f.wmap) {
            memcpy((char *)wc->stage_host + bytes, f.wmap, bytes);
            wsrc = (const float *)((char *)wc->stage_host + bytes);
        }
    }
    const size_t rbytes = (size_t)f.max_objects * sizeof(sexgpu_object);
    if (!batch_grow(wc, wc->rows_host, wc->rows_bytes, std::min(rbytes, (size_t)1 << 20))) {
        f.status = sexgpu_extract(wc, src, wsrc, f.w, f.h, f.cfg, f.objs, f.max_objects, &f.nobj, nullptr, nullptr,
                                  nullptr, &f.summary);
        return;
    }
    f.status = sexgpu_extract(wc, src, wsrc, f.w, f.h, f.cfg, nullptr, 0, &f.nobj, nullptr, nullptr, nullptr,
                              &f.summary);
    if (f.status) return;
    const int n = std::min(f.nobj, f.max_objects);
    const size_t nb = (size_t)n * sizeof(sexgpu_object);
    if (n > 0 && !batch_grow(wc, wc->rows_host, wc->rows_bytes, nb)) {
        f.status = SEXGPU_ERR_NOMEM;
        return;
    }
    if (n > 0) {
        cudaError_t e = cudaMemcpyAsync(wc->rows_host, wc->rows.p, nb, cudaMemcpyDeviceToHost, wc->stream);
        if (e == cudaSuccess) e = stream_wait(wc, wc->stream);
        if (e != cudaSuccess) {
            f.status = set_err(wc, e, "catalogue copy");
            return;
        }
        memcpy(f.objs, wc->rows_host, nb);
    }
    if (f.nobj > f.max_objects) f.status = SEXGPU_ERR_CAPACITY;
}

// Frame kind of a batch frame (size, configuration, mask, weight map).
static unsigned long long batch_kind(const sexgpu_batch_frame &f) {
    unsigned long long hsh = 1469598103934665603ull;
    auto mix = [&](const void *p, size_t n) {
        for (size_t k = 0; k < n; k++) hsh = (hsh ^ ((const unsigned char *)p)[k]) * 1099511628211ull;
    };
    if (f.cfg && f.w > 0 && f.h > 0) {
        FrameParams Pm;
        make_params(f.cfg, f.w, f.h, Pm);
        mix(&Pm, sizeof(Pm));
        if (f.cfg->filter_flag && f.cfg->conv)
            mix(f.cfg->conv, sizeof(float) * (size_t)std::max(f.cfg->conv_w, 0) * std::max(f.cfg->conv_h, 0));
    }
    const int hasw = f.wmap != nullptr;
    mix(&hasw, sizeof(hasw));
    return hsh;
}

// Frames of each worker with graphs: whole kinds to the least loaded worker
// (largest kinds first, by pixels), a kind larger than a worker's share
// frame by frame; each list largest frame first.  Deterministic, so that a
// batch repeated keeps every kind on the worker that holds its graph.
static std::vector<std::vector<int>> batch_lists(const sexgpu_batch_frame *frames, int n, int workers,
                                                 const std::vector<int> &order,
                                                 const std::vector<unsigned long long> &kind) {
    std::vector<std::vector<int>> wl(workers);
    std::vector<unsigned long long> kinds;
    std::vector<long long> kpix;
    std::vector<std::vector<int>> kfr;
    long long total = 0;
    for (int k = 0; k < n; k++) {
        const int i = order[k];
        const long long px = (long long)std::max(frames[i].w, 0) * std::max(frames[i].h, 0);
        total += px;
        size_t j = std::find(kinds.begin(), kinds.end(), kind[i]) - kinds.begin();
        if (j == kinds.size()) {
            kinds.push_back(kind[i]);
            kpix.push_back(0);
            kfr.emplace_back();
        }
        kpix[j] += px;
        kfr[j].push_back(i);
    }
    std::vector<int> ko(kinds.size());
    for (size_t j = 0; j < ko.size(); j++) ko[j] = (int)j;
    std::stable_sort(ko.begin(), ko.end(), [&](int a, int b) { return kpix[a] > kpix[b]; });
    std::vector<long long> load(workers, 0);
    auto least = [&]() { return (int)(std::min_element(load.begin(), load.end()) - load.begin()); };
    for (int j : ko) {
        if (kpix[j] * workers <= total) {
            const int w = least();
            for (int i : kfr[j]) wl[w].push_back(i);
            load[w] += kpix[j];
        } else {
            for (int i : kfr[j]) {
                const int w = least();
                wl[w].push_back(i);
                load[w] += (long long)frames[i].w * frames[i].h;
            }
        }
    }
    std::vector<int> rank(n);
    for (int k = 0; k < n; k++) rank[order[k]] = k;
    for (auto &l : wl) std::stable_sort(l.begin(), l.end(), [&](int a, int b) { return rank[a] < rank[b]; });
    return wl;
}

static bool batch_graph_valid(const sexgpu_ctx *ctx) {
    const BatchGraph *b = ctx->bgraph;
    if (!b || !b->exec || b->epochs.size() > ctx->workers.size()) return false;
    for (size_t w = 0; w < b->epochs.size(); w++)
        if (ctx->workers[w]->graph_epoch != b->epochs[w] || ctx->workers[w]->gen != b->gens[w]) return false;
    return true;
}

// Builds the one-launch form of a batch whose every frame was just replayed
// from its worker's graph (entry ids per frame).  Failure leaves no batch
// graph: the next batch takes the per-frame path again.
static void build_batch_graph(sexgpu_ctx *ctx, const sexgpu_batch_frame *frames, int n,
                              const std::vector<std::vector<int>> &wl, const std::vector<unsigned long long> &sig,
                              const std::vector<unsigned long long> &entry) {
    free_batch_graph(ctx);
    cudaSetDevice(ctx->device);
    BatchGraph *b = new BatchGraph;
    b->sig = sig;
    b->lists = wl;
    b->in_off.assign(n, 0);
    b->row_off.assign(n, 0);
    b->cap.assign(n, 0);
    b->pm.resize(n);
    b->up_img.assign(n, nullptr);
    b->up_wmap.assign(n, nullptr);
    b->dst_img.assign(n, nullptr);
    b->dst_wmap.assign(n, nullptr);
    std::vector<const GraphEntry *> ent(n, nullptr);
    size_t in = 0, rows = 0;
    const size_t S = sizeof(sexgpu_object);
    bool ok = true;
    for (size_t w = 0; w < wl.size() && ok; w++) {
        const sexgpu_ctx *wc = ctx->workers[w];
        b->epochs.push_back(wc->graph_epoch);
        b->gens.push_back(wc->gen);
        for (int i : wl[w]) {
            for (const GraphEntry &e : wc->graphs)
                if (e.id == entry[i] && e.graph && e.exec && e.gen == wc->gen) ent[i] = &e;
            if (!ent[i]) {
                ok = false;
                break;
            }
            b->cap[i] = ent[i]->cap_obj;
            b->pm[i] = ent[i]->Pm;
            const size_t bytes = (size_t)frames[i].w * frames[i].h * sizeof(float) * (frames[i].wmap ? 2 : 1);
            b->in_off[i] = in;
            in += (bytes + 255) & ~(size_t)255;
            b->row_off[i] = rows;
            rows += (size_t)b->cap[i] + 1;
        }
    }
    b->in_bytes = in;
    b->rows_total = rows;
    ok = ok && cudaHostAlloc((void **)&b->in_host, std::max(in, (size_t)256), cudaHostAllocPortable) == cudaSuccess &&
         cudaMalloc(&b->rows_dev, rows * S) == cudaSuccess &&
         cudaMalloc(&b->sc_dev, (size_t)n * sizeof(FrameScalars)) == cudaSuccess &&
         cudaHostAlloc((void **)&b->sc_host, (size_t)n * sizeof(FrameScalars), cudaHostAllocPortable) == cudaSuccess &&
         cudaHostAlloc((void **)&b->rows_host, rows * S, cudaHostAllocPortable) == cudaSuccess;
    cudaGraph_t g = nullptr;
    ok = ok && cudaGraphCreate(&g, 0) == cudaSuccess;
    std::vector<cudaGraphNode_t> tails;
    for (size_t w = 0; w < wl.size() && ok; w++) {
        sexgpu_ctx *wc = ctx->workers[w];
        cudaGraphNode_t prev = nullptr;
        for (int i : wl[w]) {
            const size_t bytes = (size_t)frames[i].w * frames[i].h * sizeof(float);
            cudaGraphNode_t in1 = nullptr, in2 = nullptr, child = nullptr, r = nullptr, sc = nullptr, join = nullptr;
            ok = ok && cudaGraphAddMemcpyNode1D(&in1, g, prev ? &prev : nullptr, prev ? 1 : 0, wc->img.p,
                                                b->in_host + b->in_off[i], bytes, cudaMemcpyHostToDevice) ==
                           cudaSuccess;
            std::vector<cudaGraphNode_t> deps{in1};
            if (ok && frames[i].wmap) {
                ok = cudaGraphAddMemcpyNode1D(&in2, g, prev ? &prev : nullptr, prev ? 1 : 0, wc->var.p,
                                              b->in_host + b->in_off[i] + bytes, bytes, cudaMemcpyHostToDevice) ==
                     cudaSuccess;
                deps.push_back(in2);
            }
            b->up_img[i] = in1;
            b->up_wmap[i] = in2;
            b->dst_img[i] = wc->img.p;
            b->dst_wmap[i] = wc->var.p;
            ok = ok && cudaGraphAddChildGraphNode(&child, g, deps.data(), deps.size(), ent[i]->graph) == cudaSuccess;
            ok = ok && cudaGraphAddMemcpyNode1D(&r, g, &child, 1, (char *)b->rows_dev + b->row_off[i] * S,
                                                wc->rows.p, ((size_t)b->cap[i] + 1) * S,
                                                cudaMemcpyDeviceToDevice) == cudaSuccess;
            ok = ok && cudaGraphAddMemcpyNode1D(&sc, g, &child, 1, (char *)b->sc_dev + (size_t)i * sizeof(FrameScalars),
                                                wc->sc.p, sizeof(FrameScalars), cudaMemcpyDeviceToDevice) ==
                           cudaSuccess;
            cudaGraphNode_t two[2] = {r, sc};
            ok = ok && cudaGraphAddEmptyNode(&join, g, two, 2) == cudaSuccess;
            prev = join;
            if (ok) b->kernels += ent[i]->kernels;
        }
        if (prev) tails.push_back(prev);
    }
    cudaGraphNode_t out = nullptr;
    ok = ok && cudaGraphAddMemcpyNode1D(&out, g, tails.data(), tails.size(), b->sc_host, b->sc_dev,
                                        (size_t)n * sizeof(FrameScalars), cudaMemcpyDeviceToHost) == cudaSuccess;
    ok = ok && cudaGraphInstantiate(&b->exec, g, 0) == cudaSuccess;
    b->graph = g;
    ctx->bgraph = b;
    if (!ok) {
        cudaGetLastError();
        free_batch_graph(ctx);
    }
}

// The batch as one graph launch.  Returns SEXGPU_OK or a frame's error;
// frames whose counts exceeded their graph's capacities are extracted again
// by their workers, and the batch graph is dropped (its capacities grew).
static int batch_launch(sexgpu_ctx *ctx, sexgpu_batch_frame *frames, int n) {
    BatchGraph *b = ctx->bgraph;
    cudaStream_t st = ctx->stream;
    const size_t S = sizeof(sexgpu_object);
    // frames in pinned host memory are uploaded from where they are; the
    // others are copied into the batch's pinned input first, one host thread
    // per worker list
    std::vector<const void *> src(n, nullptr), wsrc(n, nullptr);
    {
        auto stage = [&](size_t w) {
            for (int i : b->lists[w]) {
                const sexgpu_batch_frame &f = frames[i];
                const size_t bytes = (size_t)f.w * f.h * sizeof(float);
                src[i] = f.img;
                wsrc[i] = f.wmap;
                if (!host_pinned(f.img)) {
                    memcpy(b->in_host + b->in_off[i], f.img, bytes);
                    src[i] = b->in_host + b->in_off[i];
                }
                if (f.wmap && !host_pinned(f.wmap)) {
                    memcpy(b->in_host + b->in_off[i] + bytes, f.wmap, bytes);
                    wsrc[i] = b->in_host + b->in_off[i] + bytes;
                }
            }
        };
        std::vector<std::thread> pool;
        for (size_t w = 1; w < b->lists.size(); w++) pool.emplace_back(stage, w);
        stage(0);
        for (auto &t : pool) t.join();
    }
    for (int i = 0; i < n; i++) {
        const size_t bytes = (size_t)frames[i].w * frames[i].h * sizeof(float);
        CK(cudaGraphExecMemcpyNodeSetParams1D(b->exec, b->up_img[i], b->dst_img[i], src[i], bytes,
                                              cudaMemcpyHostToDevice));
        if (frames[i].wmap)
            CK(cudaGraphExecMemcpyNodeSetParams1D(b->exec, b->up_wmap[i], b->dst_wmap[i], wsrc[i], bytes,
                                                  cudaMemcpyHostToDevice));
    }
    CK(cudaGraphLaunch(b->exec, st));
    CK(stream_wait(ctx, st));
    std::vector<int> again;
    for (int i = 0; i < n; i++) {
        sexgpu_batch_frame &f = frames[i];
        const FrameScalars &sc = b->sc_host[i];
        const int rc = scalars_status(sc);
        f.nobj = 0;
        f.status = rc;
        if (rc == 1) {
            again.push_back(i);
            continue;
        }
        if (rc) continue;
        f.nobj = sc.nsurv;
        summary_from_scalars(sc, b->pm[i], &f.summary);
        const int k = std::min(f.nobj, f.max_objects);
        if (k > 0 && f.objs)
            CK(cudaMemcpyAsync(b->rows_host + b->row_off[i] * S, (char *)b->rows_dev + b->row_off[i] * S, (size_t)k * S,
                               cudaMemcpyDeviceToHost, st));
    }
    CK(stream_wait(ctx, st));
    for (int i = 0; i < n; i++) {
        sexgpu_batch_frame &f = frames[i];
        if (f.status) continue;
        const int k = std::min(f.nobj, f.max_objects);
        if (k > 0 && f.objs) memcpy(f.objs, b->rows_host + b->row_off[i] * S, (size_t)k * S);
        if (f.nobj > f.max_objects) f.status = SEXGPU_ERR_CAPACITY;
    }
    ctx->last_graph = 1;
    ctx->last_kernels = b->kernels;
    if (!again.empty()) {
        for (size_t w = 0; w < b->lists.size(); w++)
            for (int i : b->lists[w])
                if (std::find(again.begin(), again.end(), i) != again.end()) batch_one_frame(ctx->workers[w], frames[i]);
        free_batch_graph(ctx);
    }
    for (int i = 0; i < n; i++)
        if (frames[i].status != SEXGPU_OK) {
            ctx->err = "frame " + std::to_string(i) + " failed";
            return frames[i].status;
        }
    return SEXGPU_OK;
}

int sexgpu_extract_batch(sexgpu_ctx *ctx, sexgpu_batch_frame *frames, int nframes, int workers) {
    if (!ctx || nframes < 0 || (nframes > 0 && !frames) || workers < 0) return SEXGPU_ERR_ARG;
    if (nframes == 0) return SEXGPU_OK;
    if (workers == 0) workers = ctx->batch_workers;
    workers = std::min(workers, nframes);
    while ((int)ctx->workers.size() < workers) {
        sexgpu_ctx *w = nullptr;
        int rc = sexgpu_create(&w, ctx->device);
        if (rc) {
            ctx->err = "cannot create a batch worker context";
            return rc;
        }
        ctx->workers.push_back(w);
    }
    for (sexgpu_ctx *w : ctx->workers) {
        w->kron_warp_max = ctx->kron_warp_max;
        w->nnw_dev = ctx->nnw_dev;
        w->sync_block = ctx->batch_sync;
        w->defer_free = true;
        w->graph_mode = ctx->graph_mode;
    }
    ctx->last_graph = 0;
    ctx->last_kernels = 0;
    // largest frames first, so that the last frames to start are short
    std::vector<int> order(nframes);
    for (int i = 0; i < nframes; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)frames[a].w * frames[a].h > (long long)frames[b].w * frames[b].h;
    });
    const int div = ctx->batch_grid_div > 0 ? ctx->batch_grid_div : 1;
    // With graphs: fixed lists per worker, so that each kind stays with the
    // worker that holds its graph; a batch repeated after one whose every
    // frame replayed a graph is a single launch of the batch graph.
    std::vector<std::vector<int>> wl;
    std::vector<unsigned long long> sig, kind(nframes, 0), entry(nframes, 0);
    std::vector<char> replayed(nframes, 0);
    if (ctx->graph_mode) {
        bool args_ok = true;
        for (int i = 0; i < nframes; i++) {
            const sexgpu_batch_frame &f = frames[i];
            kind[i] = batch_kind(f);
            args_ok = args_ok && f.img && f.cfg && f.w > 0 && f.h > 0 && f.max_objects >= 0 &&
                      (f.max_objects == 0 || f.objs);
        }
        wl = batch_lists(frames, nframes, workers, order, kind);
        for (int w = 0; w < workers; w++)
            for (int i : wl[w]) {
                sig.push_back(kind[i]);
                sig.push_back(((unsigned long long)frames[i].w << 32) | (unsigned)frames[i].h);
                sig.push_back(((unsigned long long)w << 32) | (unsigned)i | (frames[i].wmap ? 1ull << 31 : 0ull));
            }
        sig.push_back((unsigned long long)div);
        if (args_ok && ctx->batch_one_launch && ctx->bgraph && ctx->bgraph->sig == sig && batch_graph_valid(ctx))
            return batch_launch(ctx, frames, nframes);
    }
    std::atomic<int> next(0);
    std::vector<size_t> cursor(workers, 0);
    auto run = [&](int wi) {
        sexgpu_ctx *wc = ctx->workers[wi];
        cudaSetDevice(wc->device);
        sx_grid_div = div;
        for (;;) {
            int fi;
            if (ctx->graph_mode) {
                if (cursor[wi] >= wl[wi].size()) break;
                fi = wl[wi][cursor[wi]++];
            } else {
                const int k = next.fetch_add(1);
                if (k >= nframes) break;
                fi = order[k];
            }
            batch_one_frame(wc, frames[fi]);
            replayed[fi] = (char)wc->last_graph;
            entry[fi] = wc->last_entry;
        }
    };
    std::vector<std::thread> pool;
    for (int i = 1; i < workers; i++) pool.emplace_back(run, i);
    run(0);
    for (auto &t : pool) t.join();
    sx_grid_div = 1;
    for (sexgpu_ctx *w : ctx->workers) {
        w->defer_free = false;
        for (void *p : w->graveyard) cudaFree(p);
        for (void *p : w->host_graveyard) cudaFreeHost(p);
        w->graveyard.clear();
        w->host_graveyard.clear();
    }
    bool all_ok = true, all_replayed = true;
    for (int i = 0; i < nframes; i++) {
        all_ok = all_ok && frames[i].status == SEXGPU_OK;
        all_replayed = all_replayed && replayed[i];
    }
    if (ctx->graph_mode && ctx->batch_one_launch && all_ok && all_replayed)
        build_batch_graph(ctx, frames, nframes, wl, sig, entry);
    for (int i = 0; i < nframes; i++)
        if (frames[i].status != SEXGPU_OK) {
            ctx->err = "frame " + std::to_string(i) + " failed";
            return frames[i].status;
        }
    return SEXGPU_OK;
}

int sexgpu_set_nnw(sexgpu_ctx *ctx, const sexgpu_nnw *net) {
    if (!ctx) return SEXGPU_ERR_ARG;
    if (!net) {
        ctx->nnw_dev = nullptr;
        return SEXGPU_OK;
    }
    if (net->nlayers < 2 || net->nlayers > SEXGPU_NNW_LAYERS || net->nn[0] != 10) return SEXGPU_ERR_ARG;
    for (int l = 0; l < net->nlayers; l++)
        if (net->nn[l] < 1 || net->nn[l] > SEXGPU_NNW_NEURONS) return SEXGPU_ERR_ARG;
    cudaSetDevice(ctx->device);
    int rc = ensure(ctx, ctx->dnnw, sizeof(sexgpu_nnw));
    if (rc) return rc;
    CK(cudaMemcpy(ctx->dnnw.p, net, sizeof(sexgpu_nnw), cudaMemcpyHostToDevice));
    ctx->nnw_dev = P<sexgpu_nnw>(ctx->dnnw);
    return SEXGPU_OK;
}

// the .nnw format (src/neurro.c getnnw): a first line starting with NNW;
// then, skipping blank and '#' lines: the layer count and the neurons per
// layer; the input biases; the input scales; for every layer l and every
// neuron j of layer l + 1 one line with the nn[l] weights into j and j's
// bias; the output biases; the output scales
int sexgpu_read_nnw(const char *path, sexgpu_nnw *net) {
    if (!path || !net) return SEXGPU_ERR_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return SEXGPU_ERR_ARG;
    memset(net, 0, sizeof(*net));
    char line[8192];
    const int rc = SEXGPU_ERR_ARG;
    if (!fgets(line, sizeof line, f) || strncmp(line, "NNW", 3)) {
        fclose(f);
        return rc;
    }
    std::vector<std::vector<double>> rows;
    while (fgets(line, sizeof line, f)) {
        const char *p = line + strspn(line, " \t");
        if (*p == '#' || *p == '\n' || *p == '\r' || !*p) continue;
        std::vector<double> v;
        char *end;
        for (;;) {
            const double d = strtod(p, &end);
            if (end == p) break;
            v.push_back(d);
            p = end;
        }
        if (!v.empty()) rows.push_back(v);
    }
    fclose(f);
    if (rows.empty()) return rc;
    const int nl = (int)rows[0][0];
    if (nl < 2 || nl > SEXGPU_NNW_LAYERS || (int)rows[0].size() < nl + 1) return rc;
    net->nlayers = nl;
    for (int l = 0; l < nl; l++) {
        net->nn[l] = (int)rows[0][l + 1];
        if (net->nn[l] < 1 || net->nn[l] > SEXGPU_NNW_NEURONS) return rc;
    }
    size_t r = 1;
    auto take = [&](double *dst, int n) {
        if (r >= rows.size() || (int)rows[r].size() < n) return false;
        for (int i = 0; i < n; i++) dst[i] = rows[r][i];
        r++;
        return true;
    };
    if (!take(net->inbias, net->nn[0]) || !take(net->inscale, net->nn[0])) return rc;
    for (int l = 0; l < nl - 1; l++)
        for (int j = 0; j < net->nn[l + 1]; j++) {
            if (r >= rows.size() || (int)rows[r].size() < net->nn[l] + 1) return rc;
            for (int i = 0; i < net->nn[l]; i++) net->w[l][i][j] = rows[r][i];
            net->b[l][j] = rows[r][net->nn[l]];
            r++;
        }
    if (!take(net->outbias, net->nn[nl - 1]) || !take(net->outscale, net->nn[nl - 1])) return rc;
    return SEXGPU_OK;
}

int sexgpu_set_param(sexgpu_ctx *ctx, const char *name, int value) {
    if (!ctx || !name) return SEXGPU_ERR_ARG;
    if (!strcmp(name, "batch_grid_div")) {
        if (value < 0) return SEXGPU_ERR_ARG;
        ctx->batch_grid_div = value;
        return SEXGPU_OK;
    }
    if (!strcmp(name, "batch_sync")) {
        if (value < 0 || value > 1) return SEXGPU_ERR_ARG;
        ctx->batch_sync = value;
        return SEXGPU_OK;
    }
    if (!strcmp(name, "kron_warp_max")) {
        if (value < 1) return SEXGPU_ERR_ARG;
        ctx->kron_warp_max = value;
        return SEXGPU_OK;
    }
    if (!strcmp(name, "batch_workers")) {
        if (value < 1 || value > 64) return SEXGPU_ERR_ARG;
        ctx->batch_workers = value;
        return SEXGPU_OK;
    }
    if (!strcmp(name, "batch_one_launch")) {
        if (value < 0 || value > 1) return SEXGPU_ERR_ARG;
        ctx->batch_one_launch = value;
        return SEXGPU_OK;
    }
    if (!strcmp(name, "graph")) {
        if (value < 0 || value > 1) return SEXGPU_ERR_ARG;
        ctx->graph_mode = value;
        return SEXGPU_OK;
    }
    if (!strcmp(name, "loop_cap")) {
        if (value < 0) return SEXGPU_ERR_ARG;
        ctx->loop_cap = value;
        return SEXGPU_OK;
    }
    ctx->err = std::string("unknown parameter ") + name;
    return SEXGPU_ERR_ARG;
}

static void tune_entry(std::vector<sexgpu_tune_entry> &out, const char *name, int value, float ms) {
    sexgpu_tune_entry e;
    memset(&e, 0, sizeof(e));
    strncpy(e.param, name, sizeof(e.param) - 1);
    e.value = value;
    e.ms = ms;
    out.push_back(e);
}

static int tune_copy_out(const std::vector<sexgpu_tune_entry> &out, sexgpu_tune_entry *entries, int max_entries) {
    if (entries)
        for (int i = 0; i < (int)out.size() && i < max_entries; i++) entries[i] = out[i];
    return (int)out.size();
}

int sexgpu_autotune(sexgpu_ctx *ctx, const float *d_img, const float *d_wmap, int w, int h,
                    const sexgpu_config *cfg, int reps, sexgpu_tune_entry *entries, int max_entries) {
    if (!ctx || !d_img || !cfg || reps < 1 || max_entries < 0) return SEXGPU_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    std::vector<sexgpu_tune_entry> out;
    std::vector<unsigned char> ref, got;
    bool have_ref = false;
    // one candidate: warm-up runs, then the best of reps timed runs; the rows
    // of its last run against the first candidate's
    auto trial = [&](const char *name, int value, float &best) -> int {
        int rc = sexgpu_set_param(ctx, name, value);
        for (int i = 0; !rc && i < 3; i++) rc = sexgpu_extract_device(ctx, d_img, d_wmap, w, h, cfg, nullptr);
        best = 3.0e38f;
        for (int i = 0; !rc && i < reps; i++) {
            cudaEventRecord(e0, st);
            rc = sexgpu_extract_device(ctx, d_img, d_wmap, w, h, cfg, nullptr);
            cudaEventRecord(e1, st);
            if (!rc && cudaEventSynchronize(e1) == cudaSuccess) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                best = std::min(best, ms);
            }
        }
        if (rc) return rc;
        got.resize((size_t)ctx->last_ns * sizeof(sexgpu_object));
        if (!got.empty())
            CK(cudaMemcpyAsync(got.data(), ctx->rows.p, got.size(), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (!have_ref) {
            ref = got;
            have_ref = true;
        } else if (got != ref) {
            ctx->err = std::string("rows differ under ") + name;
            return SEXGPU_ERR_MISMATCH;
        }
        tune_entry(out, name, value, best);
        return SEXGPU_OK;
    };
    int rc = SEXGPU_OK;
    float best_ms = 3.0e38f, ms = 0.f;
    int best_graph = ctx->graph_mode, best_kron = ctx->kron_warp_max;
    for (int g = 0; g <= 1 && !rc; g++) {
        rc = trial("graph", g, ms);
        if (!rc && ms < best_ms) {
            best_ms = ms;
            best_graph = g;
        }
    }
    if (!rc) rc = sexgpu_set_param(ctx, "graph", best_graph);
    best_ms = 3.0e38f;
    for (int v = 1024; v <= 32768 && !rc; v *= 2) {
        rc = trial("kron_warp_max", v, ms);
        if (!rc && ms < best_ms) {
            best_ms = ms;
            best_kron = v;
        }
    }
    if (!rc) rc = sexgpu_set_param(ctx, "kron_warp_max", best_kron);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    return tune_copy_out(out, entries, max_entries);
}

int sexgpu_autotune_batch(sexgpu_ctx *ctx, sexgpu_batch_frame *frames, int nframes, int reps,
                          sexgpu_tune_entry *entries, int max_entries) {
    if (!ctx || nframes <= 0 || !frames || reps < 1 || max_entries < 0) return SEXGPU_ERR_ARG;
    std::vector<sexgpu_tune_entry> out;
    std::vector<std::vector<unsigned char>> ref(nframes);
    bool have_ref = false;
    auto trial = [&](const char *name, int value, int workers, float &best) -> int {
        int rc = SEXGPU_OK;
        if (!strcmp(name, "batch_grid_div")) rc = sexgpu_set_param(ctx, name, value);
        if (!rc) rc = sexgpu_extract_batch(ctx, frames, nframes, workers);  // warm-up
        best = 3.0e38f;
        for (int i = 0; !rc && i < reps; i++) {
            auto t0 = std::chrono::steady_clock::now();
            rc = sexgpu_extract_batch(ctx, frames, nframes, workers);
            auto t1 = std::chrono::steady_clock::now();
            best = std::min(best, (float)std::chrono::duration<double, std::milli>(t1 - t0).count());
        }
        if (rc) return rc;
        for (int i = 0; i < nframes; i++) {
            const sexgpu_batch_frame &f = frames[i];
            const size_t n = f.objs ? (size_t)std::min(f.nobj, f.max_objects) * sizeof(sexgpu_object) : 0;
            std::vector<unsigned char> cur(sizeof(int32_t) + n);
            memcpy(cur.data(), &f.nobj, sizeof(int32_t));
            if (n) memcpy(cur.data() + sizeof(int32_t), f.objs, n);
            if (!have_ref)
                ref[i].swap(cur);
            else if (cur != ref[i]) {
                ctx->err = std::string("catalogues differ under ") + name;
                return SEXGPU_ERR_MISMATCH;
            }
        }
        have_ref = true;
        tune_entry(out, name, value, best);
        return SEXGPU_OK;
    };
    int rc = SEXGPU_OK, best_w = ctx->batch_workers, best_div = ctx->batch_grid_div;
    float best_ms = 3.0e38f, ms = 0.f;
    for (int wk = 4; wk <= 16 && !rc; wk += 4) {
        rc = trial("batch_workers", wk, wk, ms);
        if (!rc && ms < best_ms) {
            best_ms = ms;
            best_w = wk;
        }
    }
    if (!rc) ctx->batch_workers = best_w;
    best_ms = 3.0e38f;
    for (int d = 1; d <= 4 && !rc; d *= 2) {
        rc = trial("batch_grid_div", d, best_w, ms);
        if (!rc && ms < best_ms) {
            best_ms = ms;
            best_div = d;
        }
    }
    if (!rc) rc = sexgpu_set_param(ctx, "batch_grid_div", best_div);
    if (!rc && ctx->graph_mode) {
        int best_one = ctx->batch_one_launch;
        best_ms = 3.0e38f;
        for (int v = 0; v <= 1 && !rc; v++) {
            rc = sexgpu_set_param(ctx, "batch_one_launch", v);
            // two more warm-up batches: the batch graph is built after a
            // batch whose every frame replayed its graph
            for (int k = 0; k < 2 && !rc; k++) rc = sexgpu_extract_batch(ctx, frames, nframes, best_w);
            if (!rc) rc = trial("batch_one_launch", v, best_w, ms);
            if (!rc && ms < best_ms) {
                best_ms = ms;
                best_one = v;
            }
        }
        if (!rc) rc = sexgpu_set_param(ctx, "batch_one_launch", best_one);
    }
    if (rc) return rc;
    return tune_copy_out(out, entries, max_entries);
}

int sexgpu_graph_stats(sexgpu_ctx *ctx, int *replayed, int *kernels, int *kinds) {
    if (!ctx) return SEXGPU_ERR_ARG;
    if (replayed) *replayed = ctx->last_graph;
    if (kernels) *kernels = ctx->last_kernels;
    if (kinds) {
        int n = 0;
        for (const GraphEntry &e : ctx->graphs) n += e.exec != nullptr;
        *kinds = n;
    }
    return SEXGPU_OK;
}

int sexgpu_stage_times(sexgpu_ctx *ctx, sexgpu_stage *stages, int max) {
    if (!ctx) return SEXGPU_ERR_ARG;
    int n = (int)ctx->stage_ms.size();
    for (int i = 0; i < n && i < max; i++) {
        memset(&stages[i], 0, sizeof(stages[i]));
        strncpy(stages[i].name, ctx->stage_names[i].c_str(), sizeof(stages[i].name) - 1);
        stages[i].launches = ctx->stage_launches[i];
        stages[i].ms = ctx->stage_ms[i];
    }
    return n;
}

}  // extern "C"

// background estimation without device allocation (fixed scratch array)
#include "noalloc.cu"
