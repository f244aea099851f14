// kernels.cuh -- buffers and launchers shared by the stages of libsexgpu.
#pragma once
#include <atomic>
#include "common.cuh"

namespace sx {

struct MeshStat {
    float mean, sigma, lcut, hcut, qzero, qscale;
    int nlevels, npix;
};

struct BackBufs {
    MeshStat *ms;
    float *back, *sigma, *back2, *back3, *sigma3, *dback, *u;
    float *rownode, *rowdnode, *rowu;   // h x nbx each
    int *colk;                          // w
    float *coldx;                       // w
};

// per-root data (index = root id, first-pixel order)
struct RootBufs {
    int *size, *off, *first;            // pixels, offset in the root pixel list, first pixel
    int *ymax, *lastx;                  // completion-order keys
    float *fdpeak, *fdflux;
    int *nkept, *objbase;
    float *dthresh, *thresh;            // smallest detection / analysis threshold of its pixels
};

// per-element scratch of the deblending (index = position in the root pixel list)
struct DebBufs {
    int *par, *lev, *sz, *order, *rl0, *rl1, *nid0, *nid1;
    unsigned long long *acc;            // 4 limbs per element
    int *nd_root0, *nd_root1, *nd_flag0, *nd_flag1, *nd_nson0, *nd_nson1, *nd_okc0, *nd_okc1;
    int *nd_oka0, *nd_oka1;
    unsigned long long *kept;           // packed (level << 32) | element, per root at its offset
    int *own, *kl, *kidx;
    int *pint;                          // xmin, xmax, ymin, ymax, peak(ord), cpeak(ord), dnpix, area2
    unsigned char *arena;               // 48 B per element: the compact per-object state of k_dl_*
    int *rec;                           // merge record per element (k_dl_sweep -> k_dl_assign)
};

// Persistent grids (deblending classes, subtract/filter tiles) are sized to
// the resident capacity divided by this (set per host thread; 1 by default,
// the batch workers take the "batch_grid_div" parameter of their context:
// measured on the 64-frame batch, whole-GPU grids with 8 workers were the
// fastest).
extern thread_local int sx_grid_div;
inline int sx_share(int grid) { return sx_grid_div > 1 ? (grid + sx_grid_div - 1) / sx_grid_div : grid; }

// A value per device computed on first use (resident grid sizes, device
// attributes), for the current device.  Several host threads (batch workers)
// may ask at once: the slots are atomic, and a value computed twice is
// computed the same way; 0 means "not computed yet".
struct DevCache {
    std::atomic<int> v[64];
    template <class F> int get(F compute) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64) return compute(dev);
        int x = v[dev].load(std::memory_order_relaxed);
        if (x == 0) {
            x = compute(dev);
            v[dev].store(x, std::memory_order_relaxed);
        }
        return x;
    }
};

// Kron boxes too large for one warp, summed by whole CTAs (k_post.cu)
constexpr int KR_CHUNK = 8192;     // box pixels per CTA work item
constexpr int KR_THREADS = 256;
constexpr int KR_GRID = 2 * 148;
constexpr int KR_ITEMS = 8192;     // queued boxes per pass
constexpr int KR_CHUNKS = 65536;   // work items per pass (2^29 box pixels)
constexpr int KR_WARP_MAX = 8192;  // default: larger boxes are queued

struct KronGeo {
    float cx2, cy2, cxy, klim2;
    int xmin, xmax, ymin, ymax;
};
struct KronItem {
    int o, flags, c0, nch;  // object, FLAGS so far, first work item, items (-1: summed by its warp)
    float kron;
    KronGeo g;
};
struct KronAcc;
struct KronBufs {
    KronItem *item[2];
    int *chunk[2];    // work item -> queued box
    KronAcc *part[2]; // work item -> partial sums
    int icap, ccap, warp_max;
};

// per-object data (index = object id: root order, then (level, label))
struct ObjBufs {
    int *root, *level, *n, *off;
    int *xmin, *xmax, *ymin, *ymax, *dnpix, *flags, *singu;
    float *fdflux, *dflux, *fdpeak, *dpeak, *node_dthresh;
    double *mx, *my, *mx2, *my2, *mxy;
    float *a, *b, *theta, *abcor, *cxx, *cyy, *cxy;
    int *npix, *peakx, *peaky, *iso;    // iso: 8 per object
    float *flux, *fluxerr, *peak, *bkg, *mthresh, *fwhm;
    double *pmx2, *pmy2, *pmxy;
    int *master, *fmaster, *number;
    float *flux_isocor, *fluxerr_isocor, *flux_aper, *fluxerr_aper, *mag_aper, *magerr_aper;
    float *kron, *flux_auto, *fluxerr_auto, *mag_auto, *magerr_auto;
    float *mag_iso, *magerr_iso, *fluxerr_iso;
    int *fdnpix;
    float *dthr, *athr;                 // the raw object's detection / analysis thresholds
    float *sprob;                       // CLASS_STAR
    float *dbkg;                        // LOCAL photometry background per object, or null (GLOBAL)
    MeshStat *lstat;                    // LOCAL annulus statistics
    unsigned long long *sortkey;
    float4 *aper;                       // every aperture: (flux, error, mag, mag error), naper per object
};

void launch_background(BackBufs &B, const float *img, const FrameParams &P, FrameScalars *d_sc, cudaStream_t st,
                       int &launches);
void launch_weight_mask(const float *img, const float *wmap, int wtype, float *imgm, long long n, cudaStream_t st);
void launch_weight_var(const BackBufs &B, const float *wmap, const FrameParams &P, float *ratio, float *wvar,
                       FrameScalars *d_sc, cudaStream_t st);

// The detection mask of one extraction: row-major mw x mh values on the
// device and on the host (per context, so that contexts extracting at the
// same time with different masks do not share it).
struct ConvMask {
    const float *dev;
    const float *host;
    int mw, mh;
};

bool launch_sub_filter(const float *img, float *sub, float *cd, int *lab, const BackBufs &B,
                       const FrameParams &P, FrameScalars *d_sc, const float *d_var, const ConvMask &M,
                       cudaStream_t st, int &launches);

void launch_ccl(int *lab, int *cnt, const FrameParams &P, FrameScalars *d_sc, cudaStream_t st, int &launches,
                bool tiled);

struct DebArgs {
    const float *cd, *sub;
    const int *pos2idx;
    const unsigned *rpix;       // root pixel lists (raster order per root)
    RootBufs R;
    DebBufs D;
    ObjBufs O;
    FrameScalars *sc;
    int *alloc;                 // W*H object id map (-1 elsewhere)
    unsigned *objkey;           // object id per root-list element
    int w, h, N, debminarea;
    FastDiv wdiv;
    double mincont;
    int loop_cap;               // > 0: cap on union-find walks (failure tests); 0: the object's size
};

// the main stream, the side streams and the events that fork and join them
constexpr int DL_SIDE = 3;
struct DebStreams {
    cudaStream_t main, side[DL_SIDE];
    cudaEvent_t fork, join[DL_SIDE];
};

void launch_deblend_split(const int *size, int nroots, const int *nroots_dev, int *lists, int *counts,
                          unsigned *keys, unsigned *vals, unsigned *kalt, unsigned *valt, int *tmp, cudaStream_t st);
int deblend_split_launches(int nroots);
void launch_deblend_sweep(const DebArgs &A, const int *lists, int *counts, int nroots, const DebStreams &S);
void launch_deblend_assign(const DebArgs &A, const int *lists, int *counts, int nroots, const DebStreams &S);

}  // namespace sx
