// k_detect.cu -- background subtraction fused with the detection filter and
// the threshold, then 8-connected component labelling.
//
// Reference: src/back.c:863-899 (subbackline, x interpolation),
// src/filter.c:39-95 (convolve), src/cuda/cudadetection.cu:36-276
// (threshold + CCL).  The CCL here is a union-find over the label image
// (tile-local union in shared memory, then unions across tile borders with
// atomicMin, then path flattening); every component ends labelled with its
// smallest linear pixel index, the label the reference's iterative
// propagation converges to.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "kernels.cuh"

namespace sx {

// mask taps of the size-specialised kernels, passed by value (constant bank)
struct ConvTaps {
    float m[121];
};

constexpr int SF_TW = 32;   // output tile width
constexpr int SF_TH = 16;   // output tile height
constexpr int SF_TX = 32, SF_TY = 8;

// background at (x, y) from the per-row node splines (src/back.c:863-899)
__device__ __forceinline__ float bkg_at(int x, int y, const BackBufs &B, int nbx, int back_type, float backmean) {
    if (back_type == 1) return backmean;
    const float *nd = B.rownode + (size_t)y * nbx;
    if (nbx <= 1) return nd[0];
    const float *dnd = B.rowdnode + (size_t)y * nbx;
    int k = B.colk[x];
    float dx = B.coldx[x];
    float cdx = 1 - dx;
    return (float)(cdx * (nd[k] + (cdx * cdx - 1) * dnd[k]) + dx * (nd[k + 1] + (dx * dx - 1) * dnd[k + 1]));
}

__global__ void __launch_bounds__(SF_TX *SF_TY) k_sub_filter(const float *__restrict__ img, float *__restrict__ sub,
                                                              float *__restrict__ cd, int *__restrict__ lab,
                                                              BackBufs B, int w, int h, int nbx, int back_type,
                                                              const float *__restrict__ mask, int mw, int mh,
                                                              const float *__restrict__ wvar, int wthr, double dfac,
                                                              FrameScalars *sc) {
    extern __shared__ float tile[];
    const int rx = mw / 2, ry = mh / 2;
    const int TWp = SF_TW + mw - 1, THp = SF_TH + mh - 1;
    const int x0 = blockIdx.x * SF_TW, y0 = blockIdx.y * SF_TH;
    const float backmean = sc->backmean, dthresh = sc->dthresh;
    const int tid = threadIdx.y * SF_TX + threadIdx.x;
    int emin = 1000;
    for (int i = tid; i < TWp * THp; i += SF_TX * SF_TY) {
        int ty = i / TWp, tx = i - ty * TWp;
        int gx = x0 - rx + tx, gy = y0 - ry + ty;
        float s = 0.0f;
        if (gx >= 0 && gx < w && gy >= 0 && gy < h) {
            float raw = sx_unblank(__ldg(img + (size_t)gy * w + gx));
            s = raw - bkg_at(gx, gy, B, nbx, back_type, backmean);
            if (tx >= rx && tx < rx + SF_TW && ty >= ry && ty < ry + SF_TH) {
                sub[(size_t)gy * w + gx] = s;
                unsigned ef = (__float_as_uint(s) >> 23) & 0xff;
                if (ef) emin = min(emin, (int)ef - 127);
            }
        }
        tile[i] = s;
    }
    __syncthreads();
    int nabove = 0;
    for (int r = threadIdx.y; r < SF_TH; r += SF_TY) {
        int gx = x0 + threadIdx.x, gy = y0 + r;
        bool in = gx < w && gy < h;
        float acc = 0.0f;
        if (in) {
            const float *t0 = tile + r * TWp + threadIdx.x;
            for (int j = 0; j < mh; j++) {
                const float *tr = t0 + j * TWp;
                const float *mk = mask + j * mw;
                for (int i = 0; i < mw; i++) acc += mk[i] * tr[i];
            }
            size_t p = (size_t)gy * w + gx;
            cd[p] = acc;
            const float v = wvar ? __ldg(wvar + p) : 0.0f;
            bool fg = !(wvar && !(v < 1e30f)) && acc >= sx_pix_thr(wthr, dfac, v, dthresh);
            lab[p] = fg ? (int)p : -1;
            nabove += fg;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nabove += __shfl_down_sync(0xffffffffu, nabove, o);
        emin = min(emin, __shfl_down_sync(0xffffffffu, emin, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (nabove) atomicAdd(&sc->npix_above, nabove);
        if (emin < 1000) atomicMin(&sc->e0sub, emin);
    }
}

// ---------------------------------------------------------------------------
// The same stage with the frame tile (halo included) brought into shared
// memory by one TMA load (cp.async.bulk.tensor, zero fill outside the frame),
// 64x32 output pixels per CTA and the tile's spline column table staged in
// shared memory.  Needs rows of a multiple of 16 bytes and a 16-byte aligned
// frame; other frames take k_sub_filter.
// ---------------------------------------------------------------------------
constexpr int ST_TW = 64, ST_TH = 32, ST_THREADS = 256;
constexpr int ST_MAXBW = ST_TW + 2 * 16, ST_MAXBH = ST_TH + 2 * 15;  // masks up to 31x31
constexpr unsigned ST_WAIT_LIMIT = 1u << 24;                       // polls of the load barrier

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

constexpr int ST_RPT = 8;  // output rows per thread (64 columns x 4 row groups x 8 rows)

// Convolution of one output column segment (rows r0..r0+ST_RPT-1) from the
// shared tile.  Each input row is read once and added into every output row
// it serves; an output receives its terms in mask row-major order (mask rows
// in increasing order, columns left to right), as convolve() adds them.
template <int MW, int MH>
__device__ __forceinline__ void conv_rows(const ConvTaps &taps, const float *__restrict__ tile, int bw, int c0, int r0,
                                          float *acc) {
#pragma unroll
    for (int k = 0; k < ST_RPT; k++) acc[k] = 0.0f;
#pragma unroll
    for (int R = 0; R < ST_RPT + MH - 1; R++) {
        float v[MW];
        const float *row = tile + (r0 + R) * bw + c0;
#pragma unroll
        for (int i = 0; i < MW; i++) v[i] = row[i];
#pragma unroll
        for (int k = 0; k < ST_RPT; k++) {
            const int j = R - k;
            if (j >= 0 && j < MH) {
#pragma unroll
                for (int i = 0; i < MW; i++) acc[k] += taps.m[j * MW + i] * v[i];
            }
        }
    }
}

// any mask size (runtime loops, same order)
__device__ __forceinline__ void conv_rows_any(const float *__restrict__ mask, const float *__restrict__ tile, int bw,
                                              int c0, int r0, int mw, int mh, float *acc) {
    for (int k = 0; k < ST_RPT; k++) {
        const float *t0 = tile + (r0 + k) * bw + c0;
        float s = 0.0f;
        for (int j = 0; j < mh; j++) {
            const float *tr = t0 + j * bw;
            const float *mk = mask + j * mw;
            for (int i = 0; i < mw; i++) s += mk[i] * tr[i];
        }
        acc[k] = s;
    }
}

template <int MW, int MH>
__global__ void __launch_bounds__(ST_THREADS) k_sub_filter_tma(const __grid_constant__ CUtensorMap tmap,
                                                               float *__restrict__ sub, float *__restrict__ cd,
                                                               int *__restrict__ lab, BackBufs B, int w, int h,
                                                               int nbx, int back_type,
                                                               const __grid_constant__ ConvTaps taps,
                                                               const float *__restrict__ mask, int mw, int mh,
                                                               int rxa, const float *__restrict__ wvar, int wthr,
                                                               double dfac, FrameScalars *sc) {
    __shared__ __align__(128) float tile[ST_MAXBH * ST_MAXBW];
    __shared__ int s_colk[ST_MAXBW];
    __shared__ float s_coldx[ST_MAXBW];
    __shared__ __align__(8) unsigned long long bar;
    if constexpr (MW > 0) {
        mw = MW;
        mh = MH;
    }
    const int rx = mw / 2, ry = mh / 2;
    const int bw = ST_TW + 2 * rxa, bh = ST_TH + 2 * ry;
    const int x0 = blockIdx.x * ST_TW, y0 = blockIdx.y * ST_TH;
    const int tid = threadIdx.x, lane = tid & 31;
    const unsigned bar_a = smem_u32(&bar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar_a), "r"(1));
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a),
                     "r"((unsigned)(bw * bh * 4))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
                "r"(smem_u32(tile)),
            "l"(&tmap), "r"(x0 - rxa), "r"(y0 - ry), "r"(bar_a)
            : "memory");
    }
    // column table of the tile while the load is in flight
    for (int i = tid; i < bw; i += ST_THREADS) {
        const int gx = x0 - rxa + i;
        const bool in = gx >= 0 && gx < w;
        s_colk[i] = in ? B.colk[gx] : 0;
        s_coldx[i] = in ? B.coldx[gx] : 0.0f;
    }
    unsigned done = 0;
    for (unsigned it = 0; it < ST_WAIT_LIMIT && !done; it++)
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar_a), "r"(0u)
            : "memory");
    if (!__syncthreads_and(done)) {
        // the load did not complete in time: report it, give the copy one more
        // bounded wait so that it is not left writing into a finished CTA's
        // shared memory, and leave the outputs untouched
        if (tid == 0) {
            atomicOr(&sc->status, SX_ST_LOOP);
            for (unsigned it = 0; it < ST_WAIT_LIMIT && !done; it++)
                asm volatile(
                    "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                    : "=r"(done)
                    : "r"(bar_a), "r"(0u)
                    : "memory");
        }
        return;
    }
    const float backmean = sc->backmean, dthresh = sc->dthresh;
    // subtract the background in place, one warp per tile row; outside the
    // frame the value is 0
    int emin = 1000;
    for (int ty = tid >> 5; ty < bh; ty += ST_THREADS / 32) {
        const int gy = y0 - ry + ty;
        float *trow = tile + ty * bw;
        if (gy < 0 || gy >= h) {
            for (int tx = lane; tx < bw; tx += 32) trow[tx] = 0.0f;
            continue;
        }
        const float *nd = B.rownode + (size_t)gy * nbx;
        const float *dnd = B.rowdnode + (size_t)gy * nbx;
        const bool inner_row = ty >= ry && ty < ry + ST_TH;
        for (int tx = lane; tx < bw; tx += 32) {
            const int gx = x0 - rxa + tx;
            float s = 0.0f;
            if (gx >= 0 && gx < w) {
                float b;
                if (back_type == 1) {
                    b = backmean;
                } else if (nbx <= 1) {
                    b = __ldg(nd);
                } else {
                    const int k = s_colk[tx];
                    const float dx = s_coldx[tx], cdx = 1 - dx;
                    b = (float)(cdx * (__ldg(nd + k) + (cdx * cdx - 1) * __ldg(dnd + k)) +
                                dx * (__ldg(nd + k + 1) + (dx * dx - 1) * __ldg(dnd + k + 1)));
                }
                s = sx_unblank(trow[tx]) - b;
                if (inner_row && tx >= rxa && tx < rxa + ST_TW) {
                    sub[(size_t)gy * w + gx] = s;
                    const unsigned ef = (__float_as_uint(s) >> 23) & 0xff;
                    if (ef) emin = min(emin, (int)ef - 127);
                }
            }
            trow[tx] = s;
        }
    }
    __syncthreads();
    // convolution, threshold, label seed
    int nabove = 0;
    const int cx = tid & (ST_TW - 1), r0 = (tid / ST_TW) * ST_RPT;
    float acc[ST_RPT];
    if constexpr (MW > 0)
        conv_rows<MW, MH>(taps, tile, bw, cx + rxa - rx, r0, acc);
    else
        conv_rows_any(mask, tile, bw, cx + rxa - rx, r0, mw, mh, acc);
    const int gx = x0 + cx;
#pragma unroll
    for (int k = 0; k < ST_RPT; k++) {
        const int gy = y0 + r0 + k;
        if (gx < w && gy < h) {
            const size_t p = (size_t)gy * w + gx;
            cd[p] = acc[k];
            // with a weight map: unusable pixels never, others against the local rms
            const float v = wvar ? __ldg(wvar + p) : 0.0f;
            const bool fg = !(wvar && !(v < 1e30f)) && acc[k] >= sx_pix_thr(wthr, dfac, v, dthresh);
            lab[p] = fg ? (int)p : -1;
            nabove += fg;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nabove += __shfl_down_sync(0xffffffffu, nabove, o);
        emin = min(emin, __shfl_down_sync(0xffffffffu, emin, o));
    }
    if (lane == 0) {
        if (nabove) atomicAdd(&sc->npix_above, nabove);
        if (emin < 1000) atomicMin(&sc->e0sub, emin);
    }
}

// a 2D float tensor map of the frame with the tile box of this mask, or false
static bool make_frame_tmap(CUtensorMap *m, const float *img, int w, int h, int rxa, int ry) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
        else
            cudaGetLastError();
    }
    if (!encode || ((uintptr_t)img & 15) || (w % 4) != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h};
    const cuuint64_t strides[1] = {(cuuint64_t)w * 4};
    const cuuint32_t box[2] = {(cuuint32_t)(ST_TW + 2 * rxa), (cuuint32_t)(ST_TH + 2 * ry)};
    const cuuint32_t estr[2] = {1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)img, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void launch_sub_filter(const float *img, float *sub, float *cd, int *lab, const BackBufs &B, const FrameParams &P,
                       FrameScalars *d_sc, const float *d_var, const ConvMask &M, cudaStream_t st, int &launches) {
    const int mw = M.mw, mh = M.mh;
    const int rxa = ((mw / 2) + 3) & ~3;  // halo width rounded up to 16 bytes
    CUtensorMap tmap;
    if (make_frame_tmap(&tmap, img, P.w, P.h, rxa, mh / 2)) {
        dim3 tgrid((P.w + ST_TW - 1) / ST_TW, (P.h + ST_TH - 1) / ST_TH);
        ConvTaps taps;
        memset(&taps, 0, sizeof(taps));
        if (mw * mh <= 121) memcpy(taps.m, M.host, sizeof(float) * mw * mh);
#define SF_LAUNCH(a, b)                                                                                      \
    k_sub_filter_tma<a, b><<<tgrid, ST_THREADS, 0, st>>>(tmap, sub, cd, lab, B, P.w, P.h, P.nbx, P.back_type, \
                                                         taps, M.dev, mw, mh, rxa, d_var, P.wthr,           \
                                                         P.detect_thresh, d_sc)
        if (mw == mh && mw == 1)
            SF_LAUNCH(1, 1);
        else if (mw == mh && mw == 3)
            SF_LAUNCH(3, 3);
        else if (mw == mh && mw == 5)
            SF_LAUNCH(5, 5);
        else if (mw == mh && mw == 7)
            SF_LAUNCH(7, 7);
        else if (mw == mh && mw == 9)
            SF_LAUNCH(9, 9);
        else if (mw == mh && mw == 11)
            SF_LAUNCH(11, 11);
        else
            SF_LAUNCH(0, 0);
#undef SF_LAUNCH
        launches += 1;
        return;
    }
    dim3 grid((P.w + SF_TW - 1) / SF_TW, (P.h + SF_TH - 1) / SF_TH);
    dim3 block(SF_TX, SF_TY);
    size_t smem = sizeof(float) * (SF_TW + mw - 1) * (SF_TH + mh - 1);
    k_sub_filter<<<grid, block, smem, st>>>(img, sub, cd, lab, B, P.w, P.h, P.nbx, P.back_type, M.dev, mw, mh, d_var,
                                            P.wthr, P.detect_thresh, d_sc);
    launches += 1;
}

// ---------------------------------------------------------------------------
// union-find CCL
// ---------------------------------------------------------------------------
constexpr int CC_TW = 32, CC_TH = 16;

__device__ __forceinline__ int sfind(const int *L, int a) {
    while (L[a] != a) a = L[a];
    return a;
}

__device__ __forceinline__ void sunion(int *L, int a, int b) {
    for (int it = 0; it < 4096; it++) {
        a = sfind(L, a);
        b = sfind(L, b);
        if (a == b) return;
        if (a < b) {
            int t = a;
            a = b;
            b = t;
        }
        int old = atomicMin(&L[a], b);
        if (old == a) return;
        a = old;
    }
}

// Labels within one 32 x CC_TH tile, one warp per tile row.  A row's
// foreground is one ballot; pixels of a horizontal run are connected
// through the run's first pixel (bit arithmetic, no unions); a run joins the
// runs of the row above that touch it or its two diagonal ends (8-connected)
// with one union each, in shared memory.  Every link goes to a smaller tile
// index, so each tile component ends at its smallest pixel.
__device__ __forceinline__ int run_start(unsigned starts, int b) {  // start bit of the run holding bit b
    return 31 - __clz(starts & (0xffffffffu >> (31 - b)));
}
__device__ __forceinline__ int run_end(unsigned m, int b) {  // last bit of the run holding bit b
    return b + __ffsll(~(unsigned long long)(m >> b)) - 2;     // 64-bit: a run may reach bit 31
}

__global__ void __launch_bounds__(CC_TW *CC_TH) k_ccl_local(int *__restrict__ lab, int w, int h) {
    __shared__ int L[CC_TH * CC_TW];
    __shared__ unsigned rowm[CC_TH];
    const int lx = threadIdx.x, ly = threadIdx.y, t = ly * CC_TW + lx;
    const int gx = blockIdx.x * CC_TW + lx, gy = blockIdx.y * CC_TH + ly;
    const bool in = gx < w && gy < h;
    const bool fg = in && lab[(size_t)gy * w + gx] >= 0;
    const unsigned m = __ballot_sync(0xffffffffu, fg);
    const unsigned starts = m & ~(m << 1);
    if (lx == 0) rowm[ly] = m;
    L[t] = fg ? ly * CC_TW + run_start(starts, lx) : -1;
    __syncthreads();
    if (fg && ly > 0 && ((starts >> lx) & 1u)) {
        const int e = run_end(m, lx);
        const int s1 = lx > 0 ? lx - 1 : 0, e1 = e < 31 ? e + 1 : 31;
        const unsigned dil = (unsigned)((2ull << e1) - 1ull) & ~((1u << s1) - 1u);
        const unsigned mp = rowm[ly - 1], sp = mp & ~(mp << 1);
        unsigned ov = mp & dil;
        while (ov) {
            const int b = __ffs(ov) - 1;
            sunion(L, t, (ly - 1) * CC_TW + run_start(sp, b));
            const int eb = run_end(mp, b);
            ov = eb >= 31 ? 0u : ov & ~((2u << eb) - 1u);
        }
    }
    __syncthreads();
    if (fg) {
        int r = sfind(L, t);
        int rx = blockIdx.x * CC_TW + (r % CC_TW), ry = blockIdx.y * CC_TH + (r / CC_TW);
        lab[(size_t)gy * w + gx] = ry * w + rx;
    }
}

__device__ __forceinline__ int gfind(const int *L, int a) {
    int n = 0;
    while (true) {
        int p = L[a];
        if (p == a) return a;
        a = p;
        if (++n > (1 << 28)) return a;
    }
}

__device__ __forceinline__ void gunion(int *L, int a, int b, int *status) {
    for (int it = 0; it < (1 << 20); it++) {
        a = gfind(L, a);
        b = gfind(L, b);
        if (a == b) return;
        if (a < b) {
            int t = a;
            a = b;
            b = t;
        }
        int old = atomicMin(&L[a], b);
        if (old == a) return;
        a = old;
    }
    atomicOr(status, SX_ST_LOOP);
}

// unions across tile borders: pixels on the first row or first/last column
// of a tile look at their backward neighbours in other tiles
__global__ void k_ccl_border(int *__restrict__ lab, int w, int h, int *status) {
    int tilesx = (w + CC_TW - 1) / CC_TW;
    int tile = blockIdx.x, k = threadIdx.x;           // k < CC_TW + CC_TH
    int tx0 = (tile % tilesx) * CC_TW, ty0 = (tile / tilesx) * CC_TH;
    int x, y;
    if (k < CC_TW) {
        x = tx0 + k;
        y = ty0;
    } else {
        x = tx0;
        y = ty0 + (k - CC_TW) + 1;
        if (k - CC_TW + 1 >= CC_TH) return;
    }
    if (x >= w || y >= h) return;
    int p = y * w + x;
    if (lab[p] < 0) return;
    // W neighbour (other tile when x is the tile's first column)
    if (x == tx0 && x > 0 && lab[p - 1] >= 0) gunion(lab, p, p - 1, status);
    if (y > 0) {
        // NW: other tile when x or y is on the tile's first column/row
        if (x > 0 && (x == tx0 || y == ty0) && lab[p - w - 1] >= 0) gunion(lab, p, p - w - 1, status);
        if (y == ty0 && lab[p - w] >= 0) gunion(lab, p, p - w, status);
        if (x < w - 1 && (y == ty0 || x == tx0 + CC_TW - 1) && lab[p - w + 1] >= 0) gunion(lab, p, p - w + 1, status);
    }
}

// the last column of each tile also looks NE into the next tile (row y-1)
__global__ void k_ccl_border_ne(int *__restrict__ lab, int w, int h, int *status) {
    int tilesx = (w + CC_TW - 1) / CC_TW;
    int tile = blockIdx.x, k = threadIdx.x;  // k in [1, CC_TH)
    if (k == 0 || k >= CC_TH) return;
    int x = (tile % tilesx) * CC_TW + CC_TW - 1, y = (tile / tilesx) * CC_TH + k;
    if (x >= w - 1 || y >= h) return;
    int p = y * w + x;
    if (lab[p] >= 0 && lab[p - w + 1] >= 0) gunion(lab, p, p - w + 1, status);
}

__global__ void k_ccl_flatten(int *__restrict__ lab, long long n) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int l = lab[p];
    if (l < 0) return;
    int r = gfind(lab, (int)p);
    if (r != l) lab[p] = r;
}

void launch_ccl(int *lab, const FrameParams &P, FrameScalars *d_sc, cudaStream_t st, int &launches) {
    dim3 grid((P.w + CC_TW - 1) / CC_TW, (P.h + CC_TH - 1) / CC_TH);
    k_ccl_local<<<grid, dim3(CC_TW, CC_TH), 0, st>>>(lab, P.w, P.h);
    int ntiles = grid.x * grid.y;
    int *status = &d_sc->status;
    k_ccl_border<<<ntiles, CC_TW + CC_TH, 0, st>>>(lab, P.w, P.h, status);
    k_ccl_border_ne<<<ntiles, CC_TH, 0, st>>>(lab, P.w, P.h, status);
    long long n = (long long)P.w * P.h;
    k_ccl_flatten<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(lab, n);
    launches += 4;
}

}  // namespace sx
