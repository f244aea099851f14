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

// The background map of every pixel, the values src/back.c:790-936
// (subbackline) writes into backline and subtracts: the BACKGROUND check
// image (src/readimage.c:114); backmean everywhere for an absolute background.
__global__ void k_back_map(BackBufs B, int nbx, int back_type, const FrameScalars *sc, int w, long long n,
                           float *__restrict__ out) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int y = (int)(p / w), x = (int)(p - (long long)y * w);
    out[p] = bkg_at(x, y, B, nbx, back_type, sc->backmean);
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

// ---------------------------------------------------------------------------
// Persistent form: each CTA walks tiles t, t + G, ... with two tile buffers;
// the TMA load of the next tile is in flight while the current one is
// subtracted, filtered and thresholded.  Per tile the spline column constants
// (segment, dx, 1 - dx and the two cubic factors, all the float values the
// per-pixel formula uses) sit in each lane's registers (a lane keeps its four
// columns for the whole tile) and the row nodes of the tile's rows are staged
// in shared memory, so the per-pixel background is shared-memory reads and
// float arithmetic in the reference's order.
// ---------------------------------------------------------------------------
constexpr int SP_NK = 16;  // staged spline nodes per row (segments touching a tile + 1)

struct SpArgs {
    float *sub, *cd;
    int *lab;
    BackBufs B;
    int w, h, nbx, back_type, mw, mh, rxa, wthr, tilesx, ntiles;
    double dfac;
    const float *mask, *wvar;
    FrameScalars *sc;
};

__device__ __forceinline__ void sp_issue(const CUtensorMap *tmap, float *buf, unsigned bar, int x, int y,
                                         unsigned bytes) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::
            "r"(smem_u32(buf)),
        "l"(tmap), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ bool sp_wait(unsigned bar, unsigned parity) {
    unsigned done = 0;
    for (unsigned it = 0; it < ST_WAIT_LIMIT && !done; it++)
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
    return done != 0;
}

// ---- union-find in shared memory (tile-local components)
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

// runs of foreground bits in a row mask
__device__ __forceinline__ int run_start(unsigned starts, int b) {  // start bit of the run holding bit b
    return 31 - __clz(starts & (0xffffffffu >> (31 - b)));
}
__device__ __forceinline__ int run_end(unsigned m, int b) {  // last bit of the run holding bit b
    return b + __ffsll(~(unsigned long long)(m >> b)) - 2;     // 64-bit: a run may reach bit 31
}

// the same on 64-bit row masks (the subtract/filter kernel's 64-pixel tile rows)
__device__ __forceinline__ int run_start64(unsigned long long starts, int b) {
    return 63 - __clzll((long long)(starts & (~0ull >> (63 - b))));
}
__device__ __forceinline__ int run_end64(unsigned long long m, int b) {
    const unsigned long long r = ~(m >> b);
    return r ? b + __ffsll((long long)r) - 2 : 63;
}

template <int MW, int MH, bool WEIGHTED>
__global__ void __launch_bounds__(ST_THREADS, 4) k_sub_filter_pipe(const __grid_constant__ CUtensorMap tmap,
                                                                const __grid_constant__ SpArgs A,
                                                                const __grid_constant__ ConvTaps taps) {
    extern __shared__ __align__(128) float sp_smem[];
    __shared__ __align__(8) unsigned long long bars[2];
    __shared__ float s_nd[ST_MAXBH][SP_NK], s_dnd[ST_MAXBH][SP_NK];
    __shared__ int s_kmin, s_nk;
    __shared__ unsigned s_rowh[ST_TH][2];  // tile rows' foreground, two 32-bit halves
    __shared__ int s_L[ST_TH * ST_TW];     // tile-local union-find
    const int mw = MW > 0 ? MW : A.mw, mh = MH > 0 ? MH : A.mh;
    const int rx = mw / 2, ry = mh / 2, rxa = A.rxa;
    const int bw = ST_TW + 2 * rxa, bh = ST_TH + 2 * ry;
    const int tsz = (bw * bh + 31) & ~31;  // floats per tile buffer (128-byte multiple)
    float *const buf0 = sp_smem, *const buf1 = sp_smem + tsz;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int w = A.w, h = A.h;
    const unsigned bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);
    const unsigned tbytes = (unsigned)(bw * bh * 4);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar0), "r"(1));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar1), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int t = blockIdx.x;
    if (tid == 0 && t < A.ntiles)
        sp_issue(&tmap, buf0, bar0, (t % A.tilesx) * ST_TW - rxa, (t / A.tilesx) * ST_TH - ry, tbytes);
    const float backmean = A.sc->backmean, dthresh = A.sc->dthresh;
    int emin = 1000, nabove = 0;
    bool failed = false;
    for (int it = 0; t < A.ntiles; it++, t += gridDim.x) {
        const int cur = it & 1;
        float *const tile = cur ? buf1 : buf0;
        const int x0 = (t % A.tilesx) * ST_TW, y0 = (t / A.tilesx) * ST_TH;
        // next tile into the other buffer (free: the previous iteration ended
        // with a barrier after its last read)
        const int tn = t + gridDim.x;
        if (tid == 0 && tn < A.ntiles)
            sp_issue(&tmap, cur ? buf0 : buf1, cur ? bar0 : bar1, (tn % A.tilesx) * ST_TW - rxa,
                     (tn / A.tilesx) * ST_TH - ry, tbytes);
        // spline row nodes of this tile's rows, while the load is in flight
        const int gxa = x0 - rxa;
        const bool spline = A.back_type != 1 && A.nbx > 1;
        if (spline && tid == 0) {
            const int ka = A.B.colk[max(gxa, 0)], kb = A.B.colk[min(gxa + bw, w) - 1];
            s_kmin = ka;
            s_nk = kb - ka + 2;
        }
        __syncthreads();
        const int kmin = spline ? s_kmin : 0, nk = spline ? s_nk : 0;
        const bool staged = nk <= SP_NK;
        if (spline && staged)
            for (int i = tid; i < bh * nk; i += ST_THREADS) {
                const int ty = i / nk, j = i - ty * nk, gy = y0 - ry + ty;
                const int k = min(kmin + j, A.nbx - 1);
                const bool in = gy >= 0 && gy < h;
                s_nd[ty][j] = in ? A.B.rownode[(size_t)gy * A.nbx + k] : 0.0f;
                s_dnd[ty][j] = in ? A.B.rowdnode[(size_t)gy * A.nbx + k] : 0.0f;
            }
        // this lane's tile columns: 4*lane .. 4*lane+3 (lanes beyond the tile idle)
        int ck[4];
        float cdx[4], cb[4], cx[4], cdd[4];
        bool cin[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int tx = 4 * lane + q, gx = gxa + tx;
            cin[q] = tx < bw && gx >= 0 && gx < w;
            const int gxc = min(max(gx, 0), w - 1);
            const float dx = A.B.coldx[gxc];
            ck[q] = A.B.colk[gxc] - kmin;
            cx[q] = dx;
            cdx[q] = 1 - dx;
            cb[q] = cdx[q] * cdx[q] - 1;
            cdd[q] = dx * dx - 1;
        }
        // every thread polls; the outcome is made uniform before anyone acts on it
        if (!__syncthreads_and(sp_wait(cur ? bar1 : bar0, (unsigned)((it >> 1) & 1)))) {
            failed = true;
            break;
        }
        // subtract the background in place, one warp per tile row, four
        // columns per lane; outside the frame the value is 0
        for (int ty = wid; ty < bh; ty += ST_THREADS / 32) {
            const int gy = y0 - ry + ty;
            if (4 * lane >= bw) continue;
            float4 *tp = reinterpret_cast<float4 *>(tile + ty * bw) + lane;
            float4 v = *tp;
            float *vv = reinterpret_cast<float *>(&v);
            const bool rin = gy >= 0 && gy < h;
            const bool inner = ty >= ry && ty < ry + ST_TH;
            float *srow = A.sub + (size_t)(rin ? gy : 0) * w;
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float s = 0.0f;
                if (rin && cin[q]) {
                    float b;
                    if (!spline) {
                        b = A.back_type == 1 ? backmean : __ldg(A.B.rownode + (size_t)gy * A.nbx);
                    } else if (staged) {
                        const int k = ck[q];
                        b = (float)(cdx[q] * (s_nd[ty][k] + cb[q] * s_dnd[ty][k]) +
                                    cx[q] * (s_nd[ty][k + 1] + cdd[q] * s_dnd[ty][k + 1]));
                    } else {
                        const float *nd = A.B.rownode + (size_t)gy * A.nbx, *dnd = A.B.rowdnode + (size_t)gy * A.nbx;
                        const int k = ck[q] + kmin;
                        b = (float)(cdx[q] * (__ldg(nd + k) + cb[q] * __ldg(dnd + k)) +
                                    cx[q] * (__ldg(nd + k + 1) + cdd[q] * __ldg(dnd + k + 1)));
                    }
                    s = sx_unblank(vv[q]) - b;
                    const int tx = 4 * lane + q;
                    if (inner && tx >= rxa && tx < rxa + ST_TW) {
                        srow[gxa + tx] = s;
                        const unsigned ef = (__float_as_uint(s) >> 23) & 0xff;
                        if (ef) emin = min(emin, (int)ef - 127);
                    }
                }
                vv[q] = s;
            }
            *tp = v;
        }
        __syncthreads();
        // convolution, threshold, label seed: one column, ST_RPT rows per thread
        const int cxo = tid & (ST_TW - 1), r0 = (tid / ST_TW) * ST_RPT;
        float acc[ST_RPT];
        if constexpr (MW > 0)
            conv_rows<MW, MH>(taps, tile, bw, cxo + rxa - rx, r0, acc);
        else
            conv_rows_any(A.mask, tile, bw, cxo + rxa - rx, r0, mw, mh, acc);
        const int gx = x0 + cxo;
        unsigned fgb = 0u;  // bit k: pixel (cxo, r0 + k) above its threshold
#pragma unroll
        for (int k = 0; k < ST_RPT; k++) {
            const int gy = y0 + r0 + k;
            if (gx < w && gy < h) {
                const int p = gy * w + gx;
                A.cd[p] = acc[k];
                bool fg;
                if (WEIGHTED) {
                    const float v = __ldg(A.wvar + p);
                    fg = (v < 1e30f) && acc[k] >= sx_pix_thr(A.wthr, A.dfac, v, dthresh);
                } else {
                    fg = acc[k] >= dthresh;
                }
                fgb |= (unsigned)fg << k;
                nabove += fg;
            }
        }
        // Components within the tile (the first step of the CCL, done here
        // while the tile's foreground is on chip): each tile row's foreground
        // as 64 bits from two ballots; the pixels of a horizontal run join
        // the run's first pixel; a run joins the runs of the row above that
        // touch it or its diagonal ends.  Every link goes to a smaller tile
        // index, so a tile component ends at its smallest pixel, which is
        // written as the label of each of its pixels (global index).
#pragma unroll
        for (int k = 0; k < ST_RPT; k++) {
            const unsigned m = __ballot_sync(0xffffffffu, (fgb >> k) & 1u);
            if (lane == 0) s_rowh[r0 + k][cxo >> 5] = m;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < ST_RPT; k++) {
            const int ty = r0 + k, t = ty * ST_TW + cxo;
            const unsigned long long m = ((unsigned long long)s_rowh[ty][1] << 32) | s_rowh[ty][0];
            s_L[t] = (fgb >> k) & 1u ? ty * ST_TW + run_start64(m & ~(m << 1), cxo) : -1;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < ST_RPT; k++) {
            const int ty = r0 + k;
            if (!((fgb >> k) & 1u) || ty == 0) continue;
            const unsigned long long m = ((unsigned long long)s_rowh[ty][1] << 32) | s_rowh[ty][0];
            if (!((m >> cxo) & 1ull) || (cxo > 0 && ((m >> (cxo - 1)) & 1ull))) continue;  // run starts only
            const int e = run_end64(m, cxo);
            const int s1 = cxo > 0 ? cxo - 1 : 0, e1 = e < 63 ? e + 1 : 63;
            const unsigned long long dil = (e1 == 63 ? ~0ull : ((2ull << e1) - 1ull)) & ~((1ull << s1) - 1ull);
            const unsigned long long mp = ((unsigned long long)s_rowh[ty - 1][1] << 32) | s_rowh[ty - 1][0];
            const unsigned long long sp = mp & ~(mp << 1);
            unsigned long long ov = mp & dil;
            while (ov) {
                const int b = __ffsll((long long)ov) - 1;
                sunion(s_L, ty * ST_TW + cxo, (ty - 1) * ST_TW + run_start64(sp, b));
                const int eb = run_end64(mp, b);
                ov = eb >= 63 ? 0ull : ov & ~((2ull << eb) - 1ull);
            }
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < ST_RPT; k++) {
            const int gy = y0 + r0 + k;
            if (gx < w && gy < h) {
                int l = -1;
                if ((fgb >> k) & 1u) {
                    const int r = sfind(s_L, (r0 + k) * ST_TW + cxo);
                    l = (y0 + r / ST_TW) * w + x0 + r % ST_TW;
                }
                A.lab[gy * w + gx] = l;
            }
        }
        __syncthreads();
    }
    if (failed) {
        // A load did not complete in time: report it, and give the copies
        // still in flight one more bounded wait before the CTA exits.  A copy
        // that outlasts that wait too may still write into shared memory after
        // the CTA has gone, so this status (SEXGPU_ERR_LOAD) tells the caller
        // to destroy the context rather than use it again.
        if (tid == 0) {
            atomicOr(&A.sc->status, SX_ST_LOAD);
            sp_wait(bar0, 0);
            sp_wait(bar0, 1);
            sp_wait(bar1, 0);
            sp_wait(bar1, 1);
        }
        return;
    }
    for (int o = 16; o > 0; o >>= 1) {
        nabove += __shfl_down_sync(0xffffffffu, nabove, o);
        emin = min(emin, __shfl_down_sync(0xffffffffu, emin, o));
    }
    if (lane == 0) {
        if (nabove) atomicAdd(&A.sc->npix_above, nabove);
        if (emin < 1000) atomicMin(&A.sc->e0sub, emin);
    }
}

// a 2D float tensor map of the frame with the tile box of this mask, or false
static bool make_frame_tmap(CUtensorMap *m, const float *img, int w, int h, int rxa, int ry) {
    // the driver's encoder, looked up once (a function-local static is
    // initialised once even when host threads arrive together)
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return (PFN_cuTensorMapEncodeTiled_v12000)fn;
        cudaGetLastError();
        return nullptr;
    }();
    if (!encode || ((uintptr_t)img & 15) || (w % 4) != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h};
    const cuuint64_t strides[1] = {(cuuint64_t)w * 4};
    const cuuint32_t box[2] = {(cuuint32_t)(ST_TW + 2 * rxa), (cuuint32_t)(ST_TH + 2 * ry)};
    const cuuint32_t estr[2] = {1, 1};
    return encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)img, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Returns true when the labels written are already tile-local components
// (the subtract/filter pipeline's 64 x 32 tiles), false when they are seeds
// (every foreground pixel its own label).
bool launch_sub_filter(const float *img, float *sub, float *cd, int *lab, const BackBufs &B, const FrameParams &P,
                       FrameScalars *d_sc, const float *d_var, const ConvMask &M, cudaStream_t st, int &launches) {
    const int mw = M.mw, mh = M.mh;
    const int rxa = ((mw / 2) + 3) & ~3;  // halo width rounded up to 16 bytes
    CUtensorMap tmap;
    if (make_frame_tmap(&tmap, img, P.w, P.h, rxa, mh / 2)) {
        SpArgs A;
        A.sub = sub;
        A.cd = cd;
        A.lab = lab;
        A.B = B;
        A.w = P.w;
        A.h = P.h;
        A.nbx = P.nbx;
        A.back_type = P.back_type;
        A.mw = mw;
        A.mh = mh;
        A.rxa = rxa;
        A.wthr = P.wthr;
        A.tilesx = (P.w + ST_TW - 1) / ST_TW;
        A.ntiles = A.tilesx * ((P.h + ST_TH - 1) / ST_TH);
        A.dfac = P.detect_thresh;
        A.mask = M.dev;
        A.wvar = d_var;
        A.sc = d_sc;
        ConvTaps taps;
        memset(&taps, 0, sizeof(taps));
        if (mw * mh <= 121) memcpy(taps.m, M.host, sizeof(float) * mw * mh);
        const int bw = ST_TW + 2 * rxa, bh = ST_TH + 2 * (mh / 2);
        const size_t smem = 2 * sizeof(float) * (size_t)((bw * bh + 31) & ~31);
        static DevCache nsm_cache;
        const int nsm = nsm_cache.get([](int dev) {
            int n = 148;
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
            return n > 0 ? n : 148;
        });
#define SP_LAUNCH(a, b, wt)                                                                              \
    do {                                                                                                \
        auto kern = k_sub_filter_pipe<a, b, wt>;                                                        \
        /* (smem << 8) | resident CTAs of this instance, per device */                                 \
        static std::atomic<long long> cached[64];                                                       \
        int dev_ = 0;                                                                                   \
        cudaGetDevice(&dev_);                                                                           \
        std::atomic<long long> &slot = cached[dev_ >= 0 && dev_ < 64 ? dev_ : 0];                      \
        long long c = slot.load(std::memory_order_relaxed);                                             \
        int per = (int)(c & 255);                                                                       \
        if ((c >> 8) != (long long)smem) {                                                              \
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);        \
            per = 1;                                                                                    \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, ST_THREADS, smem);                \
            per = std::min(std::max(per, 1), 255);                                                      \
            slot.store(((long long)smem << 8) | per, std::memory_order_relaxed);                        \
        }                                                                                               \
        const int grid = std::max(1, std::min(A.ntiles, sx_share(nsm * per)));                         \
        kern<<<grid, ST_THREADS, smem, st>>>(tmap, A, taps);                                            \
    } while (0)
#define SP_MASK(wt)                    \
    if (mw == mh && mw == 1)           \
        SP_LAUNCH(1, 1, wt);           \
    else if (mw == mh && mw == 3)      \
        SP_LAUNCH(3, 3, wt);           \
    else if (mw == mh && mw == 5)      \
        SP_LAUNCH(5, 5, wt);           \
    else if (mw == mh && mw == 7)      \
        SP_LAUNCH(7, 7, wt);           \
    else if (mw == mh && mw == 9)      \
        SP_LAUNCH(9, 9, wt);           \
    else if (mw == mh && mw == 11)     \
        SP_LAUNCH(11, 11, wt);         \
    else                               \
        SP_LAUNCH(0, 0, wt)
        if (d_var) {
            SP_MASK(true);
        } else {
            SP_MASK(false);
        }
#undef SP_MASK
#undef SP_LAUNCH
        launches += 1;
        return true;
    }
    dim3 grid((P.w + SF_TW - 1) / SF_TW, (P.h + SF_TH - 1) / SF_TH);
    dim3 block(SF_TX, SF_TY);
    size_t smem = sizeof(float) * (SF_TW + mw - 1) * (SF_TH + mh - 1);
    k_sub_filter<<<grid, block, smem, st>>>(img, sub, cd, lab, B, P.w, P.h, P.nbx, P.back_type, M.dev, mw, mh, d_var,
                                            P.wthr, P.detect_thresh, d_sc);
    launches += 1;
    return false;
}

// ---------------------------------------------------------------------------
// union-find CCL
// ---------------------------------------------------------------------------
constexpr int CC_TW = 32, CC_TH = 16;

// Labels within one 32 x CC_TH tile, one warp per tile row (frames that the
// subtract/filter kernel could not label itself).  A row's foreground is one
// ballot; pixels of a horizontal run are connected through the run's first
// pixel (bit arithmetic, no unions); a run joins the runs of the row above
// that touch it or its two diagonal ends (8-connected) with one union each,
// in shared memory.  Every link goes to a smaller tile index, so each tile
// component ends at its smallest pixel.
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

// walk to the root; a walk longer than cap steps sets SX_ST_LOOP and stops
__device__ __forceinline__ int gfind(const int *L, int a, int cap, int *status) {
    for (int n = 0; n <= cap; n++) {
        int p = L[a];
        if (p == a) return a;
        a = p;
    }
    atomicOr(status, SX_ST_LOOP);
    return a;
}

// walk and link caps: the built-in ones, or a smaller cap set for a test
__device__ __forceinline__ int ccl_walk_cap(int loop_cap) { return loop_cap > 0 ? loop_cap : (1 << 28); }
__device__ __forceinline__ int ccl_link_cap(int loop_cap) { return loop_cap > 0 ? loop_cap : (1 << 20); }

__device__ __forceinline__ void gunion(int *L, int a, int b, int *status, int loop_cap) {
    const int wcap = ccl_walk_cap(loop_cap), lcap = ccl_link_cap(loop_cap);
    for (int it = 0; it < lcap; it++) {
        a = gfind(L, a, wcap, status);
        b = gfind(L, b, wcap, status);
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

// unions across tile borders (TW x TH tiles): pixels on the first row or
// first/last column of a tile look at their backward neighbours in other tiles
template <int TW, int TH>
__global__ void k_ccl_border(int *__restrict__ lab, int w, int h, int *status, int loop_cap) {
    int tilesx = (w + TW - 1) / TW;
    int tile = blockIdx.x, k = threadIdx.x;           // k < TW + TH
    int tx0 = (tile % tilesx) * TW, ty0 = (tile / tilesx) * TH;
    int x, y;
    if (k < TW) {
        x = tx0 + k;
        y = ty0;
    } else {
        x = tx0;
        y = ty0 + (k - TW) + 1;
        if (k - TW + 1 >= TH) return;
    }
    if (x >= w || y >= h) return;
    int p = y * w + x;
    if (lab[p] < 0) return;
    // W neighbour (other tile when x is the tile's first column)
    if (x == tx0 && x > 0 && lab[p - 1] >= 0) gunion(lab, p, p - 1, status, loop_cap);
    if (y > 0) {
        // NW: other tile when x or y is on the tile's first column/row
        if (x > 0 && (x == tx0 || y == ty0) && lab[p - w - 1] >= 0) gunion(lab, p, p - w - 1, status, loop_cap);
        if (y == ty0 && lab[p - w] >= 0) gunion(lab, p, p - w, status, loop_cap);
        if (x < w - 1 && (y == ty0 || x == tx0 + TW - 1) && lab[p - w + 1] >= 0) gunion(lab, p, p - w + 1, status, loop_cap);
    }
}

// the last column of each tile also looks NE into the next tile (row y-1)
template <int TW, int TH>
__global__ void k_ccl_border_ne(int *__restrict__ lab, int w, int h, int *status, int loop_cap) {
    int tilesx = (w + TW - 1) / TW;
    int tile = blockIdx.x, k = threadIdx.x;  // k in [1, TH)
    if (k == 0 || k >= TH) return;
    int x = (tile % tilesx) * TW + TW - 1, y = (tile / tilesx) * TH + k;
    if (x >= w - 1 || y >= h) return;
    int p = y * w + x;
    if (lab[p] >= 0 && lab[p - w + 1] >= 0) gunion(lab, p, p - w + 1, status, loop_cap);
}

// every pixel to its root, and the component sizes: lanes of a warp holding
// the same root add once to cnt (zeroed before).  Four consecutive pixels a
// thread, their labels read and written as one 16-byte word where all four
// are in the frame: each entry written is -1 (background, which nothing else
// writes) or the pixel's root, so a concurrent walk through it still reads an
// ancestor (the walks only read).
__global__ void k_ccl_flatten(int *__restrict__ lab, long long n, int *__restrict__ cnt, int *status, int loop_cap) {
    const long long base = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const bool vec = base + 3 < n && (reinterpret_cast<uintptr_t>(lab) & 15) == 0;
    int l[4], r[4];
    if (vec) {
        const int4 v = *reinterpret_cast<const int4 *>(lab + base);
        l[0] = v.x;
        l[1] = v.y;
        l[2] = v.z;
        l[3] = v.w;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) l[k] = base + k < n ? lab[base + k] : -1;
    }
    bool changed = false;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        r[k] = l[k] >= 0 ? gfind(lab, (int)(base + k), ccl_walk_cap(loop_cap), status) : -1;
        changed |= r[k] != l[k];
    }
    if (changed) {
        if (vec) {
            *reinterpret_cast<int4 *>(lab + base) = make_int4(r[0], r[1], r[2], r[3]);
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (r[k] != l[k]) lab[base + k] = r[k];
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const unsigned same = __match_any_sync(0xffffffffu, r[k]);
        if (r[k] >= 0 && (threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&cnt[r[k]], __popc(same));
    }
}

// cnt: zeroed, w*h ints; receives the size of every component at its root
// tiled: the labels are already the tile-local components of the
// subtract/filter pipeline's ST_TW x ST_TH tiles (else seeds, labelled here
// in CC_TW x CC_TH tiles first)
void launch_ccl(int *lab, int *cnt, const FrameParams &P, FrameScalars *d_sc, cudaStream_t st, int &launches,
                bool tiled) {
    int *status = &d_sc->status;
    if (tiled) {
        const int ntiles = ((P.w + ST_TW - 1) / ST_TW) * ((P.h + ST_TH - 1) / ST_TH);
        k_ccl_border<ST_TW, ST_TH><<<ntiles, ST_TW + ST_TH, 0, st>>>(lab, P.w, P.h, status, P.loop_cap);
        k_ccl_border_ne<ST_TW, ST_TH><<<ntiles, ST_TH, 0, st>>>(lab, P.w, P.h, status, P.loop_cap);
        launches += 3;
    } else {
        dim3 grid((P.w + CC_TW - 1) / CC_TW, (P.h + CC_TH - 1) / CC_TH);
        k_ccl_local<<<grid, dim3(CC_TW, CC_TH), 0, st>>>(lab, P.w, P.h);
        const int ntiles = grid.x * grid.y;
        k_ccl_border<CC_TW, CC_TH><<<ntiles, CC_TW + CC_TH, 0, st>>>(lab, P.w, P.h, status, P.loop_cap);
        k_ccl_border_ne<CC_TW, CC_TH><<<ntiles, CC_TH, 0, st>>>(lab, P.w, P.h, status, P.loop_cap);
        launches += 4;
    }
    long long n = (long long)P.w * P.h;
    k_ccl_flatten<<<(unsigned)((n + 1023) / 1024), 256, 0, st>>>(lab, n, cnt, status, P.loop_cap);
}

}  // namespace sx
