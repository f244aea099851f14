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
#include "common.cuh"
#include "kernels.cuh"

namespace sx {

__constant__ float c_mask[SX_MAXCONV * SX_MAXCONV];

void set_conv_mask(const float *mask, int mw, int mh, cudaStream_t st) {
    cudaMemcpyToSymbolAsync(c_mask, mask, sizeof(float) * mw * mh, 0, cudaMemcpyHostToDevice, st);
}

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
                                                              int mw, int mh, FrameScalars *sc) {
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
                const float *mk = c_mask + j * mw;
                for (int i = 0; i < mw; i++) acc += mk[i] * tr[i];
            }
            size_t p = (size_t)gy * w + gx;
            cd[p] = acc;
            bool fg = acc >= dthresh;
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

void launch_sub_filter(const float *img, float *sub, float *cd, int *lab, const BackBufs &B, const FrameParams &P,
                       FrameScalars *d_sc, const float *d_var, cudaStream_t st, int &launches) {
    (void)d_var;
    dim3 grid((P.w + SF_TW - 1) / SF_TW, (P.h + SF_TH - 1) / SF_TH);
    dim3 block(SF_TX, SF_TY);
    int mw = P.filter_flag ? P.conv_w : 1, mh = P.filter_flag ? P.conv_h : 1;
    size_t smem = sizeof(float) * (SF_TW + mw - 1) * (SF_TH + mh - 1);
    k_sub_filter<<<grid, block, smem, st>>>(img, sub, cd, lab, B, P.w, P.h, P.nbx, P.back_type, mw, mh, d_sc);
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

// labels within one tile, union in shared memory
__global__ void __launch_bounds__(CC_TW *CC_TH) k_ccl_local(int *__restrict__ lab, int w, int h) {
    __shared__ int L[CC_TH * CC_TW];
    int lx = threadIdx.x, ly = threadIdx.y, t = ly * CC_TW + lx;
    int gx = blockIdx.x * CC_TW + lx, gy = blockIdx.y * CC_TH + ly;
    bool in = gx < w && gy < h;
    bool fg = in && lab[(size_t)gy * w + gx] >= 0;
    L[t] = fg ? t : -1;
    __syncthreads();
    if (fg) {
        if (lx > 0 && L[t - 1] >= 0) sunion(L, t, t - 1);
        if (ly > 0) {
            if (lx > 0 && L[t - CC_TW - 1] >= 0) sunion(L, t, t - CC_TW - 1);
            if (L[t - CC_TW] >= 0) sunion(L, t, t - CC_TW);
            if (lx < CC_TW - 1 && L[t - CC_TW + 1] >= 0) sunion(L, t, t - CC_TW + 1);
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
