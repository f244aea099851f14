// k_back.cu -- background estimation (reference: src/back.c makeback,
// backstat, backhisto, backguess, filterback, makebackspline, subbackline and
// the CUDA driver src/cuda/cudaback.cu:1212).
//
// Results are bit-identical to the reference's CPU functions:
//  * the per-mesh mean/sigma are the reference's sequential double sums, run
//    one thread per mesh in the same pixel order;
//  * histogram sums are exact integers, so they are reduced in parallel;
//  * the two-pointer median walk of backguess is replaced by a binary search
//    on the merge path of the two cumulative sums, which lands on the same
//    split;
//  * spline and interpolation arithmetic is float, in the reference's order.
#include "common.cuh"
#include "kernels.cuh"

namespace sx {

// src/back.c:214-279 for one mesh: the reference's two sequential double
// passes, in its pixel order.  `row0` points at the mesh's first pixel, rows
// `stride` floats apart.  A pixel left out adds +0.0 instead of skipping the
// addition: the sums start at +0.0 and so are never -0.0, hence s + 0.0 == s
// exactly, and the select stays off the dependent chain of additions (the
// chain is the cost of these loops: two passes over 64 x 64 meshes take about
// 33 cycles per pixel and pass on B200).
__device__ __forceinline__ void mesh_stat_seq(const float *row0, int stride, int mw, int mh, MeshStat &o) {
    double pix, sig, mean = 0.0, sigma = 0.0;
    const double step = sqrt(2 / SX_PI) * SX_QUANTIF_NSIGMA / SX_QUANTIF_AMIN;
    int npix = 0;
    o.mean = o.sigma = o.lcut = o.hcut = o.qzero = o.qscale = 0.f;
    o.nlevels = o.npix = 0;
    for (int y = 0; y < mh; y++) {
        const float *row = row0 + (size_t)y * stride;
        // unrolled so that loads and conversions run ahead of the two
        // accumulation chains; the additions stay in pixel order
#pragma unroll 8
        for (int x = 0; x < mw; x++) {
            pix = row[x];
            const bool in = pix > -SX_BIG;
            mean += in ? pix : 0.0;
            sigma += in ? pix * pix : 0.0;
            npix += in;
        }
    }
    if ((float)npix < (float)(mw * mh * SX_BACK_MINGOODFRAC)) {
        o.mean = o.sigma = -SX_BIG;
        return;
    }
    mean /= (double)npix;
    sigma = (sig = sigma / npix - mean * mean) > 0.0 ? sqrt(sig) : 0.0;
    const float lcut = o.lcut = (float)(mean - 2.0 * sigma);
    const float hcut = o.hcut = (float)(mean + 2.0 * sigma);
    mean = sigma = 0.0;
    npix = 0;
    for (int y = 0; y < mh; y++) {
        const float *row = row0 + (size_t)y * stride;
#pragma unroll 8
        for (int x = 0; x < mw; x++) {
            pix = row[x];
            const bool in = pix <= hcut && pix >= lcut;
            mean += in ? pix : 0.0;
            sigma += in ? pix * pix : 0.0;
            npix += in;
        }
    }
    o.npix = npix;
    mean /= (double)npix;
    sig = sigma / npix - mean * mean;
    sigma = sig > 0.0 ? sqrt(sig) : 0.0;
    o.mean = mean;
    o.sigma = sigma;
    if ((o.nlevels = (int)(step * npix + 1)) > SX_QUANTIF_NMAXLEVELS) o.nlevels = SX_QUANTIF_NMAXLEVELS;
    o.qscale = sigma > 0.0 ? 2 * SX_QUANTIF_NSIGMA * sigma / o.nlevels : 1.0;
    o.qzero = mean - SX_QUANTIF_NSIGMA * sigma;
}

__device__ __forceinline__ void mesh_geometry(int m, int w, int h, int bw, int bh, int nbx, int nby, int &x0, int &y0,
                                              int &mw, int &mh) {
    const int mx = m % nbx, my = m / nbx;
    x0 = mx * bw;
    y0 = my * bh;
    mw = (mx == nbx - 1 && w % bw) ? w % bw : bw;
    mh = (my == nby - 1 && h % bh) ? h % bh : bh;
}

// one thread per mesh, straight from the frame (meshes too large to stage)
__global__ void k_mesh_stat(const float *__restrict__ img, int w, int h, int bw, int bh, int nbx, int nby,
                            MeshStat *__restrict__ ms) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nbx * nby) return;
    int x0, y0, mw, mh;
    mesh_geometry(m, w, h, bw, bh, nbx, nby, x0, y0, mw, mh);
    MeshStat o;
    mesh_stat_seq(img + (size_t)y0 * w + x0, w, mw, mh, o);
    ms[m] = o;
}

// One warp per row band of 32 meshes, one lane per mesh.  The band's pixel
// rows are staged in shared memory by cp.async (coalesced across the band) in
// a ring of BAND_STAGES rows, so that the loads of the next rows are in
// flight while the lanes add the current one; every lane then adds its mesh's
// part of the row to its own sums, so each lane performs the reference's
// sequential double sums in the reference's pixel order.  Mesh j of the band
// sits at j * stride in a row buffer.  VEC (frame width and mesh width
// multiples of 4): 16-byte copies, float4 reads, stride = 4 (mod 8) so that
// the eight lanes of a float4 read phase hit distinct banks; otherwise 4-byte
// copies and an odd stride.
constexpr int BAND_STAGES = 4;

// Copy c of a row (c = lane, lane + 32, ...; float4s when VEC, else floats)
// is element r of mesh j, c = j q + r with q the copies per mesh row; (j0, r0)
// is the lane's first and (dj, dr) the step of 32 copies, so no division is
// needed per copy.
struct BandCopy {
    int q, j0, r0, dj, dr;
};

template <bool VEC>
__device__ __forceinline__ void band_row_async(float *dst, const float *img, int w, int gy, int x0, int tw,
                                               int stride, const BandCopy &bc) {
    const int lane = threadIdx.x & 31;
    const float *src = img + (size_t)gy * w + x0;
    int j = bc.j0, r = bc.r0;
    if (VEC) {
        for (int c = lane; 4 * c < tw; c += 32) {
            const unsigned d = (unsigned)__cvta_generic_to_shared(dst + j * stride + 4 * r);
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src + 4 * c) : "memory");
            r += bc.dr;
            j += bc.dj;
            if (r >= bc.q) {
                r -= bc.q;
                j++;
            }
        }
    } else {
        for (int c = lane; c < tw; c += 32) {
            const unsigned d = (unsigned)__cvta_generic_to_shared(dst + j * stride + r);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src + c) : "memory");
            r += bc.dr;
            j += bc.dj;
            if (r >= bc.q) {
                r -= bc.q;
                j++;
            }
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// the two accumulation loops of one row (pass 0: valid pixels; pass 1:
// pixels inside [lcut, hcut]).  The tests are made on the float: a float
// compares with the float cuts as its double does, and f > (float)-BIG as
// (double)f > -BIG (the float nearest -1e30 lies below it, the next one up
// above it).  The square of a float is exact in double, so fma(p, p, s) is
// s + p * p rounded once, as the reference adds it.
template <int PASS>
__device__ __forceinline__ void band_add(float f, float lcut, float hcut, double &mean, double &sigma, int &npix) {
    const bool in = PASS == 0 ? f > (float)-SX_BIG : (f <= hcut && f >= lcut);
    const double pix = (double)(in ? f : 0.0f);
    mean += pix;
    sigma = fma(pix, pix, sigma);
    npix += in;
}

template <int PASS, bool VEC>
__device__ __forceinline__ void band_row_add(const float *row, int mw, float lcut, float hcut, double &mean,
                                             double &sigma, int &npix) {
    if (VEC) {
        const float4 *r4 = reinterpret_cast<const float4 *>(row);
#pragma unroll 4
        for (int q = 0; q < (mw >> 2); q++) {
            const float4 v = r4[q];
            band_add<PASS>(v.x, lcut, hcut, mean, sigma, npix);
            band_add<PASS>(v.y, lcut, hcut, mean, sigma, npix);
            band_add<PASS>(v.z, lcut, hcut, mean, sigma, npix);
            band_add<PASS>(v.w, lcut, hcut, mean, sigma, npix);
        }
    } else {
#pragma unroll 8
        for (int x = 0; x < mw; x++) band_add<PASS>(row[x], lcut, hcut, mean, sigma, npix);
    }
}

template <bool VEC>
__global__ void __launch_bounds__(32) k_mesh_stat_band(const float *__restrict__ img, int w, int h, int bw, int bh,
                                                       int nbx, int nby, int stride, MeshStat *__restrict__ ms) {
    extern __shared__ __align__(16) float band_smem[];
    const int lane = threadIdx.x;
    const int mx0 = blockIdx.x * 32, my = blockIdx.y;
    const int nmesh = min(32, nbx - mx0);
    const int x0 = mx0 * bw, y0 = my * bh;
    const int mh = (my == nby - 1 && h % bh) ? h % bh : bh;
    const int mw_last = (mx0 + nmesh == nbx && w % bw) ? w % bw : bw;
    const int tw = (nmesh - 1) * bw + mw_last;  // band width in pixels
    const bool active = lane < nmesh;
    const int mw = lane == nmesh - 1 ? mw_last : bw;
    const int rowf = 32 * stride;  // floats per staged row
    BandCopy bc;
    bc.q = VEC ? bw >> 2 : bw;
    bc.j0 = lane / bc.q;
    bc.r0 = lane - bc.j0 * bc.q;
    bc.dj = 32 / bc.q;
    bc.dr = 32 - bc.dj * bc.q;
    double sig, mean = 0.0, sigma = 0.0;
    const double step = sqrt(2 / SX_PI) * SX_QUANTIF_NSIGMA / SX_QUANTIF_AMIN;
    int npix = 0;
    float lcut = 0.0f, hcut = 0.0f;
    bool bad = false;
    for (int pass = 0; pass < 2; pass++) {
        for (int y = 0; y < BAND_STAGES - 1; y++) {
            if (y < mh)
                band_row_async<VEC>(band_smem + y * rowf, img, w, y0 + y, x0, tw, stride, bc);
            else
                asm volatile("cp.async.commit_group;" ::: "memory");
        }
        for (int y = 0; y < mh; y++) {
            const int ya = y + BAND_STAGES - 1;
            if (ya < mh)
                band_row_async<VEC>(band_smem + (ya % BAND_STAGES) * rowf, img, w, y0 + ya, x0, tw, stride, bc);
            else
                asm volatile("cp.async.commit_group;" ::: "memory");
            asm volatile("cp.async.wait_group %0;" ::"n"(BAND_STAGES - 1) : "memory");
            __syncwarp();
            if (active) {
                const float *row = band_smem + (y % BAND_STAGES) * rowf + lane * stride;
                if (pass == 0)
                    band_row_add<0, VEC>(row, mw, lcut, hcut, mean, sigma, npix);
                else
                    band_row_add<1, VEC>(row, mw, lcut, hcut, mean, sigma, npix);
            }
            __syncwarp();
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncwarp();
        if (pass == 0) {
            // src/back.c:249: too few valid pixels: a bad mesh
            if ((float)npix < (float)(mw * mh * SX_BACK_MINGOODFRAC)) bad = true;
            mean /= (double)npix;
            sigma = (sig = sigma / npix - mean * mean) > 0.0 ? sqrt(sig) : 0.0;
            lcut = (float)(mean - 2.0 * sigma);
            hcut = (float)(mean + 2.0 * sigma);
            mean = sigma = 0.0;
            npix = 0;
            if (__all_sync(0xffffffffu, bad || !active)) break;
        }
    }
    if (!active) return;
    MeshStat o;
    o.mean = o.sigma = o.lcut = o.hcut = o.qzero = o.qscale = 0.f;
    o.nlevels = o.npix = 0;
    if (bad) {
        o.mean = o.sigma = -SX_BIG;
    } else {
        o.lcut = lcut;
        o.hcut = hcut;
        o.npix = npix;
        mean /= (double)npix;
        sig = sigma / npix - mean * mean;
        sigma = sig > 0.0 ? sqrt(sig) : 0.0;
        o.mean = mean;
        o.sigma = sigma;
        if ((o.nlevels = (int)(step * npix + 1)) > SX_QUANTIF_NMAXLEVELS) o.nlevels = SX_QUANTIF_NMAXLEVELS;
        o.qscale = sigma > 0.0 ? 2 * SX_QUANTIF_NSIGMA * sigma / o.nlevels : 1.0;
        o.qzero = mean - SX_QUANTIF_NSIGMA * sigma;
    }
    ms[my * nbx + mx0 + lane] = o;
}

constexpr int GUESS_THREADS = 256;

// src/back.c:297-339 (backhisto) + :347-432 (backguess), one CTA per mesh
// src/back.c:347-432 (backguess) on a histogram already in shared memory,
// for the whole CTA: the prefix sums, the clipping iteration with exact
// integer moments and the median split, the mode; thread 0 writes the mode
// and sigma to *back_out, *sig_out.
__device__ void guess_from_hist(int *hist, int *pfx, const MeshStat &bm, float *back_out, float *sig_out) {
    __shared__ long long red[3][GUESS_THREADS / 32];
    __shared__ int sh_lcut, sh_hcut, sh_go;
    const int nlevels = bm.nlevels;
    // exclusive prefix of the histogram: 17 consecutive bins per thread
    {
        constexpr int PER = (SX_QUANTIF_NMAXLEVELS + 2 + GUESS_THREADS - 1) / GUESS_THREADS;
        __shared__ int wsum[32];
        int base = threadIdx.x * PER, loc = 0;
        for (int k = 0; k < PER; k++)
            if (base + k < SX_QUANTIF_NMAXLEVELS + 2) loc += hist[base + k];
        int tot;
        int run = block_exclusive_scan(loc, wsum, tot);
        for (int k = 0; k < PER; k++)
            if (base + k < SX_QUANTIF_NMAXLEVELS + 2) {
                pfx[base + k] = run;
                run += hist[base + k];
            }
    }
    __syncthreads();

    int nlevelsm1 = nlevels - 1;
    double sig_ = 10.0 * nlevelsm1, sig1 = 1.0, mea = bm.mean, med = bm.mean;
    if (threadIdx.x == 0) {
        sh_lcut = 0;
        sh_hcut = nlevelsm1;
    }
    for (int n = 100;;) {
        if (threadIdx.x == 0) sh_go = (n-- && (sig_ >= 0.1) && (fabs(sig_ / sig1 - 1.0) > SX_EPS));
        __syncthreads();
        if (!sh_go) break;
        int lcut = sh_lcut, hcut = sh_hcut;
        // exact integer sums over [lcut, hcut]
        long long s0 = 0, s1 = 0, s2 = 0;
        for (int i = lcut + threadIdx.x; i <= hcut; i += GUESS_THREADS) {
            long long pv = hist[i];
            s0 += pv;
            s1 += pv * i;
            s2 += pv * i * (long long)i;
        }
        for (int o = 16; o > 0; o >>= 1) {
            s0 += __shfl_down_sync(0xffffffffu, s0, o);
            s1 += __shfl_down_sync(0xffffffffu, s1, o);
            s2 += __shfl_down_sync(0xffffffffu, s2, o);
        }
        if ((threadIdx.x & 31) == 0) {
            red[0][threadIdx.x >> 5] = s0;
            red[1][threadIdx.x >> 5] = s1;
            red[2][threadIdx.x >> 5] = s2;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            long long sum = 0, t1 = 0, t2 = 0;
            for (int k = 0; k < GUESS_THREADS / 32; k++) {
                sum += red[0][k];
                t1 += red[1][k];
                t2 += red[2][k];
            }
            // split of the two-pointer walk: smallest a with NOT(A(a) < B(nn-1-a))
            int nn = hcut - lcut + 1, lo = 0, hi = nn;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                int A = pfx[lcut + mid] - pfx[lcut];
                int B = pfx[hcut + 1] - pfx[hcut + 1 - (nn - 1 - mid)];
                if (A < B)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            int il = lcut + lo, ih = il - 1;
            unsigned long lowsum = (unsigned long)(pfx[il] - pfx[lcut]);
            unsigned long highsum = (unsigned long)(pfx[hcut + 1] - pfx[il]);
            double ftemp;
            sig1 = sig_;
            sig_ = (double)t2;
            mea = (double)t1;
            long hl = hist[il], hh = ih >= 0 ? hist[ih] : 0;
            med = ih >= 0 ? ((double)ih + 0.5 + ((double)highsum - lowsum) / (2.0 * (hl > hh ? hl : hh))) : 0.0;
            if (sum) {
                mea /= (double)sum;
                sig_ = sig_ / sum - mea * mea;
            }
            sig_ = sig_ > 0.0 ? sqrt(sig_) : 0.0;
            sh_lcut = (ftemp = med - 3.0 * sig_) > 0.0 ? (int)(ftemp > 0.0 ? ftemp + 0.5 : ftemp - 0.5) : 0;
            sh_hcut = (ftemp = med + 3.0 * sig_) < nlevelsm1 ? (int)(ftemp > 0.0 ? ftemp + 0.5 : ftemp - 0.5)
                                                               : nlevelsm1;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        float mean;
        // src/back.c:408: the C library abs(int) applied to the double sig
        if (abs((int)sig_) > 0.0) {
            if (fabs((mea - med) / sig_) < 0.3)
                mean = bm.qzero + (2.5 * med - 1.5 * mea) * bm.qscale;
            else
                mean = bm.qzero + med * bm.qscale;
        } else
            mean = bm.qzero + mea * bm.qscale;
        *back_out = mean;
        *sig_out = sig_ * bm.qscale;
    }
}

__global__ void __launch_bounds__(GUESS_THREADS) k_mesh_guess(const float *__restrict__ img, int w, int h, int bw,
                                                                int bh, int nbx, int nby,
                                                                const MeshStat *__restrict__ ms,
                                                                float *__restrict__ back, float *__restrict__ sig) {
    __shared__ int hist[SX_QUANTIF_NMAXLEVELS + 2];
    __shared__ int pfx[SX_QUANTIF_NMAXLEVELS + 2];   // pfx[i] = sum_{k<i} hist[k]
    int m = blockIdx.x;
    int mx = m % nbx, my = m / nbx;
    MeshStat bm = ms[m];
    if (bm.mean <= -SX_BIG) {
        if (threadIdx.x == 0) back[m] = sig[m] = -SX_BIG;
        return;
    }
    int x0 = mx * bw, y0 = my * bh;
    int mw = (mx == nbx - 1 && w % bw) ? w % bw : bw;
    int mh = (my == nby - 1 && h % bh) ? h % bh : bh;
    for (int i = threadIdx.x; i < SX_QUANTIF_NMAXLEVELS + 2; i += GUESS_THREADS) hist[i] = 0;
    __syncthreads();
    int nlevels = bm.nlevels;
    float qscale = bm.qscale;
    float cste = 0.499999 - bm.qzero / qscale;
    // one warp per mesh row, lanes along the row (no index division)
    for (int r = threadIdx.x >> 5; r < mh; r += GUESS_THREADS / 32) {
        const float *row = img + (size_t)(y0 + r) * w + x0;
        for (int x = threadIdx.x & 31; x < mw; x += 32) {
            float b = __ldg(row + x) / qscale + cste;
            if (b != b) continue;  // NaN: the host conversion yields INT_MIN
            int bin = (int)b;
            if (bin >= 0 && bin < nlevels) atomicAdd(&hist[bin], 1);
        }
    }
    __syncthreads();
    guess_from_hist(hist, pfx, bm, back + m, sig + m);
}

// ---------------------------------------------------------------------------
// backhisto + backguess with one warp per mesh, for meshes of fewer than
// 65536 pixels (no bin count reaches 2^16).  The histogram is kept as 16-bit
// counts, two per word, and summarised per chunk of 32 bins: the counts
// below each chunk (cp) and each chunk's first and second moments (c1, c2).
// A clipping iteration then reads the two partial chunks at the ends of its
// cut range and the chunk sums between them, and finds the median split from
// the chunk prefix and one chunk's scan, instead of walking the cut range.
// The integer sums, the split and the double arithmetic are those of
// guess_from_hist, so the mode and sigma are the same bits.
constexpr int GW_WARPS = 4;                        // meshes (warps) per CTA
constexpr int GW_CH = (SX_QUANTIF_NMAXLEVELS + 2 + 31) / 32;  // 32-bin chunks
constexpr int GW_WORDS = GW_CH * 16;              // 16-bit counts of GW_CH * 32 bins

struct GuessWarpSmem {
    long long c2[GW_CH];    // sum over the chunk of bin^2 * count
    int c1[GW_CH];          // sum over the chunk of bin * count (< 2^28)
    int cp[GW_CH + 1];      // counts of the bins below chunk c
    unsigned hw[GW_WORDS];  // bin b: bits 16 (b & 1) .. of word b >> 1
};

__device__ __forceinline__ int gw_hist(const GuessWarpSmem &S, int b) {
    return (int)((S.hw[b >> 1] >> ((b & 1) << 4)) & 0xffffu);
}

// counts of the bins below bin i (0 <= i <= 32 GW_CH), whole warp
__device__ __forceinline__ int gw_pfx(const GuessWarpSmem &S, int i, int lane) {
    const int c = i >> 5, r = i & 31;
    const int v = lane < r ? gw_hist(S, 32 * c + lane) : 0;
    return S.cp[c] + (int)__reduce_add_sync(0xffffffffu, (unsigned)v);
}

__global__ void __launch_bounds__(32 * GW_WARPS) k_mesh_guess_warp(const float *__restrict__ img, int w, int h, int bw,
                                                                    int bh, int nbx, int nby,
                                                                    const MeshStat *__restrict__ ms,
                                                                    float *__restrict__ back,
                                                                    float *__restrict__ sig) {
    __shared__ GuessWarpSmem smem[GW_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int m = blockIdx.x * GW_WARPS + wid;
    if (m >= nbx * nby) return;  // whole warp
    GuessWarpSmem &S = smem[wid];
    const MeshStat bm = ms[m];
    if (bm.mean <= -SX_BIG) {
        if (lane == 0) back[m] = sig[m] = -SX_BIG;
        return;
    }
    const int mx = m % nbx, my = m / nbx;
    const int x0 = mx * bw, y0 = my * bh;
    const int mw = (mx == nbx - 1 && w % bw) ? w % bw : bw;
    const int mh = (my == nby - 1 && h % bh) ? h % bh : bh;
    for (int i = lane; i < GW_WORDS; i += 32) S.hw[i] = 0u;
    __syncwarp();
    const int nlevels = bm.nlevels;
    const float qscale = bm.qscale;
    const float cste = 0.499999 - bm.qzero / qscale;
    // the mesh's pixels k = lane, lane + 32, ... in row-major order, GW_LOADS
    // loads in flight per lane; (row, col) of k advance by (drow, dcol) per 32
    {
        constexpr int GW_LOADS = 16;
        const int npx = mw * mh;
        const int drow = 32 / mw, dcol = 32 - drow * mw;
        int row = lane / mw, col = lane - row * mw;
        for (int k0 = 0; k0 < npx; k0 += 32 * GW_LOADS) {
            float v[GW_LOADS];
#pragma unroll
            for (int g = 0; g < GW_LOADS; g++) {
                // beyond the mesh: NaN, which the histogram skips as it does a NaN pixel
                v[g] = k0 + 32 * g + lane < npx ? __ldg(img + (size_t)(y0 + row) * w + x0 + col)
                                                : __int_as_float(0x7fffffff);
                row += drow;
                col += dcol;
                if (col >= mw) {
                    col -= mw;
                    row++;
                }
            }
#pragma unroll
            for (int g = 0; g < GW_LOADS; g++) {
                const float b = v[g] / qscale + cste;
                if (b != b) continue;  // NaN: the host conversion yields INT_MIN
                const int bin = (int)b;
                if (bin >= 0 && bin < nlevels) atomicAdd(&S.hw[bin >> 1], 1u << ((bin & 1) << 4));
            }
        }
    }
    __syncwarp();
    // chunk sums: lane owns chunks lane, lane + 32, ...; words read in an
    // order rotated by the lane (at most two lanes on a bank)
    int carry = 0;
    for (int c0 = 0; c0 < GW_CH; c0 += 32) {
        const int c = c0 + lane;
        int s0 = 0, k1 = 0, k2 = 0;
        if (c < GW_CH) {
#pragma unroll 4
            for (int t = 0; t < 16; t++) {
                const int tw = (t + lane) & 15;
                const unsigned wv = S.hw[16 * c + tw];
                const int n0 = (int)(wv & 0xffffu), n1 = (int)(wv >> 16), k = 2 * tw;
                s0 += n0 + n1;
                k1 += k * n0 + (k + 1) * n1;
                k2 += k * k * n0 + (k + 1) * (k + 1) * n1;
            }
            S.c1[c] = 32 * c * s0 + k1;
            S.c2[c] = (long long)(32 * c) * (32 * c) * s0 + (long long)(64 * c) * k1 + k2;
        }
        int inc = s0;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        if (c < GW_CH) S.cp[c] = carry + inc - s0;
        carry += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) S.cp[GW_CH] = carry;
    __syncwarp();

    // src/back.c:347-432, every lane computing the same values
    const int nlevelsm1 = nlevels - 1;
    double sig_ = 10.0 * nlevelsm1, sig1 = 1.0, mea = bm.mean, med = bm.mean;
    int lcut = 0, hcut = nlevelsm1;
    for (int n = 100;;) {
        if (!(n-- && (sig_ >= 0.1) && (fabs(sig_ / sig1 - 1.0) > SX_EPS))) break;
        const int nn = hcut - lcut + 1;
        // exact integer sums over [lcut, hcut]
        long long sum = 0, t1 = 0, t2 = 0;
        int il = lcut;
        const int base = gw_pfx(S, lcut, lane);
        if (nn > 0) {
            const int cl = lcut >> 5, ch = hcut >> 5;
            int p0 = 0, p1 = 0;
            long long p2 = 0;
            {
                const int b = 32 * cl + lane;
                if (b >= lcut && b <= hcut) {
                    const int v = gw_hist(S, b);
                    p0 += v;
                    p1 += b * v;
                    p2 += (long long)b * b * v;
                }
            }
            if (ch != cl) {
                const int b = 32 * ch + lane;
                if (b <= hcut) {
                    const int v = gw_hist(S, b);
                    p0 += v;
                    p1 += b * v;
                    p2 += (long long)b * b * v;
                }
            }
            for (int c = cl + 1 + lane; c < ch; c += 32) {
                p0 += S.cp[c + 1] - S.cp[c];
                p1 += S.c1[c];
                p2 += S.c2[c];
            }
            sum = (int)__reduce_add_sync(0xffffffffu, (unsigned)p0);
            t1 = (int)__reduce_add_sync(0xffffffffu, (unsigned)p1);
            for (int o = 16; o > 0; o >>= 1) p2 += __shfl_xor_sync(0xffffffffu, p2, o);
            t2 = p2;
            // split of the two-pointer walk: the smallest bin i >= lcut with
            // pfx(i) + pfx(i + 1) >= sum + 2 pfx(lcut) (bin hcut qualifies);
            // first the chunk whose last bin qualifies, then the bin in it
            const int T = (int)sum + 2 * base;
            int cstar = ch;
            for (int c0 = cl; c0 <= ch; c0 += 32) {
                const int c = c0 + lane;
                const bool ok = c <= ch && 2 * S.cp[c + 1] - gw_hist(S, 32 * c + 31) >= T;
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (bal) {
                    cstar = c0 + __ffs(bal) - 1;
                    break;
                }
            }
            const int hk = gw_hist(S, 32 * cstar + lane);
            int inc = hk;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += v;
            }
            const int pk = S.cp[cstar] + inc - hk;  // pfx(32 cstar + lane)
            const unsigned bal = __ballot_sync(0xffffffffu, 2 * pk + hk >= T);
            il = max(32 * cstar + (bal ? __ffs(bal) - 1 : 31), lcut);
        }
        const int ih = il - 1;
        const int pil = gw_pfx(S, il, lane), phc = gw_pfx(S, hcut + 1, lane);
        const unsigned long lowsum = (unsigned long)(pil - base);
        const unsigned long highsum = (unsigned long)(phc - pil);
        sig1 = sig_;
        sig_ = (double)t2;
        mea = (double)t1;
        const long hl = gw_hist(S, il), hh = ih >= 0 ? gw_hist(S, ih) : 0;
        med = ih >= 0 ? ((double)ih + 0.5 + ((double)highsum - lowsum) / (2.0 * (hl > hh ? hl : hh))) : 0.0;
        if (sum) {
            mea /= (double)sum;
            sig_ = sig_ / sum - mea * mea;
        }
        sig_ = sig_ > 0.0 ? sqrt(sig_) : 0.0;
        double ftemp;
        lcut = (ftemp = med - 3.0 * sig_) > 0.0 ? (int)(ftemp > 0.0 ? ftemp + 0.5 : ftemp - 0.5) : 0;
        hcut = (ftemp = med + 3.0 * sig_) < nlevelsm1 ? (int)(ftemp > 0.0 ? ftemp + 0.5 : ftemp - 0.5) : nlevelsm1;
    }
    if (lane == 0) {
        float mean;
        // src/back.c:408: the C library abs(int) applied to the double sig
        if (abs((int)sig_) > 0.0) {
            if (fabs((mea - med) / sig_) < 0.3)
                mean = bm.qzero + (2.5 * med - 1.5 * mea) * bm.qscale;
            else
                mean = bm.qzero + med * bm.qscale;
        } else
            mean = bm.qzero + mea * bm.qscale;
        back[m] = mean;
        sig[m] = sig_ * bm.qscale;
    }
}

// ---------------------------------------------------------------------------
// BACKPHOTO_TYPE LOCAL, src/back.c:568-660 (localback): the mode of the
// background-subtracted pixels in a rectangular annulus, BACKPHOTO_THICK
// wide, around the object's box widened by a quarter of its size.  The
// reference collects the annulus pixels (per row the left and right strips,
// then the rows above the box, then the rows below) and runs backstat (two
// sequential double passes in that order), the histogram and backguess.
// ---------------------------------------------------------------------------
struct LocalBox {
    int ok, ixmin, ixmax, iymin, iymax, bxmin, bxmax, bymin, bymax;
};

__device__ __forceinline__ LocalBox local_box(int xmin, int xmax, int ymin, int ymax, int w, int h, int pbs) {
    LocalBox B;
    const int oxsize = xmax - xmin + 1, oysize = ymax - ymin + 1;
    const int bxnml = oxsize < w / 2 ? oxsize / 4 : (w - oxsize) / 4;
    const int bynml = oysize < h / 2 ? oysize / 4 : (h - oysize) / 4;
    B.ixmin = xmin - bxnml;
    B.ixmax = xmax + 1 + bxnml;
    B.iymin = ymin - bynml;
    B.iymax = ymax + 1 + bynml;
    B.bxmin = B.ixmin - pbs;
    B.bxmax = B.ixmax + pbs;
    B.bymin = B.iymin - pbs;
    B.bymax = B.iymax + pbs;
    B.ok = B.bymin >= 0 && B.bymax < h && B.bxmin >= 0 && B.bxmax < w;
    return B;
}

// the annulus pixels in the reference's collection order
template <class F>
__device__ __forceinline__ void local_visit(const float *__restrict__ sub, int w, const LocalBox &B, int pbs, F f) {
    for (int y = B.bymin; y < B.bymax; y++) {
        const float *row = sub + (size_t)y * w;
        for (int x = B.bxmin; x < B.bxmin + pbs; x++) f(row[x]);
        for (int x = B.ixmax; x < B.ixmax + pbs; x++) f(row[x]);
    }
    for (int y = B.bymin; y < B.iymin; y++)
        for (int x = B.ixmin; x < B.ixmax; x++) f(sub[(size_t)y * w + x]);
    for (int y = B.iymax; y < B.bymax; y++)
        for (int x = B.ixmin; x < B.ixmax; x++) f(sub[(size_t)y * w + x]);
}

// one thread per object: backstat over the valid annulus pixels (one mesh of
// one column); nlevels = -1 marks "no local background" (annulus outside the
// frame, or no valid pixel)
__global__ void k_local_stat(const float *__restrict__ sub, int w, int h, int pbs, const int *__restrict__ xmin,
                             const int *__restrict__ xmax, const int *__restrict__ ymin,
                             const int *__restrict__ ymax, int n, const int *n_dev, MeshStat *__restrict__ ls) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= sx_count(n, n_dev)) return;
    MeshStat s;
    s.mean = s.sigma = s.lcut = s.hcut = s.qzero = s.qscale = 0.f;
    s.nlevels = -1;
    s.npix = 0;
    const LocalBox B = local_box(xmin[o], xmax[o], ymin[o], ymax[o], w, h, pbs);
    if (!B.ok) {
        ls[o] = s;
        return;
    }
    const double step = sqrt(2 / SX_PI) * SX_QUANTIF_NSIGMA / SX_QUANTIF_AMIN;
    double mean = 0.0, sigma = 0.0, sig;
    int npix = 0;
    // a pixel left out adds +0.0 (the sums are never -0.0), see mesh_stat_seq
    local_visit(sub, w, B, pbs, [&](float p) {
        const double pix = p;
        const bool in = pix > -SX_BIG;
        mean += in ? pix : 0.0;
        sigma += in ? pix * pix : 0.0;
        npix += in;
    });
    if (!npix) {
        ls[o] = s;
        return;
    }
    mean /= (double)npix;
    sigma = (sig = sigma / npix - mean * mean) > 0.0 ? sqrt(sig) : 0.0;
    const float lcut = s.lcut = (float)(mean - 2.0 * sigma);
    const float hcut = s.hcut = (float)(mean + 2.0 * sigma);
    mean = sigma = 0.0;
    int npix2 = 0;
    local_visit(sub, w, B, pbs, [&](float p) {
        const double pix = p;
        const bool in = pix > -SX_BIG && pix <= hcut && pix >= lcut;
        mean += in ? pix : 0.0;
        sigma += in ? pix * pix : 0.0;
        npix2 += in;
    });
    s.npix = npix2;
    mean /= (double)npix2;
    sig = sigma / npix2 - mean * mean;
    sigma = sig > 0.0 ? sqrt(sig) : 0.0;
    s.mean = mean;
    s.sigma = sigma;
    if ((s.nlevels = (int)(step * npix2 + 1)) > SX_QUANTIF_NMAXLEVELS) s.nlevels = SX_QUANTIF_NMAXLEVELS;
    s.qscale = sigma > 0.0 ? 2 * SX_QUANTIF_NSIGMA * sigma / s.nlevels : 1.0;
    s.qzero = mean - SX_QUANTIF_NSIGMA * sigma;
    ls[o] = s;
}

// one CTA per object: the annulus histogram (integer counts, any order) and
// backguess; dbkg = its mode, 0 without a local background
__global__ void __launch_bounds__(GUESS_THREADS) k_local_guess(const float *__restrict__ sub, int w, int h, int pbs,
                                                                 const int *__restrict__ xmin,
                                                                 const int *__restrict__ xmax,
                                                                 const int *__restrict__ ymin,
                                                                 const int *__restrict__ ymax, int n,
                                                                 const int *n_dev,
                                                                 const MeshStat *__restrict__ ls, float *dbkg) {
    __shared__ int hist[SX_QUANTIF_NMAXLEVELS + 2];
    __shared__ int pfx[SX_QUANTIF_NMAXLEVELS + 2];
    const int o = blockIdx.x;
    if (o >= sx_count(n, n_dev)) return;
    const MeshStat bm = ls[o];
    if (bm.nlevels < 0) {
        if (threadIdx.x == 0) dbkg[o] = 0.0f;
        return;
    }
    const LocalBox B = local_box(xmin[o], xmax[o], ymin[o], ymax[o], w, h, pbs);
    for (int i = threadIdx.x; i < SX_QUANTIF_NMAXLEVELS + 2; i += GUESS_THREADS) hist[i] = 0;
    __syncthreads();
    const int nlevels = bm.nlevels;
    const float qscale = bm.qscale, cste = 0.499999 - bm.qzero / qscale;
    auto bin_of = [&](float p) {
        if (!(p > -SX_BIG)) return;
        const float b = p / qscale + cste;
        if (b != b) return;
        const int bin = (int)b;
        if (bin >= 0 && bin < nlevels) atomicAdd(&hist[bin], 1);
    };
    const int sw = 2 * pbs, rows = B.bymax - B.bymin, iw = B.ixmax - B.ixmin;
    for (int i = threadIdx.x; i < rows * sw; i += GUESS_THREADS) {
        const int r = i / sw, c = i - r * sw;
        bin_of(sub[(size_t)(B.bymin + r) * w + (c < pbs ? B.bxmin + c : B.ixmax + c - pbs)]);
    }
    const int nt = B.iymin - B.bymin, nb2 = B.bymax - B.iymax;
    for (int i = threadIdx.x; i < (nt + nb2) * iw; i += GUESS_THREADS) {
        const int r = i / iw, c = i - r * iw;
        const int y = r < nt ? B.bymin + r : B.iymax + (r - nt);
        bin_of(sub[(size_t)y * w + B.ixmin + c]);
    }
    __syncthreads();
    float sg;
    guess_from_hist(hist, pfx, bm, dbkg + o, &sg);
}

// src/back.c:455-480: bad meshes take the mean of the nearest valid meshes.
// Writes back2 (all meshes) and fixes sigma in place for bad meshes.
__global__ void k_mesh_badfill(const float *__restrict__ back, float *__restrict__ sigma, float *__restrict__ back2,
                               int nx, int ny) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return;
    float b = back[i];
    back2[i] = b;
    if (b > -SX_BIG) return;
    int px = i % nx, py = i / nx;
    float d2min = SX_BIG, val = 0.f, sval = 0.f, d2;
    int nmin = 0;
    for (int j = 0, y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++, j++)
            if (back[j] > -SX_BIG) {
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

__device__ __forceinline__ float median_small(float *v, int n) {
    for (int i = 1; i < n; i++) {
        float t = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > t) {
            v[j + 1] = v[j];
            j--;
        }
        v[j + 1] = t;
    }
    return n & 1 ? v[n / 2] : (float)((v[n / 2 - 1] + v[n / 2]) / 2.0);
}

// src/back.c:482-533: median filter of the mesh maps (window shrunk at edges)
__global__ void k_mesh_median(const float *__restrict__ back, const float *__restrict__ sigma,
                              float *__restrict__ back3, float *__restrict__ sigma3, int nx, int ny, int npx,
                              int npy, float fthresh) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx * ny) return;
    int px = i % nx, py = i / nx;
    int npx2 = nx - px - 1, npy2 = ny - py - 1;
    if (npx2 > npx) npx2 = npx;
    if (npx2 > px) npx2 = px;
    if (npy2 > npy) npy2 = npy;
    if (npy2 > py) npy2 = py;
    float bm[121], sm[121];
    int n = 0;
    for (int dy = -npy2; dy <= npy2; dy++)
        for (int dx = -npx2; dx <= npx2; dx++) {
            int j = (py + dy) * nx + px + dx;
            bm[n] = back[j];
            sm[n++] = sigma[j];
        }
    float med = median_small(bm, n);
    if (fabs(med - back[i]) >= fthresh) {
        back3[i] = med;
        sigma3[i] = median_small(sm, n);
    } else {
        back3[i] = back[i];
        sigma3[i] = sigma[i];
    }
}

// k-th smallest (0-based) of n floats (orderable keys), single CTA radix select
__device__ unsigned select_kth(const float *v, int n, int k, unsigned lowkey, unsigned *hist) {
    unsigned prefix = 0, mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            unsigned key = f2ord(v[i]);
            if (key < lowkey) continue;
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 255], 1u);
        }
        __syncthreads();
        __shared__ unsigned s_digit, s_k;
        if (threadIdx.x < 32) {
            // the digit holding rank k: lane l owns bins 8l..8l+7, a warp scan
            // of the lane totals finds the owner, the owner its bin
            const int lane = threadIdx.x;
            unsigned c[8], tot = 0;
#pragma unroll
            for (int t = 0; t < 8; t++) tot += (c[t] = hist[lane * 8 + t]);
            unsigned incl = tot;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const unsigned sel = __ballot_sync(0xffffffffu, incl > (unsigned)k);
            const int owner = sel ? __ffs(sel) - 1 : 31;
            if (lane == owner) {
                unsigned below = incl - tot, d = lane * 8;
#pragma unroll
                for (int t = 0; t < 8; t++)
                    if (d == (unsigned)(lane * 8 + t) && below + c[t] <= (unsigned)k && t < 7) {
                        below += c[t];
                        d++;
                    }
                s_digit = d;
                s_k = k - below;
            }
        }
        __syncthreads();
        prefix |= s_digit << shift;
        mask |= 255u << shift;
        k = s_k;
        __syncthreads();
    }
    return prefix;
}

// global medians of the filtered maps (src/back.c:536-557), one CTA
__global__ void k_back_medians(const float *__restrict__ back3, const float *__restrict__ sigma3, int nb,
                               FrameScalars *sc, int back_type, float back_value, int thresh_type,
                               double dthr, double athr) {
    __shared__ unsigned hist[256];
    __shared__ unsigned s_npos;
    float med[2];
    for (int q = 0; q < 2; q++) {
        const float *v = q ? sigma3 : back3;
        if (nb & 1) {
            med[q] = ord2f(select_kth(v, nb, nb / 2, 0u, hist));
        } else {
            float a = ord2f(select_kth(v, nb, nb / 2 - 1, 0u, hist));
            float b = ord2f(select_kth(v, nb, nb / 2, 0u, hist));
            med[q] = (float)((a + b) / 2.0);
        }
    }
    float backsig = med[1];
    if (backsig <= 0.0) {
        // median of the strictly positive sigmas, else 1.0
        if (threadIdx.x == 0) s_npos = 0;
        __syncthreads();
        unsigned c = 0;
        for (int i = threadIdx.x; i < nb; i += blockDim.x) c += sigma3[i] > 0.0f;
        atomicAdd(&s_npos, c);
        __syncthreads();
        int npos = (int)s_npos;
        unsigned low = f2ord(__uint_as_float(1u));  // smallest positive float
        if (npos > 0 && npos < nb) {
            if (npos & 1)
                backsig = ord2f(select_kth(sigma3, nb, npos / 2, low, hist));
            else {
                float a = ord2f(select_kth(sigma3, nb, npos / 2 - 1, low, hist));
                float b = ord2f(select_kth(sigma3, nb, npos / 2, low, hist));
                backsig = (float)((a + b) / 2.0);
            }
        } else
            backsig = 1.0;
    }
    if (threadIdx.x == 0) {
        sc->backmean = back_type == 1 ? back_value : med[0];
        sc->backsig = backsig;
        if (thresh_type == 1) {
            sc->dthresh = (float)dthr;
            sc->thresh = (float)athr;
        } else {
            sc->dthresh = (float)(dthr * backsig);
            sc->thresh = (float)(athr * backsig);
        }
        sc->e0cd = fexpo(sc->dthresh);
    }
}

// src/back.c:739-773 (makebackspline), one thread per mesh column
__global__ void k_back_spline(const float *__restrict__ map, float *__restrict__ dmap, float *__restrict__ u,
                              int nbx, int nby) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nbx) return;
    float temp;
    if (nby > 1) {
        // the previous step's values are carried in registers, not read back
        // from the arrays just written (same operations, same order)
        float *ux = u + (size_t)x * nby;
        float dprev = 0.0f, uprev = 0.0f;
        dmap[x] = ux[0] = 0.0;
        for (int y = 1; y < nby - 1; y++) {
            temp = -1 / (dprev + 4);
            dmap[(size_t)y * nbx + x] = dprev = temp;
            temp *= uprev - 6 * (map[(size_t)(y + 1) * nbx + x] + map[(size_t)(y - 1) * nbx + x]
                                 - 2 * map[(size_t)y * nbx + x]);
            ux[y] = uprev = temp;
        }
        dmap[(size_t)(nby - 1) * nbx + x] = 0.0;
        float dnext = 0.0f;
        for (int y = nby - 2; y >= 1; y--)
            dmap[(size_t)y * nbx + x] = dnext = (dmap[(size_t)y * nbx + x] * dnext + ux[y]) / 6.0;
    } else
        dmap[x] = 0.0;
}

// src/back.c:938-1040 (backrmsline): the rms map of every pixel from the
// row nodes of the sigma map, the same x interpolation as the background
// square: write rms * rms (the variance of WEIGHT_TYPE BACKGROUND)
__global__ void k_rms_map(const float *__restrict__ node, const float *__restrict__ dnode, const int *__restrict__ colk,
                          const float *__restrict__ coldx, int nbx, int w, long long n, float *__restrict__ out,
                          int square) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int y = (int)(p / w), x = (int)(p - (long long)y * w);
    const float *nd = node + (size_t)y * nbx, *dnd = dnode + (size_t)y * nbx;
    float v;
    if (nbx <= 1) {
        v = nd[0];
    } else {
        const int k = colk[x];
        const float dx = coldx[x], cdx = 1 - dx;
        v = (float)(cdx * (nd[k] + (cdx * cdx - 1) * dnd[k]) + dx * (nd[k + 1] + (dx * dx - 1) * dnd[k + 1]));
    }
    out[p] = square ? v * v : v;
}

// src/back.c:790-862: y-interpolated nodes of every image row and their
// x-direction second derivatives (one thread per row)
__global__ void k_row_nodes(const float *__restrict__ back, const float *__restrict__ dback, int nbx, int nby,
                            int backh, int h, float *__restrict__ node, float *__restrict__ dnode,
                            float *__restrict__ u) {
    int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= h) return;
    float *nd = node + (size_t)y * nbx, *dnd = dnode + (size_t)y * nbx, *uu = u + (size_t)y * nbx;
    if (nby > 1) {
        int yl;
        float dy, dy3, cdy, cdy3, temp;
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
        const float *blo = back + (size_t)nbx * yl, *bhi = blo + nbx;
        const float *dblo = dback + (size_t)nbx * yl, *dbhi = dblo + nbx;
        for (int x = 0; x < nbx; x++) nd[x] = cdy * blo[x] + dy * bhi[x] + cdy3 * dblo[x] + dy3 * dbhi[x];
        if (nbx > 1) {
            // node values recomputed and the previous step carried in
            // registers instead of read back from this thread's own stores
            // (the same operations in the same order, so the same values)
            auto node_at = [&](int x) { return cdy * blo[x] + dy * bhi[x] + cdy3 * dblo[x] + dy3 * dbhi[x]; };
            float dprev = 0.0f, uprev = 0.0f, nm = node_at(0), n0 = node_at(1);
            dnd[0] = uu[0] = 0.0;
            for (int x = 1; x < nbx - 1; x++) {
                const float np = node_at(x + 1);
                temp = -1 / (dprev + 4);
                dnd[x] = dprev = temp;
                temp *= uprev - 6 * (np + nm - 2 * n0);
                uu[x] = uprev = temp;
                nm = n0;
                n0 = np;
            }
            dnd[nbx - 1] = 0.0;
            float dnext = 0.0f;
            for (int x = nbx - 2; x >= 1; x--) dnd[x] = dnext = (dnd[x] * dnext + uu[x]) / 6.0;
        } else
            dnd[0] = 0.0;
    } else {
        for (int x = 0; x < nbx; x++) {
            nd[x] = back[x];
            dnd[x] = dback[x];
        }
    }
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// weight maps: blank the unusable pixels, then (after the background) the
// scale factor sigfac and the calibrated variance map
// ---------------------------------------------------------------------------
__global__ void k_weight_mask(const float *__restrict__ img, const float *__restrict__ wmap, int wtype,
                              float *__restrict__ imgm, long long n) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) imgm[p] = sx_rel_var(__ldg(wmap + p), wtype) < 1e30f ? __ldg(img + p) : -1e30f;
}

// one warp per mesh: exact mean of the relative variance over its usable
// pixels; ratio = mesh rms / sqrt(mean) for a usable mesh, -1 otherwise
__global__ void k_weight_ratio(const float *__restrict__ wmap, int wtype, int w, int h, int bw, int bh, int nbx,
                               int nby, const float *__restrict__ sigma, float *__restrict__ ratio) {
    const int lane = threadIdx.x & 31;
    const int m = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (m >= nbx * nby) return;
    int x0, y0, mw, mh;
    mesh_geometry(m, w, h, bw, bh, nbx, nby, x0, y0, mw, mh);
    XSum sv;
    xs_init(sv);
    int n = 0;
    for (int y = 0; y < mh; y++) {
        const float *row = wmap + (size_t)(y0 + y) * w + x0;
        for (int x = lane; x < mw; x += 32) {
            const float r = sx_rel_var(__ldg(row + x), wtype);
            if (r < 1e30f) {
                xs_add(sv, r);
                n++;
            }
        }
    }
    sv = xs_warp_sum(sv);
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if (lane) return;
    float rt = -1.0f;
    if (!((float)n < (float)(mw * mh * SX_BACK_MINGOODFRAC))) {
        const double vmean = xs_double(sv) / n;
        const float sm = sigma[m];
        if (vmean > 0.0 && sm > 0.0f) rt = (float)(sm / sqrt(vmean));
    }
    ratio[m] = rt;
}

// sigfac: median of the usable meshes' ratios (hmedian, src/misc.c:30), 1 if none
__global__ void k_weight_sigfac(const float *__restrict__ ratio, int nb, FrameScalars *sc) {
    __shared__ unsigned hist[256];
    __shared__ unsigned s_npos;
    if (threadIdx.x == 0) s_npos = 0;
    __syncthreads();
    unsigned c = 0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) c += ratio[i] > 0.0f;
    atomicAdd(&s_npos, c);
    __syncthreads();
    const int npos = (int)s_npos;
    const unsigned low = f2ord(__uint_as_float(1u));  // smallest positive float
    float f = 1.0f;
    if (npos & 1) {
        f = ord2f(select_kth(ratio, nb, npos / 2, low, hist));
    } else if (npos) {
        const float a = ord2f(select_kth(ratio, nb, npos / 2 - 1, low, hist));
        const float b = ord2f(select_kth(ratio, nb, npos / 2, low, hist));
        f = (float)((a + b) / 2.0);
    }
    if (threadIdx.x == 0) sc->sigfac = f;
}

__global__ void k_weight_var(const float *__restrict__ wmap, int wtype, const FrameScalars *sc,
                             float *__restrict__ wvar, long long n) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const float sigfac = sc->sigfac, sigfac2 = sigfac * sigfac;
    if (p < n) wvar[p] = sx_calib_var(__ldg(wmap + p), wtype, sigfac2);
}

void launch_weight_mask(const float *img, const float *wmap, int wtype, float *imgm, long long n, cudaStream_t st) {
    if (n > 0) k_weight_mask<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(img, wmap, wtype, imgm, n);
}

// after launch_background: sigfac from the filtered mesh rms map, then the
// calibrated variance of every pixel
void launch_weight_var(const BackBufs &B, const float *wmap, const FrameParams &P, float *ratio, float *wvar,
                       FrameScalars *d_sc, cudaStream_t st) {
    const int nb = P.nbx * P.nby;
    const long long n = (long long)P.w * P.h;
    if (P.wtype != 2) {
        k_weight_ratio<<<(nb + 3) / 4, 128, 0, st>>>(wmap, P.wtype, P.w, P.h, P.bw, P.bh, P.nbx, P.nby, B.sigma3,
                                                     ratio);
        k_weight_sigfac<<<1, 1024, 0, st>>>(ratio, nb, d_sc);
    }
    k_weight_var<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(wmap, P.wtype, d_sc, wvar, n);
}

void launch_background(BackBufs &B, const float *img, const FrameParams &P, FrameScalars *d_sc,
                       cudaStream_t st, int &launches) {
    int nb = P.nbx * P.nby;
    // row-band kernel when BAND_STAGES rows of 32 meshes fit in 200 KB of
    // shared memory
    const bool vec = (P.w % 4) == 0 && (P.bw % 4) == 0 && ((uintptr_t)img & 15) == 0;
    int stride;
    if (vec) {
        stride = (P.bw + 3) & ~3;
        if (((stride >> 2) & 1) == 0) stride += 4;  // stride / 4 odd
    } else {
        stride = P.bw | 1;  // odd
    }
    const size_t band_bytes = (size_t)BAND_STAGES * 32 * stride * sizeof(float);
    constexpr int BAND_SMEM_MAX = 200 * 1024;
    if (band_bytes <= BAND_SMEM_MAX) {
        // the shared memory limit of both instances, once per device (host
        // threads of a batch may get here at the same time)
        static DevCache attr_set;
        attr_set.get([](int) {
            cudaFuncSetAttribute(k_mesh_stat_band<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, BAND_SMEM_MAX);
            cudaFuncSetAttribute(k_mesh_stat_band<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, BAND_SMEM_MAX);
            return 1;
        });
        dim3 grid((P.nbx + 31) / 32, P.nby);
        if (vec)
            k_mesh_stat_band<true><<<grid, 32, band_bytes, st>>>(img, P.w, P.h, P.bw, P.bh, P.nbx, P.nby, stride, B.ms);
        else
            k_mesh_stat_band<false><<<grid, 32, band_bytes, st>>>(img, P.w, P.h, P.bw, P.bh, P.nbx, P.nby, stride,
                                                                   B.ms);
    } else {
        k_mesh_stat<<<(nb + 127) / 128, 128, 0, st>>>(img, P.w, P.h, P.bw, P.bh, P.nbx, P.nby, B.ms);
    }
    if ((long long)P.bw * P.bh < 65536)
        k_mesh_guess_warp<<<(nb + GW_WARPS - 1) / GW_WARPS, 32 * GW_WARPS, 0, st>>>(img, P.w, P.h, P.bw, P.bh, P.nbx,
                                                                                   P.nby, B.ms, B.back, B.sigma);
    else
        k_mesh_guess<<<nb, GUESS_THREADS, 0, st>>>(img, P.w, P.h, P.bw, P.bh, P.nbx, P.nby, B.ms, B.back, B.sigma);
    k_mesh_badfill<<<(nb + 127) / 128, 128, 0, st>>>(B.back, B.sigma, B.back2, P.nbx, P.nby);
    k_mesh_median<<<(nb + 127) / 128, 128, 0, st>>>(B.back2, B.sigma, B.back3, B.sigma3, P.nbx, P.nby, P.nfx / 2,
                                                   P.nfy / 2, P.fthresh);
    k_back_medians<<<1, 1024, 0, st>>>(B.back3, B.sigma3, nb, d_sc, P.back_type, P.back_value, P.thresh_type,
                                       P.detect_thresh, P.analysis_thresh);
    k_back_spline<<<(P.nbx + 127) / 128, 128, 0, st>>>(B.back3, B.dback, B.u, P.nbx, P.nby);
    k_row_nodes<<<(P.h + 127) / 128, 128, 0, st>>>(B.back3, B.dback, P.nbx, P.nby, P.bh, P.h, B.rownode,
                                                  B.rowdnode, B.rowu);
    launches += 7;
}

}  // namespace sx
