// prim.cu -- device-wide exclusive scan and stable LSD radix sort of
// (key, value) pairs, written for this library (no CUB/Thrust/CUDPP).
//
// These replace the CUDPP cudppScan / cudppCompact / cudppRadixSort calls of
// the reference (src/cuda/cudadetection.cu:720-1072, cudadeblend.cu:792-1901).
#include "prim.cuh"

namespace sx {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// block-wide exclusive scan of one int per thread; returns the block total
__device__ __forceinline__ int block_exclusive_scan(int v, int *sh_warp, int &total) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int s = lane < nw ? sh_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh_warp[lane] = s;
    }
    __syncthreads();
    int base = wid ? sh_warp[wid - 1] : 0;
    total = sh_warp[nw - 1];
    __syncthreads();
    return base + x - v;
}

// The element count of a scan or sort: n, or, when the count is only known on
// the device (a launch sized before the count exists, as in a captured graph),
// the smaller of n and *n_dev.
__device__ __forceinline__ int dev_count(int n, const int *n_dev) { return n_dev ? min(n, max(*n_dev, 0)) : n; }

__global__ void k_tile_sums(const int *__restrict__ in, int n, int *__restrict__ sums, const int *n_dev) {
    __shared__ int sh[32];
    n = dev_count(n, n_dev);
    long long base = (long long)blockIdx.x * SCAN_TILE;
    int acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        if (i < n) acc += in[i];
    }
    int tot;
    block_exclusive_scan(acc, sh, tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_tile_scan(const int *__restrict__ in, int *__restrict__ out, int n,
                            const int *__restrict__ offs, int *total, const int *n_dev) {
    __shared__ int sh[32];
    n = dev_count(n, n_dev);
    long long base = (long long)blockIdx.x * SCAN_TILE;
    int v[SCAN_ITEMS], acc = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        v[k] = i < n ? in[i] : 0;
        acc += v[k];
    }
    int tot;
    int pre = block_exclusive_scan(acc, sh, tot) + (offs ? offs[blockIdx.x] : 0);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        long long i = base + (long long)threadIdx.x * SCAN_ITEMS + k;
        if (i < n) out[i] = pre;
        pre += v[k];
    }
    if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *total = pre;
}

size_t scan_temp_ints(long long n) {
    size_t t = 0;
    while (n > SCAN_TILE) {
        n = (n + SCAN_TILE - 1) / SCAN_TILE;
        t += 2 * n + 2;
    }
    return t + 2;
}

// out[i] = sum_{j<i} in[j]; *total (device, may be NULL) = sum of all.
// in and out may alias.  tmp: scan_temp_ints(n) ints.  n_dev (device, may
// be NULL): the count, at most n, when only the device knows it; the launch
// is sized for n.
void exclusive_scan(const int *in, int *out, long long n, int *total, int *tmp, cudaStream_t st, const int *n_dev) {
    if (n <= 0) {
        if (total) cudaMemsetAsync(total, 0, sizeof(int), st);
        return;
    }
    int nt = (int)((n + SCAN_TILE - 1) / SCAN_TILE);
    if (nt == 1) {
        k_tile_scan<<<1, SCAN_THREADS, 0, st>>>(in, out, (int)n, nullptr, total, n_dev);
        return;
    }
    int *sums = tmp, *offs = tmp + nt;
    k_tile_sums<<<nt, SCAN_THREADS, 0, st>>>(in, (int)n, sums, n_dev);
    exclusive_scan(sums, offs, nt, nullptr, tmp + 2 * nt + 2, st, nullptr);
    k_tile_scan<<<nt, SCAN_THREADS, 0, st>>>(in, out, (int)n, offs, total, n_dev);
}

// ---------------------------------------------------------------------------
// radix sort
// ---------------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;                 // per thread
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr int RS_WARP_TILE = RS_TILE / RS_WARPS;
constexpr int RS_BITS = 8;
constexpr int RS_DIGITS = 1 << RS_BITS;

__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const unsigned *__restrict__ keys, int n, int shift,
                                                          int ntiles, int *__restrict__ hist, const int *n_dev) {
    __shared__ int h[RS_DIGITS];
    n = dev_count(n, n_dev);
    for (int i = threadIdx.x; i < RS_DIGITS; i += RS_THREADS) h[i] = 0;
    __syncthreads();
    long long base = (long long)blockIdx.x * RS_TILE;
    for (int k = 0; k < RS_ITEMS; k++) {
        long long i = base + (long long)k * RS_THREADS + threadIdx.x;
        if (i < n) atomicAdd(&h[(keys[i] >> shift) & (RS_DIGITS - 1)], 1);
    }
    __syncthreads();
    // digit-major layout: hist[d * ntiles + tile]
    for (int d = threadIdx.x; d < RS_DIGITS; d += RS_THREADS) hist[(long long)d * ntiles + blockIdx.x] = h[d];
}

__global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const unsigned *__restrict__ kin,
                                                             const unsigned *__restrict__ vin,
                                                             unsigned *__restrict__ kout,
                                                             unsigned *__restrict__ vout, int n, int shift,
                                                             int ntiles, const int *__restrict__ offs,
                                                             const int *n_dev, int *__restrict__ posmap) {
    __shared__ int cnt[RS_WARPS][RS_DIGITS];
    n = dev_count(n, n_dev);
    __shared__ int gbase[RS_DIGITS];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < RS_WARPS * RS_DIGITS; i += RS_THREADS) (&cnt[0][0])[i] = 0;
    for (int d = threadIdx.x; d < RS_DIGITS; d += RS_THREADS) gbase[d] = offs[(long long)d * ntiles + blockIdx.x];
    __syncthreads();
    long long wbase = (long long)blockIdx.x * RS_TILE + (long long)wid * RS_WARP_TILE;
    unsigned key[RS_ITEMS], val[RS_ITEMS];
    int rank[RS_ITEMS];
    unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        long long i = wbase + r * 32 + lane;
        bool ok = i < n;
        key[r] = ok ? kin[i] : 0xffffffffu;
        val[r] = ok ? vin[i] : 0u;
        int d = ok ? (int)((key[r] >> shift) & (RS_DIGITS - 1)) : -1;
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int before = d >= 0 ? cnt[wid][d] : 0;
        rank[r] = before + __popc(peers & lt);
        __syncwarp();
        if (d >= 0 && (peers & lt) == 0) cnt[wid][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps for each digit (warp order == tile order)
    for (int d = threadIdx.x; d < RS_DIGITS; d += RS_THREADS) {
        int s = 0;
        for (int w = 0; w < RS_WARPS; w++) {
            int c = cnt[w][d];
            cnt[w][d] = s;
            s += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; r++) {
        long long i = wbase + r * 32 + lane;
        if (i < n) {
            int d = (int)((key[r] >> shift) & (RS_DIGITS - 1));
            int pos = gbase[d] + cnt[wid][d] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
            if (posmap) posmap[val[r]] = pos;
        }
    }
}

size_t radix_temp_ints(long long n) {
    long long nt = (n + RS_TILE - 1) / RS_TILE;
    long long h = nt * RS_DIGITS;
    return (size_t)(2 * h + scan_temp_ints(h) + 4);
}

__global__ void k_copy_pairs(const unsigned *__restrict__ ka, const unsigned *__restrict__ va,
                             unsigned *__restrict__ kb, unsigned *__restrict__ vb, int n, const int *n_dev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < dev_count(n, n_dev)) {
        kb[i] = ka[i];
        if (va) vb[i] = va[i];
    }
}

// a one-element sort with a final value array: the value and its position
__global__ void k_copy_one(const unsigned *__restrict__ vals, unsigned *__restrict__ vfinal, int *__restrict__ posmap,
                           const int *n_dev) {
    if (dev_count(1, n_dev) < 1) return;
    vfinal[0] = vals[0];
    if (posmap) posmap[vals[0]] = 0;
}

// Stable sort by the low keybits bits of keys.  Result ends in (keys, vals);
// (kalt, valt) are scratch of n elements each.  n_dev (device, may be NULL):
// the count, at most n, when only the device knows it (elements beyond it
// are left as they are).  With vfinal (n elements), the last pass writes the
// sorted values there instead, and with posmap also posmap[value] = its
// sorted position (the values then index posmap); vals is left as scratch.
void radix_sort_pairs(unsigned *keys, unsigned *vals, unsigned *kalt, unsigned *valt, long long n,
                      int keybits, int *tmp, cudaStream_t st, const int *n_dev, unsigned *vfinal, int *posmap) {
    if (n <= 1) {
        // nothing to sort: the one value (if any) and its position
        if (vfinal && n == 1)
            k_copy_one<<<1, 1, 0, st>>>(vals, vfinal, posmap, n_dev);
        return;
    }
    int nt = (int)((n + RS_TILE - 1) / RS_TILE);
    long long h = (long long)nt * RS_DIGITS;
    int *hist = tmp, *offs = tmp + h, *stmp = tmp + 2 * h;
    unsigned *ka = keys, *va = vals, *kb = kalt, *vb = valt;
    int passes = (keybits + RS_BITS - 1) / RS_BITS;
    for (int p = 0; p < passes; p++) {
        int shift = p * RS_BITS;
        const bool last = p == passes - 1;
        unsigned *vo = last && vfinal ? vfinal : vb;
        k_rs_hist<<<nt, RS_THREADS, 0, st>>>(ka, (int)n, shift, nt, hist, n_dev);
        exclusive_scan(hist, offs, h, nullptr, stmp, st, nullptr);
        k_rs_scatter<<<nt, RS_THREADS, 0, st>>>(ka, va, kb, vo, (int)n, shift, nt, offs, n_dev,
                                                last ? posmap : nullptr);
        unsigned *t = ka; ka = kb; kb = t;
        t = va; va = vb; vb = t;
    }
    if (vfinal) {
        // the values are in vfinal; the keys go back if they ended in kalt
        if (ka != keys) {
            if (n_dev)
                k_copy_pairs<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ka, nullptr, keys, nullptr, (int)n, n_dev);
            else
                cudaMemcpyAsync(keys, ka, n * sizeof(unsigned), cudaMemcpyDeviceToDevice, st);
        }
        return;
    }
    if (ka != keys) {
        if (n_dev) {
            // only the sorted elements: those beyond the count stay as they are
            k_copy_pairs<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(ka, va, keys, vals, (int)n, n_dev);
        } else {
            cudaMemcpyAsync(keys, ka, n * sizeof(unsigned), cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(vals, va, n * sizeof(unsigned), cudaMemcpyDeviceToDevice, st);
        }
    }
}

int radix_launches(int keybits, long long n) {
    if (n <= 1) return 0;
    int passes = (keybits + RS_BITS - 1) / RS_BITS;
    long long nt = (n + RS_TILE - 1) / RS_TILE;
    return passes * (2 + scan_launches(nt * RS_DIGITS));
}

int scan_launches(long long n) {
    if (n <= 0) return 0;
    long long nt = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nt == 1) return 1;
    return 2 + scan_launches(nt);
}

}  // namespace sx
