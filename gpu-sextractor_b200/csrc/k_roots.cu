// k_roots.cu -- raw objects ("roots"): connected components of at least
// DETECT_MINAREA pixels, numbered in order of their first pixel, with their
// pixel lists contiguous and in raster order.
//
// Reference: src/cuda/cudadetection.cu:677-897 (compact_and_sort: sort by
// label, segment counts, minarea prune, consecutive relabel) and :899-1105
// (pre_analyse: fdpeak / fdflux per raw object).
#include "common.cuh"
#include "kernels.cuh"
#include "prim.cuh"

namespace sx {

// Each raw object's thresholds: the smallest detection and analysis threshold
// of its pixels (the global ones without a weight map); rdthr/rathr start at a
// large positive float and are lowered through their bit patterns (positive
// floats order like their bits).  The fixed-point scale of the exact branch
// sums, sc->e0cd, becomes the exponent of the smallest of them.
__global__ void k_root_thresholds(const int *__restrict__ lab, const int *__restrict__ cnt,
                                  const int *__restrict__ rid, long long n, int minarea, const float *__restrict__ wvar,
                                  int wthr, double dfac, double afac, FrameScalars *sc, int *rdthr, int *rathr) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int r = -1, idt = 0x7fffffff, iat = 0x7fffffff, e = 0x7fffffff;
    if (p < n) {
        const int l = lab[p];
        if (l >= 0 && cnt[l] >= minarea) {
            r = rid[l];
            const float v = wvar ? __ldg(wvar + p) : 0.0f;
            const float dt = sx_pix_thr(wthr, dfac, v, sc->dthresh), at = sx_pix_thr(wthr, afac, v, sc->thresh);
            idt = __float_as_int(dt);
            iat = __float_as_int(at);
            e = fexpo(dt);
        }
    }
    // the minima are taken in the warp first (neighbouring pixels mostly
    // share their raw object), then one atomic per raw object and warp
    e = __reduce_min_sync(0xffffffffu, e);
    if ((threadIdx.x & 31) == 0 && e != 0x7fffffff) atomicMin(&sc->e0cd, e);
    const unsigned grp = __match_any_sync(0xffffffffu, r);
    if (r >= 0) {
        idt = __reduce_min_sync(grp, idt);
        iat = __reduce_min_sync(grp, iat);
        if ((int)(threadIdx.x & 31) == __ffs(grp) - 1) {
            atomicMin(rdthr + r, idt);
            atomicMin(rathr + r, iat);
        }
    }
}

// without a weight map every raw object has the global thresholds
__global__ void k_root_thresholds_global(int nroots, const int *nroots_dev, const FrameScalars *sc, float *rdthr,
                                         float *rathr) {
    nroots = sx_count(nroots, nroots_dev);
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nroots) {
        rdthr[r] = sc->dthresh;
        rathr[r] = sc->thresh;
    }
}

// ---- the raw-object numbering and the kept-pixel compaction as two scans
// whose inputs are computed on the fly (a root: lab[p] == p with at least
// minarea pixels; a kept pixel: its root has at least minarea pixels).  The
// tiles of SCAN_TILE pixels are those of the scan primitive (1024 threads, 4
// consecutive pixels each), so the per-tile counts of k_root_tile_counts and
// the in-tile prefixes of k_root_number / k_root_compact line up.
// The flags of a thread's SCAN_ITEMS (= 4) consecutive pixels from base (a
// multiple of 4), with one 16-byte load of their labels where all four are
// in the frame and the label array is 16-byte aligned.
__device__ __forceinline__ void root_kept_flags4(const int *__restrict__ lab, const int *__restrict__ cnt,
                                                 long long base, long long n, int minarea, int *isroot, int *kept,
                                                 int *l) {
    static_assert(SCAN_ITEMS == 4, "four pixels per thread");
    if (base + 3 < n && ((reinterpret_cast<uintptr_t>(lab) & 15) == 0)) {
        const int4 v = *reinterpret_cast<const int4 *>(lab + base);
        l[0] = v.x;
        l[1] = v.y;
        l[2] = v.z;
        l[3] = v.w;
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) l[k] = base + k < n ? lab[base + k] : -1;
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        kept[k] = l[k] >= 0 && cnt[l[k]] >= minarea;
        isroot[k] = kept[k] && l[k] == (int)(base + k);
    }
}

// per tile: number of roots and of kept pixels
__global__ void __launch_bounds__(SCAN_THREADS) k_root_tile_counts(const int *__restrict__ lab,
                                                                  const int *__restrict__ cnt, long long n,
                                                                  int minarea, int *__restrict__ troots,
                                                                  int *__restrict__ tkept) {
    __shared__ int sh[32];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int cr = 0, ck = 0, r[SCAN_ITEMS], kp[SCAN_ITEMS], l[SCAN_ITEMS];
    root_kept_flags4(lab, cnt, base, n, minarea, r, kp, l);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        cr += r[k];
        ck += kp[k];
    }
    int tot;
    block_exclusive_scan(cr, sh, tot);
    if (threadIdx.x == 0) troots[blockIdx.x] = tot;
    block_exclusive_scan(ck, sh, tot);
    if (threadIdx.x == 0) tkept[blockIdx.x] = tot;
}

// roots numbered in raster order: rid at the root pixel, size and first pixel
__global__ void __launch_bounds__(SCAN_THREADS) k_root_number(const int *__restrict__ lab, const int *__restrict__ cnt,
                                                             long long n, int minarea, const int *__restrict__ toff,
                                                             int *__restrict__ rid, int *__restrict__ rsize,
                                                             int *__restrict__ rfirst) {
    __shared__ int sh[32];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int fr[SCAN_ITEMS], kp[SCAN_ITEMS], l[SCAN_ITEMS], c = 0;
    root_kept_flags4(lab, cnt, base, n, minarea, fr, kp, l);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) c += fr[k];
    int tot;
    int id = block_exclusive_scan(c, sh, tot) + toff[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
        if (fr[k]) {
            const long long p = base + k;
            rid[p] = id;
            rsize[id] = cnt[p];
            rfirst[id] = (int)p;
            id++;
        }
}

// kept pixels compacted in raster order with their root id as sort key; the
// allocation map starts as "unassigned object pixel" / background and the
// pixel -> list index map as -1
__global__ void __launch_bounds__(SCAN_THREADS) k_root_compact(const int *__restrict__ lab, const int *__restrict__ cnt,
                                                              long long n, int minarea, const int *__restrict__ toff,
                                                              const int *__restrict__ rid, unsigned *__restrict__ keys,
                                                              unsigned *__restrict__ vals, int *__restrict__ alloc,
                                                              int *__restrict__ pos2idx) {
    __shared__ int sh[32];
    const long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    int fk[SCAN_ITEMS], lb[SCAN_ITEMS], fr[SCAN_ITEMS], c = 0;
    root_kept_flags4(lab, cnt, base, n, minarea, fr, fk, lb);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) c += fk[k];
    int tot;
    int j = block_exclusive_scan(c, sh, tot) + toff[blockIdx.x];
    const bool vec = base + 3 < n && ((reinterpret_cast<uintptr_t>(alloc) | reinterpret_cast<uintptr_t>(pos2idx)) & 15) == 0;
    if (vec) {
        *reinterpret_cast<int4 *>(alloc + base) =
            make_int4(lb[0] >= 0 ? SX_ALLOC_OTHER : -1, lb[1] >= 0 ? SX_ALLOC_OTHER : -1,
                      lb[2] >= 0 ? SX_ALLOC_OTHER : -1, lb[3] >= 0 ? SX_ALLOC_OTHER : -1);
        *reinterpret_cast<int4 *>(pos2idx + base) = make_int4(-1, -1, -1, -1);
    }
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        const long long p = base + k;
        if (p >= n) break;
        if (!vec) {
            alloc[p] = lb[k] >= 0 ? SX_ALLOC_OTHER : -1;
            pos2idx[p] = -1;
        }
        if (fk[k]) {
            keys[j] = (unsigned)rid[lb[k]];
            vals[j] = (unsigned)p;
            j++;
        }
    }
}

int bits_for(long long v) {
    int b = 1;
    while ((1ll << b) <= v) b++;
    return b;
}

}  // namespace sx
