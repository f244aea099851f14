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

// lanes of a warp holding the same label add once (neighbouring pixels
// mostly share a component, so this removes most of the atomic traffic)
__global__ void k_count_labels(const int *__restrict__ lab, int *__restrict__ cnt, long long n) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int l = p < n ? lab[p] : -1;
    const unsigned same = __match_any_sync(0xffffffffu, l);
    if (l >= 0 && (threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(&cnt[l], __popc(same));
}

// flag[p] = 1 if p is the root (smallest pixel) of a component >= minarea
__global__ void k_root_flags(const int *__restrict__ lab, const int *__restrict__ cnt, int *__restrict__ flag,
                             long long n, int minarea) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    flag[p] = (lab[p] == (int)p && cnt[p] >= minarea) ? 1 : 0;
}

// flag2[p] = 1 if p belongs to a kept component (cnt at its root >= minarea)
__global__ void k_pix_flags(const int *__restrict__ lab, const int *__restrict__ cnt, int *__restrict__ flag,
                            long long n, int minarea) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int l = lab[p];
    flag[p] = (l >= 0 && cnt[l] >= minarea) ? 1 : 0;
}

// per root: size, first pixel; scanned root flags give the root id
__global__ void k_root_setup(const int *__restrict__ lab, const int *__restrict__ cnt, const int *__restrict__ rid,
                             int *__restrict__ rsize, int *__restrict__ rfirst, long long n, int minarea) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    if (lab[p] == (int)p && cnt[p] >= minarea) {
        int r = rid[p];
        rsize[r] = cnt[p];
        rfirst[r] = (int)p;
    }
}

// compaction of kept pixels in raster order with their root id as sort key
__global__ void k_pix_compact(const int *__restrict__ lab, const int *__restrict__ cnt, const int *__restrict__ rid,
                              const int *__restrict__ pos, unsigned *__restrict__ keys, unsigned *__restrict__ vals,
                              long long n, int minarea) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    int l = lab[p];
    if (l >= 0 && cnt[l] >= minarea) {
        int j = pos[p];
        keys[j] = (unsigned)rid[l];
        vals[j] = (unsigned)p;
    }
}

__global__ void k_pos2idx(const unsigned *__restrict__ vals, int *__restrict__ pos2idx, int m) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < m) pos2idx[vals[j]] = j;
}

// Each raw object's thresholds: the smallest detection and analysis threshold
// of its pixels (the global ones without a weight map); rdthr/rathr start at a
// large positive float and are lowered through their bit patterns (positive
// floats order like their bits).  The fixed-point scale of the exact branch
// sums, sc->e0cd, becomes the exponent of the smallest of them.
__global__ void k_root_thresholds(const int *__restrict__ lab, const int *__restrict__ cnt,
                                  const int *__restrict__ rid, long long n, int minarea, const float *__restrict__ wvar,
                                  int wthr, double dfac, double afac, FrameScalars *sc, int *rdthr, int *rathr) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int l = lab[p];
    if (l < 0 || cnt[l] < minarea) return;
    const int r = rid[l];
    const float v = wvar ? __ldg(wvar + p) : 0.0f;
    const float dt = sx_pix_thr(wthr, dfac, v, sc->dthresh), at = sx_pix_thr(wthr, afac, v, sc->thresh);
    atomicMin(rdthr + r, __float_as_int(dt));
    atomicMin(rathr + r, __float_as_int(at));
    atomicMin(&sc->e0cd, fexpo(dt));
}

// without a weight map every raw object has the global thresholds
__global__ void k_root_thresholds_global(int nroots, const FrameScalars *sc, float *rdthr, float *rathr) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nroots) {
        rdthr[r] = sc->dthresh;
        rathr[r] = sc->thresh;
    }
}

int bits_for(long long v) {
    int b = 1;
    while ((1ll << b) <= v) b++;
    return b;
}

}  // namespace sx
