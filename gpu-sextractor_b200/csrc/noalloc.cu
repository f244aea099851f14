// noalloc.cu -- background estimation and subtraction without any device
// allocation: sexgpu_background_noalloc().
//
// Who this is for: code that must not call cudaMalloc/cudaFree at all, for
// example a pipeline that runs inside a memory pool owned by another
// framework, a process with a hard device-memory budget fixed at start-up,
// or a real-time loop where an allocation (and the implicit device
// synchronisation it can cause) is not allowed.  Such a caller owns every
// buffer it passes (the frame, the subtracted frame, the two mesh maps); the
// library only needs working memory of bounded size, which lives in the
// fixed device array below instead of being allocated per call.
//
// The array is a file-scope static __device__ object, so every GPU that
// loads this library holds it (about 13.2 MB) for the life of the process.
// In host code its name is only a host-side stand-in, so its device address
// is looked up once per device with cudaGetSymbolAddress (with that device
// current) and passed to the kernels.  All calls share the array and it
// keeps the last call's contents; everything that must start at zero is
// cleared by each call.  Calls that overlap on the GPU (different streams or
// host threads at the same time) race on it and must be serialised by the
// caller.
#include <atomic>
#include <mutex>

namespace sx_noalloc {

// limits of one call (also in include/sexgpu.h)
constexpr int MAX_W = 16384;                 // frame width
constexpr int MAX_H = 16384;                 // frame height
constexpr int MAX_MESH = 16384;              // nbackx * nbacky
constexpr long long MAX_ROWNODES = 1 << 20;  // height * nbackx

constexpr size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

constexpr size_t OFF_SC = 0;
constexpr size_t OFF_MS = al256(OFF_SC + sizeof(FrameScalars));
constexpr size_t OFF_BACK = al256(OFF_MS + sizeof(sx::MeshStat) * MAX_MESH);
constexpr size_t OFF_SIGMA = al256(OFF_BACK + 4 * (size_t)MAX_MESH);
constexpr size_t OFF_BACK2 = al256(OFF_SIGMA + 4 * (size_t)MAX_MESH);
constexpr size_t OFF_DBACK = al256(OFF_BACK2 + 4 * (size_t)MAX_MESH);
constexpr size_t OFF_U = al256(OFF_DBACK + 4 * (size_t)MAX_MESH);
constexpr size_t OFF_ROWNODE = al256(OFF_U + 4 * (size_t)MAX_MESH);
constexpr size_t OFF_ROWDNODE = al256(OFF_ROWNODE + 4 * (size_t)MAX_ROWNODES);
constexpr size_t OFF_ROWU = al256(OFF_ROWDNODE + 4 * (size_t)MAX_ROWNODES);
constexpr size_t OFF_COLK = al256(OFF_ROWU + 4 * (size_t)MAX_ROWNODES);
constexpr size_t OFF_COLDX = al256(OFF_COLK + 4 * (size_t)MAX_W);
constexpr size_t SCRATCH_BYTES = al256(OFF_COLDX + 4 * (size_t)MAX_W);

}  // namespace sx_noalloc

static __device__ __align__(256) unsigned char sx_noalloc_scratch[sx_noalloc::SCRATCH_BYTES];

namespace sx_noalloc {

constexpr int MAX_DEVICES = 64;
static unsigned char *g_scratch[MAX_DEVICES];
static std::once_flag g_once[MAX_DEVICES];
static cudaError_t g_setup_err[MAX_DEVICES];

// device address of the scratch array on the current device (looked up once)
static cudaError_t scratch_on_current_device(unsigned char **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::call_once(g_once[dev], [dev]() {
        void *p = nullptr;
        g_setup_err[dev] = cudaGetSymbolAddress(&p, sx_noalloc_scratch);
        g_scratch[dev] = (unsigned char *)p;
    });
    if (g_setup_err[dev] != cudaSuccess) return g_setup_err[dev];
    *out = g_scratch[dev];
    return cudaSuccess;
}

// Column table of src/back.c:863-899 computed on the device: for column j the
// segment index k and the interpolation offset dx.  dx is replayed with the
// reference's float additions from the last restart of the sequence, so it
// equals the value of the sequential loop.
__global__ void k_col_table(int width, int nbx, int backw, int *colk, float *coldx) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= width) return;
    if (nbx <= 1) {
        colk[j] = 0;
        coldx[j] = 0.f;
        return;
    }
    const int nx = backw, changepoint = nx / 2;
    const float xstep = 1.0 / nx;
    // In the reference loop the in-mesh counter i equals the column up to nx,
    // then restarts at 1 after every nx columns, and the mesh counter x is
    // (column-1)/nx.  The node pointers advance where i == nx/2 and
    // 0 < x < nbx-1, i.e. at columns nx*x + nx/2 for x = 1 .. nbx-2 (never
    // when nx/2 == 0).
    int k = 0, last = -1;
    if (changepoint > 0 && j >= nx + changepoint) {
        k = (j - changepoint) / nx;
        if (k > nbx - 2) k = nbx - 2;
        if (k > 0) last = nx * k + changepoint;
    }
    float dx;
    int from;
    if (last >= 0) {
        dx = ((nx + 1) % 2) * xstep / 2;
        from = last;
    } else {
        dx = (xstep - 1) / 2;
        from = 0;
    }
    for (int c = from; c < j; c++) dx += xstep;
    colk[j] = k;
    coldx[j] = dx;
}

// background subtraction only (the subtraction half of k_sub_filter)
__global__ void k_sub_only(const float *__restrict__ img, float *__restrict__ sub, sx::BackBufs B, int w, int h,
                           int nbx, int back_type, const FrameScalars *sc) {
    long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= (long long)w * h) return;
    int x = (int)(p % w), y = (int)(p / w);
    sub[p] = sx_unblank(img[p]) - sx::bkg_at(x, y, B, nbx, back_type, sc->backmean);
}

}  // namespace sx_noalloc

extern "C" int sexgpu_background_meshes(int w, int h, int back_size, int *nbackx, int *nbacky) {
    if (w <= 0 || h <= 0 || back_size < 1 || !nbackx || !nbacky) return SEXGPU_ERR_ARG;
    const int bw = back_size < w ? back_size : w, bh = back_size < h ? back_size : h;  // src/field.c:124-127
    *nbackx = (w - 1) / bw + 1;
    *nbacky = (h - 1) / bh + 1;
    return SEXGPU_OK;
}

extern "C" int sexgpu_background_noalloc(const float *d_img, float *d_sub, int w, int h, const sexgpu_config *cfg,
                                         float *d_back, float *d_sigma, int mesh_capacity, sexgpu_summary *sum,
                                         void *stream) {
    using namespace sx_noalloc;
    if (!d_img || !d_sub || !d_back || !d_sigma || !cfg || w <= 0 || h <= 0) return SEXGPU_ERR_ARG;
    if (cfg->back_size < 1 || cfg->back_filtersize < 1 || cfg->back_filtersize > 11) return SEXGPU_ERR_ARG;
    FrameParams Pm;
    make_params(cfg, w, h, Pm);
    if (w > MAX_W || h > MAX_H || (long long)Pm.nbx * Pm.nby > MAX_MESH ||
        (long long)h * Pm.nbx > MAX_ROWNODES)
        return SEXGPU_ERR_NOALLOC_LIMIT;
    // the caller's mesh maps must hold nbackx * nbacky floats each
    if ((long long)mesh_capacity < (long long)Pm.nbx * Pm.nby) return SEXGPU_ERR_ARG;
    unsigned char *base = nullptr;
    cudaError_t e = scratch_on_current_device(&base);
    if (e != cudaSuccess) return SEXGPU_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    FrameScalars *d_sc = (FrameScalars *)(base + OFF_SC);
    sx::BackBufs B;
    B.ms = (sx::MeshStat *)(base + OFF_MS);
    B.back = (float *)(base + OFF_BACK);
    B.sigma = (float *)(base + OFF_SIGMA);
    B.back2 = (float *)(base + OFF_BACK2);
    B.back3 = d_back;    // caller's outputs receive the filtered maps
    B.sigma3 = d_sigma;
    B.dback = (float *)(base + OFF_DBACK);
    B.u = (float *)(base + OFF_U);
    B.rownode = (float *)(base + OFF_ROWNODE);
    B.rowdnode = (float *)(base + OFF_ROWDNODE);
    B.rowu = (float *)(base + OFF_ROWU);
    B.colk = (int *)(base + OFF_COLK);
    B.coldx = (float *)(base + OFF_COLDX);
    int nl = 0;
    k_init_scalars<<<1, 1, 0, st>>>(d_sc);  // the pipeline's initial scalars (sigfac 1)
    k_col_table<<<(w + 255) / 256, 256, 0, st>>>(w, Pm.nbx, Pm.bw, B.colk, B.coldx);
    sx::launch_background(B, d_img, Pm, d_sc, st, nl);
    long long n = (long long)w * h;
    k_sub_only<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d_img, d_sub, B, w, h, Pm.nbx, Pm.back_type, d_sc);
    if (cudaGetLastError() != cudaSuccess) return SEXGPU_ERR_CUDA;
    if (sum) {
        FrameScalars hs;
        if (cudaMemcpyAsync(&hs, d_sc, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess) return SEXGPU_ERR_CUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return SEXGPU_ERR_CUDA;
        memset(sum, 0, sizeof(*sum));
        sum->nbackx = Pm.nbx;
        sum->nbacky = Pm.nby;
        sum->backmean = hs.backmean;
        sum->backsig = hs.backsig;
        sum->dthresh = hs.dthresh;
        sum->thresh = hs.thresh;
    }
    return SEXGPU_OK;
}
