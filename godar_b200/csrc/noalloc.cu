// Candidate-pair search that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host program whose own memory
// manager has already reserved the GPU's memory, or a time-critical loop that
// must not pay cudaMalloc's implicit device synchronisation.  This entry point
// runs the same neighbour search as the step (cell keys, radix sort, cell
// ranges, exact radius predicate) but keeps all of its scratch in one
// file-scope device array of fixed size (about 2.4 MB).
//
// When the array exists on a device: CUDA loads a library's device code
// lazily by default, so the array (with the module's code) is allocated on a
// device by the CUDA driver when this file's module is first used there -
// the first call on that device, or the set-up call (n = 0) - and it stays
// until the process exits.  A caller whose own allocator is about to reserve
// the device's memory should therefore make the set-up call first.
//
// Limits: at most GODAR_NOALLOC_MAX_FLOES floes, at most 256 x 256 cells.
// The scratch array is shared by every call on a device and keeps the last
// call's contents, so calls that overlap on the GPU (from several host
// threads, each on its own per-thread stream) race on it; callers must
// serialise them.  The call that sets a device up looks up the array's device
// address (cudaGetSymbolAddress) and should therefore come before any stream
// capture on that device.
#include <cmath>
#include <mutex>

#include "../../include/godar_gpu.h"
#include "common.cuh"
#include "kernels.h"

namespace godar {
namespace {

constexpr int NA_MAXN = GODAR_NOALLOC_MAX_FLOES;
constexpr int NA_MAXC = 256 * 256;
constexpr int NA_TILES = (NA_MAXN + 2047) / 2048;

struct NaGrid {
    double cw, ch;
    int ncx, ncy;
    int total;        // candidate pairs found
    int pad;
};

struct NaScratch {
    uint32_t keys[NA_MAXN], keys_alt[NA_MAXN];
    int vals[NA_MAXN], vals_alt[NA_MAXN];
    int counts[256 * NA_TILES + 1];
    int scan[4096];
    int cstart[NA_MAXC], cend[NA_MAXC];
    int cnt[NA_MAXN + 1], off[NA_MAXN + 1];
    NaGrid grid;
};

}  // namespace

static __device__ __align__(256) NaScratch g_noalloc_scratch;

namespace {

__global__ void k_na_grid(const double *r, int n, double nx, double ny, double rtree, NaScratch *S)
{
    __shared__ double sm[256];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = r[i] > m ? r[i] : m;
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o && sm[threadIdx.x + o] > sm[threadIdx.x]) sm[threadIdx.x] = sm[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // cells at least as wide as the largest search radius, at most 256
        // per axis, tiling the domain exactly
        // (clamped in double before the integer conversion: nx / R can be
        // far beyond the int range when R is tiny)
        const double R = sm[0] + rtree;
        const double Rs = R > 0.0 ? R : 1.0;
        const double fx = fmin(fmax(floor(nx / Rs), 1.0), 256.0), fy = fmin(fmax(floor(ny / Rs), 1.0), 256.0);
        const int ncx = (int)fx, ncy = (int)fy;
        S->grid.ncx = ncx;
        S->grid.ncy = ncy;
        S->grid.cw = nx / ncx;
        S->grid.ch = ny / ncy;
        S->grid.total = 0;
    }
}

// A coordinate of a periodic axis brought into [0, L): callers may pass
// positions any number of periods outside the domain.  Exact (the identity)
// for coordinates already in [0, L), so that distances round as in the step.
__device__ __forceinline__ double na_wrap(double x, double L, bool per)
{
    if (!per || (x >= 0.0 && x < L)) return x;
    double w = x - floor(x / L) * L;
    if (w >= L) w = w - L;
    if (!(w >= 0.0)) w = 0.0;
    return w;
}

__device__ __forceinline__ void na_cell(const NaGrid &G, double x, double y, int &cx, int &cy)
{
    double fx = x / G.cw, fy = y / G.ch;
    if (!(fx >= 0.0)) fx = 0.0;
    if (!(fy >= 0.0)) fy = 0.0;
    if (fx > (double)G.ncx) fx = (double)G.ncx;
    if (fy > (double)G.ncy) fy = (double)G.ncy;
    cx = (int)floor(fx);
    cy = (int)floor(fy);
    cx = cx >= G.ncx ? G.ncx - 1 : cx;
    cy = cy >= G.ncy ? G.ncy - 1 : cy;
}

__global__ void k_na_keys(const double *x, const double *y, int n, double nx, double ny, int boundary, NaScratch *S)
{
    const NaGrid G = S->grid;
    const bool px = boundary & GODAR_BC_PERIODIC_X, py = boundary & GODAR_BC_PERIODIC_Y;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int cx, cy;
        na_cell(G, na_wrap(x[i], nx, px), na_wrap(y[i], ny, py), cx, cy);
        S->keys[i] = (uint32_t)(cy * G.ncx + cx);
        S->vals[i] = i;
    }
}

__global__ void k_na_ranges(int n, NaScratch *S)
{
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t c = S->keys[k];
        if (k == 0 || S->keys[k - 1] != c) S->cstart[c] = k;
        if (k == n - 1 || S->keys[k + 1] != c) S->cend[c] = k + 1;
    }
}

// FILL = false: count the candidates j > i of floe i = vals[k]; true: write
// them.  Predicate as in the step: sqrt(dx^2 + dy^2) <= r_i + rtree in FP64
// (this file is compiled with --fmad=false), on coordinates wrapped into the
// domain along periodic axes.
template <bool FILL>
__global__ void k_na_pairs(const double *x, const double *y, const double *r, int n, double nx, double ny,
                           double rtree, int boundary, NaScratch *S, int32_t *pi, int32_t *pj, int cap)
{
    const NaGrid G = S->grid;
    const bool px = boundary & GODAR_BC_PERIODIC_X, py = boundary & GODAR_BC_PERIODIC_Y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = S->vals[k];
        const double xi = na_wrap(x[i], nx, px), yi = na_wrap(y[i], ny, py), R = r[i] + rtree;
        int cx, cy;
        na_cell(G, xi, yi, cx, cy);
        int xs[3], ys[3], nxs = 0, nys = 0;
        for (int d = -1; d <= 1; d++) {
            int c = cx + d;
            if (px) c = ((c % G.ncx) + G.ncx) % G.ncx;
            else if (c < 0 || c >= G.ncx) continue;
            bool dup = false;
            for (int q = 0; q < nxs; q++) dup |= xs[q] == c;
            if (!dup) xs[nxs++] = c;
        }
        for (int d = -1; d <= 1; d++) {
            int c = cy + d;
            if (py) c = ((c % G.ncy) + G.ncy) % G.ncy;
            else if (c < 0 || c >= G.ncy) continue;
            bool dup = false;
            for (int q = 0; q < nys; q++) dup |= ys[q] == c;
            if (!dup) ys[nys++] = c;
        }
        int m = 0;
        const int base = FILL ? S->off[k] : 0;
        for (int a = 0; a < nys; a++)
            for (int b = 0; b < nxs; b++) {
                const int c = ys[a] * G.ncx + xs[b];
                for (int t = S->cstart[c]; t < S->cend[c]; t++) {
                    const int j = S->vals[t];
                    if (j <= i) continue;
                    const double dx = wrap_d(xi - na_wrap(x[j], nx, px), nx, px);
                    const double dy = wrap_d(yi - na_wrap(y[j], ny, py), ny, py);
                    if (sqrt(dx * dx + dy * dy) <= R) {
                        if (FILL && base + m < cap) {
                            pi[base + m] = i;
                            pj[base + m] = j;
                        }
                        m++;
                    }
                }
            }
        if (!FILL) S->cnt[k] = m;
    }
}

// The array's device address per device, valid for the context it was
// looked up in: after a context is destroyed and re-created (cudaDeviceReset)
// the module, and with it the array, may load at another address.
typedef int (*CtxGetCurrentFn)(void **);
std::mutex g_na_mutex;
void *g_na_ptr[64] = {nullptr};
void *g_na_ctx[64] = {nullptr};
CtxGetCurrentFn g_ctx_get = nullptr;
bool g_ctx_get_tried = false;

// The calling thread's current CUDA context (driver API, fetched through the
// runtime so that no extra link dependency is needed); null if unknown.
void *current_context()
{
    if (!g_ctx_get_tried) {
        g_ctx_get_tried = true;
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get = (CtxGetCurrentFn)fn;
        cudaGetLastError();
    }
    void *ctx = nullptr;
    if (g_ctx_get && g_ctx_get(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// Set-up of the calling thread's device: the array's address, looked up once
// per device and context.  Loads this file's module on the device if it is
// not loaded yet (CUDA's lazy loading), which is when the driver allocates
// the array there.
int na_scratch(NaScratch **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return GODAR_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lk(g_na_mutex);
    void *ctx = current_context();
    if (!g_na_ptr[dev] || !ctx || ctx != g_na_ctx[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            g_na_ptr[dev] = nullptr;
            return GODAR_ERR_CUDA;
        }
        g_na_ptr[dev] = p;
        // the look-up made the device's primary context current if none was
        g_na_ctx[dev] = current_context();
    }
    *out = (NaScratch *)g_na_ptr[dev];
    return GODAR_OK;
}

}  // namespace
}  // namespace godar

using namespace godar;

extern "C" int godar_gpu_candidates_noalloc(const double *x, const double *y, const double *r, int n, double nx,
                                            double ny, double rtree, int boundary, int32_t *pair_i,
                                            int32_t *pair_j, int cap, int *count)
{
    if (count) *count = 0;
    if (n == 0) {
        // the set-up call: no field, only the device's scratch address
        NaScratch *S = nullptr;
        return na_scratch(&S);
    }
    if (!x || !y || !r || !count || (cap > 0 && (!pair_i || !pair_j)) || n < 0 || cap < 0) return GODAR_ERR_BAD_INPUT;
    if (!(nx > 0.0) || !(ny > 0.0) || !(rtree >= 0.0)) return GODAR_ERR_BAD_INPUT;
    if (n > NA_MAXN) return GODAR_ERR_CAPACITY;   // beyond the fixed scratch array
    NaScratch *S = nullptr;
    const int rc = na_scratch(&S);
    if (rc != GODAR_OK) return rc;
    cudaStream_t st = cudaStreamPerThread;
    // an error left over from earlier work of the caller is not this call's
    cudaGetLastError();
    const int grid = std::min((n + 255) / 256, 148 * 8);
    k_na_grid<<<1, 256, 0, st>>>(r, n, nx, ny, rtree, S);
    k_na_keys<<<grid, 256, 0, st>>>(x, y, n, nx, ny, boundary, S);
    radix_sort(S->keys, S->vals, S->keys_alt, S->vals_alt, n, 16, S->counts, S->scan, st);
    if (cudaMemsetAsync(S->cstart, 0, sizeof(S->cstart), st) != cudaSuccess ||
        cudaMemsetAsync(S->cend, 0, sizeof(S->cend), st) != cudaSuccess) {
        cudaGetLastError();
        return GODAR_ERR_CUDA;
    }
    k_na_ranges<<<grid, 256, 0, st>>>(n, S);
    k_na_pairs<false><<<grid, 128, 0, st>>>(x, y, r, n, nx, ny, rtree, boundary, S, nullptr, nullptr, 0);
    scan_excl(S->cnt, S->off, n, S->scan, st);
    k_na_pairs<true><<<grid, 128, 0, st>>>(x, y, r, n, nx, ny, rtree, boundary, S, pair_i, pair_j, cap);
    // a launch that failed (configuration, missing kernel image) is reported
    // here: the synchronisation below would not show it, and the count would
    // be an earlier call's
    if (cudaGetLastError() != cudaSuccess) return GODAR_ERR_CUDA;
    int total = 0;
    if (cudaMemcpyAsync(&total, &S->off[n], sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return GODAR_ERR_CUDA;
    }
    *count = total;
    return total > cap ? GODAR_ERR_CAPACITY : GODAR_OK;
}
