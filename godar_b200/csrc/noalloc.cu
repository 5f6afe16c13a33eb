// Candidate-pair search that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host program whose own memory
// manager has already reserved the GPU's memory, or a time-critical loop that
// must not pay cudaMalloc's implicit device synchronisation.  This entry point
// runs the same neighbour search as the step (cell keys, radix sort, cell
// ranges, exact radius predicate) but keeps all of its scratch in one
// file-scope device array of fixed size.  Every GPU that loads the library
// holds that array (about 2.4 MB) until the process exits.
//
// Limits: at most GODAR_NOALLOC_MAX_FLOES floes, at most 256 x 256 cells.
// The scratch array is shared by every call on a device and keeps the last
// call's contents, so calls that overlap on the GPU (from several host
// threads, each on its own per-thread stream) race on it; callers must
// serialise them.  The first call on each device looks up the array's device
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
        const double R = sm[0] + rtree;
        int ncx = (int)floor(nx / (R > 0.0 ? R : 1.0)), ncy = (int)floor(ny / (R > 0.0 ? R : 1.0));
        ncx = ncx < 1 ? 1 : (ncx > 256 ? 256 : ncx);
        ncy = ncy < 1 ? 1 : (ncy > 256 ? 256 : ncy);
        S->grid.ncx = ncx;
        S->grid.ncy = ncy;
        S->grid.cw = nx / ncx;
        S->grid.ch = ny / ncy;
        S->grid.total = 0;
    }
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

__global__ void k_na_keys(const double *x, const double *y, int n, NaScratch *S)
{
    const NaGrid G = S->grid;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int cx, cy;
        na_cell(G, x[i], y[i], cx, cy);
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
// (this file is compiled with --fmad=false).
template <bool FILL>
__global__ void k_na_pairs(const double *x, const double *y, const double *r, int n, double nx, double ny,
                           double rtree, int boundary, NaScratch *S, int32_t *pi, int32_t *pj, int cap)
{
    const NaGrid G = S->grid;
    const bool px = boundary & GODAR_BC_PERIODIC_X, py = boundary & GODAR_BC_PERIODIC_Y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = S->vals[k];
        const double xi = x[i], yi = y[i], R = r[i] + rtree;
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
                    const double dx = wrap_d(xi - x[j], nx, px), dy = wrap_d(yi - y[j], ny, py);
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

std::mutex g_na_mutex;
void *g_na_ptr[64] = {nullptr};

}  // namespace
}  // namespace godar

using namespace godar;

extern "C" int godar_gpu_candidates_noalloc(const double *x, const double *y, const double *r, int n, double nx,
                                            double ny, double rtree, int boundary, int32_t *pair_i,
                                            int32_t *pair_j, int cap, int *count)
{
    if (count) *count = 0;
    if (!x || !y || !r || !count || (cap > 0 && (!pair_i || !pair_j)) || n < 0 || cap < 0) return GODAR_ERR_BAD_INPUT;
    if (!(nx > 0.0) || !(ny > 0.0) || !(rtree >= 0.0)) return GODAR_ERR_BAD_INPUT;
    if (n > NA_MAXN) return GODAR_ERR_CAPACITY;   // beyond the fixed scratch array
    if (n == 0) return GODAR_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return GODAR_ERR_NO_DEVICE;
    }
    NaScratch *S = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_na_mutex);
        if (!g_na_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();
                return GODAR_ERR_CUDA;
            }
            g_na_ptr[dev] = p;
        }
        S = (NaScratch *)g_na_ptr[dev];
    }
    cudaStream_t st = cudaStreamPerThread;
    const int grid = std::min((n + 255) / 256, 148 * 8);
    k_na_grid<<<1, 256, 0, st>>>(r, n, nx, ny, rtree, S);
    k_na_keys<<<grid, 256, 0, st>>>(x, y, n, S);
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
    int total = 0;
    if (cudaMemcpyAsync(&total, &S->off[n], sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return GODAR_ERR_CUDA;
    }
    *count = total;
    return total > cap ? GODAR_ERR_CAPACITY : GODAR_OK;
}
