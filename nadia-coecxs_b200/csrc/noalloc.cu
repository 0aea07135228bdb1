// noalloc.cu -- shrinkwrap on caller-owned device buffers, allocating nothing.
//
// Some callers cannot allocate device memory at the moment they want a
// support update: a server stepping many reconstructions on concurrent
// streams, where cudaMalloc/cudaFree would synchronise the whole device and
// stall every other stream, or a process whose device memory is already
// committed to an admission budget or to another allocator.  This entry
// point takes the estimate and the output support as device pointers and
// keeps its only working memory -- one partial maximum per 32x32 tile -- in
// a fixed array compiled into the library (file-scope static __device__),
// which every GPU that loads this part of the library holds until the
// process exits.
//
// The array holds kMaxTiles tiles' partial maxima twice (blurred values and
// thresholded values), 128 KB, so grids are limited to kMaxTiles 32x32
// tiles (4096 x 4096).  Its contents persist from call to call; every entry a
// call reads is written by that call first, so nothing needs clearing.
// Calls whose work overlaps on the GPU (different streams, or different
// devices sharing nothing but this code) race on the array of their device:
// serialise them.
//
// The array's device address is looked up once per device, on the first call
// made with that device current (cudaGetSymbolAddress); make that first call
// before capturing any stream on that device.
#include <mutex>

#include "common.h"

namespace nadia {
namespace noalloc {

constexpr int kTile = 32;
constexpr int kCut = 4; // BaseCDI::apply_shrinkwrap's pixel cut-off (BaseCDI.c++:432-433)
constexpr int kHalo = kTile + 2 * kCut;
constexpr int kMaxTiles = 16384;
constexpr int kMaxDevices = 64;

// [0, kMaxTiles): tile maxima of the blurred magnitude; [kMaxTiles, 2*kMaxTiles):
// tile maxima of the thresholded values; the two reduced maxima follow.
static __device__ __align__(256) float g_scratch[2 * kMaxTiles + 2];

struct Taps {
    float w[kCut + 1];
};

__device__ __forceinline__ float block_max256(float m)
{
    __shared__ float red[256];
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    red[t] = m;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (t < off) red[t] = fmaxf(red[t], red[t + off]);
        __syncthreads();
    }
    return red[0];
}

// |x| blurred by the truncated, unnormalised Gaussian of BaseCDI::convolve
// (BaseCDI.c++:432-474; square window, neighbours outside the grid skipped),
// one 32x32 output tile per block computed from a 40x40 halo tile in shared
// memory: rows first, then columns.  Writes the blurred values to `out` and
// the tile maximum to scratch[tile].
__global__ void k_blur_tiles(const float2 *__restrict__ x, float *out, int nx, int ny, Taps g,
                             float *scratch)
{
    __shared__ float in[kHalo][kHalo + 1];
    __shared__ float rowb[kHalo][kTile + 1];
    const int i0 = blockIdx.y * kTile - kCut, j0 = blockIdx.x * kTile - kCut;
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    for (int e = t; e < kHalo * kHalo; e += blockDim.x * blockDim.y) {
        const int a = e / kHalo, b = e % kHalo;
        const int i = i0 + a, j = j0 + b;
        float v = 0.f;
        if (i >= 0 && i < nx && j >= 0 && j < ny) {
            const float2 c = x[(size_t)i * ny + j];
            v = sqrtf(c.x * c.x + c.y * c.y);
        }
        in[a][b] = v;
    }
    __syncthreads();
    for (int e = t; e < kHalo * kTile; e += blockDim.x * blockDim.y) {
        const int a = e / kTile, b = e % kTile;
        float acc = 0.f;
#pragma unroll
        for (int d = -kCut; d <= kCut; ++d) acc += g.w[d < 0 ? -d : d] * in[a][b + kCut + d];
        rowb[a][b] = acc;
    }
    __syncthreads();
    float m = -INFINITY;
    for (int e = t; e < kTile * kTile; e += blockDim.x * blockDim.y) {
        const int a = e / kTile, b = e % kTile;
        const int i = blockIdx.y * kTile + a, j = blockIdx.x * kTile + b;
        if (i >= nx || j >= ny) continue;
        float acc = 0.f;
#pragma unroll
        for (int d = -kCut; d <= kCut; ++d) acc += g.w[d < 0 ? -d : d] * rowb[a + kCut + d][b];
        out[(size_t)i * ny + j] = acc;
        m = fmaxf(m, acc);
    }
    m = block_max256(m);
    if (t == 0) scratch[blockIdx.y * gridDim.x + blockIdx.x] = m;
}

__global__ void k_reduce_max(const float *part, int count, float *dst)
{
    float m = -INFINITY;
    for (int b = threadIdx.y * blockDim.x + threadIdx.x; b < count; b += blockDim.x * blockDim.y)
        m = fmaxf(m, part[b]);
    m = block_max256(m);
    if (threadIdx.x == 0 && threadIdx.y == 0) *dst = m;
}

// BaseCDI::apply_threshold (BaseCDI.c++:477-492) with its loop bounds
// i < nx, j < nx: element L = i*ny + j is visited once per pair
// (i', j' = L - i'*ny) with 0 <= j' < nx, and reads 0 where j' > ny.  Then
// the tile maximum of the thresholded values goes to part[tile].
__global__ void k_threshold_tiles(float *a, int nx, int ny, double t, const float *dmax,
                                  float *part)
{
    const double lim = t * (double)(*dmax);
    float m = -INFINITY;
    const int tt = threadIdx.y * blockDim.x + threadIdx.x;
    for (int e = tt; e < kTile * kTile; e += blockDim.x * blockDim.y) {
        const int i = blockIdx.y * kTile + e / kTile, j = blockIdx.x * kTile + e % kTile;
        if (i >= nx || j >= ny) continue;
        const long long L = (long long)i * ny + j;
        long long ilo = L - nx + 1 < 0 ? 0 : (L - nx + 1 + ny - 1) / ny;
        long long ihi = L / ny;
        if (ihi > nx - 1) ihi = nx - 1;
        float cur = a[L];
        if (ilo <= ihi) {
            for (long long ii = ilo; ii <= ihi; ++ii) {
                const long long jj = L - ii * ny;
                const float v = (jj > ny) ? 0.f : cur;
                cur = ((double)v < lim) ? 0.f : 1.f;
            }
            a[L] = cur;
        }
        m = fmaxf(m, cur);
    }
    m = block_max256(m);
    if (tt == 0) part[blockIdx.y * gridDim.x + blockIdx.x] = m;
}

// BaseCDI::set_support's division by the maximum (BaseCDI.c++:95-102)
__global__ void k_divide_tiles(float *a, int nx, int ny, const float *dmax)
{
    const float m = *dmax;
    const int i = blockIdx.y * kTile + threadIdx.y * 4, j = blockIdx.x * kTile + threadIdx.x;
    for (int r = 0; r < 4; ++r)
        if (i + r < nx && j < ny) a[(size_t)(i + r) * ny + j] /= m;
}

// device address of g_scratch, looked up once per device
float *scratch_for_current_device()
{
    static std::mutex mu;
    static float *addr[kMaxDevices] = {};
    int dev = 0;
    NADIA_CUDA(cudaGetDevice(&dev));
    NADIA_REQUIRE(dev >= 0 && dev < kMaxDevices, NADIA_ERR_UNSUPPORTED, "device index too large");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        NADIA_CUDA(cudaGetSymbolAddress(&p, g_scratch));
        NADIA_REQUIRE(p != nullptr, NADIA_ERR_CUDA, "no device address for the scratch array");
        addr[dev] = static_cast<float *>(p);
    }
    return addr[dev];
}

void shrinkwrap(const float *esw, float *support, int nx, int ny, double gauss_width,
                double threshold, cudaStream_t st)
{
    NADIA_REQUIRE(esw && support, NADIA_ERR_INVALID, "null device pointer");
    NADIA_REQUIRE(nx >= 1 && ny >= 1, NADIA_ERR_INVALID, "grid sizes must be positive");
    NADIA_REQUIRE(gauss_width > 0, NADIA_ERR_INVALID, "gauss_width must be positive");
    const long long tx = (ny + kTile - 1) / kTile, ty = (nx + kTile - 1) / kTile;
    NADIA_REQUIRE(tx * ty <= kMaxTiles, NADIA_ERR_INVALID,
                  "grid too large for the no-allocation shrinkwrap: at most 16384 tiles of "
                  "32x32 pixels (4096 x 4096)");
    float *scratch = scratch_for_current_device();
    Taps g;
    for (int d = 0; d <= kCut; ++d)
        g.w[d] = (float)exp(-(double)(d * d) / (2.0 * gauss_width * gauss_width));
    const int ntiles = (int)(tx * ty);
    dim3 grid((unsigned)tx, (unsigned)ty), block(32, 8);
    k_blur_tiles<<<grid, block, 0, st>>>(reinterpret_cast<const float2 *>(esw), support, nx, ny,
                                         g, scratch);
    k_reduce_max<<<1, block, 0, st>>>(scratch, ntiles, scratch + 2 * kMaxTiles);
    k_threshold_tiles<<<grid, block, 0, st>>>(support, nx, ny, threshold,
                                              scratch + 2 * kMaxTiles, scratch + kMaxTiles);
    k_reduce_max<<<1, block, 0, st>>>(scratch + kMaxTiles, ntiles, scratch + 2 * kMaxTiles + 1);
    k_divide_tiles<<<grid, block, 0, st>>>(support, nx, ny, scratch + 2 * kMaxTiles + 1);
    NADIA_CUDA(cudaGetLastError());
}

} // namespace noalloc
} // namespace nadia
