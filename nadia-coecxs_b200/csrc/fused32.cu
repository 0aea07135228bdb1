// fused32.cu -- the fused single-precision iteration.
//
// Every array of a reconstruction lives in the panel layout: element (x, y)
// of the nx-by-ny grid sits at ((y/K)*nx + x)*K + y%K (K = 4), so a block of
// K whole columns is one contiguous run and K*L row segments of L rows are
// contiguous too.  One iteration of BaseCDI::iterate (BaseCDI.c++:297-387)
// for any algorithm without the PfPs term is two passes over HBM:
//
//   column pass: P holds the row transforms of x_k.  Per K columns: forward
//     column FFT -> modulus projection of BaseCDI::scale_intensity
//     (BaseCDI.c++:163-189; FresnelCDI adds/subtracts the white field,
//     FresnelCDI.c++:217-236) with FP64 partial sums of the error metric ->
//     inverse column FFT, written back in place.  The quadrant swaps and
//     1/sqrt(N) scalings of the propagators (Complex_2D::invert,
//     Complex_2D.c++:318-353) are folded in: sqrt(I) is stored in transform
//     order, and for Fresnel the (-1)^(kx+ky) sign of the swap joins the
//     quadratic phase factor of FresnelCDI::multiply_factors.
//   row pass: per L rows: inverse row FFT (-> y = Pf x_k), the combine of
//     BaseCDI.c++:346-383 with the support constraint of BaseCDI.c++:136-154,
//     write x_{k+1}, forward row FFT, write P.  Block 0 also finishes the
//     error metric of the column pass.
//
// Traffic per pixel and iteration: column pass 8 (P) + 4 (sqrt I) read, 8
// written; row pass 8 (P) + 8 (x) + 4 (support) read, 8 + 8 written: 56 bytes
// (48 for ER, which does not read x_k).
#include "fused32.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <tuple>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "batch.h"
#include "fused32_kernels.cuh"
#include "solver.h"

namespace nadia {
namespace f32 {

// ------------------------------------------------------------- shrinkwrap

// separable, edge-skipping blur along y (within rows); absolute value of a
// complex input or a real input
template <bool CPLX>
__global__ void k_blur_y(const void *in, float *out, int nx, int ny, Gauss g)
{
    const size_t n = (size_t)nx * ny;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x) {
        const int kk = (int)(a % kPanel);
        const size_t r = a / kPanel;
        const int i = (int)(r % nx);
        const int p = (int)(r / nx) * kPanel + kk;
        float acc = 0.f;
        for (int d = -g.cut; d <= g.cut; ++d) {
            const int q = p + d;
            if (q < 0 || q >= ny) continue;
            const size_t b = paddr(i, q, nx);
            float val;
            if (CPLX) {
                const float2 c = __ldg(&((const float2 *)in)[b]);
                val = sqrtf(c.x * c.x + c.y * c.y);
            } else {
                val = __ldg(&((const float *)in)[b]);
            }
            acc += g.w[d < 0 ? -d : d] * val;
        }
        out[a] = acc;
    }
}

// blur along x, with a block maximum of the result
__global__ void k_blur_x(const float *in, float *out, int nx, int ny, Gauss g, float *maxpart)
{
    const size_t n = (size_t)nx * ny;
    float m = -INFINITY;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x) {
        const size_t r = a / kPanel;
        const int i = (int)(r % nx);
        float acc = 0.f;
        for (int d = -g.cut; d <= g.cut; ++d) {
            const int q = i + d;
            if (q < 0 || q >= nx) continue;
            acc += g.w[d < 0 ? -d : d] * __ldg(&in[a + (ptrdiff_t)d * kPanel]);
        }
        out[a] = acc;
        m = fmaxf(m, acc);
    }
    __shared__ float red[256];
    red[threadIdx.x] = m;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x == 0) maxpart[blockIdx.x] = red[0];
}

// |x| (or a real input) blurred by the truncated Gaussian over one 32x32 tile
// of the grid, from a 40x40 halo tile in shared memory (rows then columns);
// writes the blurred values and the tile maximum.  Panel layout in and out.
// CUT > 0 fixes the cut-off at compile time (apply_shrinkwrap's 4): the taps
// unroll and the weights stay in registers; CUT = 0 reads it from g.
// Launched with kSwThreads threads (block 32 x 8); every loop has a fixed
// trip count, so a thread issues all its halo loads before it uses one.
// Row strides of 44 and 36 words put the 8 rows x 4 panel columns that a
// warp touches in the halo and column phases on 32 different banks.
constexpr int kSwTile = 32;
constexpr int kSwThreads = 256;
template <bool CPLX, int CUT>
__global__ void __launch_bounds__(kSwThreads) k_blur_tiles(const void *in, float *out, int nx,
                                                           int ny, Gauss g, float *maxpart)
{
    static_assert(CUT >= 0 && CUT <= 4, "the halo holds a cut-off of at most 4");
    constexpr int H = kSwTile + 8; // cut-off up to 4 on each side
    constexpr int NT = kSwThreads;
    __shared__ float tile[H][H + 4];
    __shared__ float rows[H][kSwTile + 4];
    const int cut = CUT > 0 ? CUT : g.cut;
    const int i0 = blockIdx.y * kSwTile - 4, j0 = blockIdx.x * kSwTile - 4;
    const int t = threadIdx.y * blockDim.x + threadIdx.x;
    // halo: panel-major so that each panel's rows are one contiguous run
#pragma unroll
    for (int k = 0; k < (H * H + NT - 1) / NT; ++k) {
        const int e = t + k * NT;
        if (e < H * H) {
            const int jj = e % kPanel, a = (e / kPanel) % H, pb = e / (kPanel * H);
            const int i = i0 + a, j = j0 + pb * kPanel + jj;
            float v = 0.f;
            if (i >= 0 && i < nx && j >= 0 && j < ny) {
                const size_t ad = paddr(i, j, nx);
                if (CPLX) {
                    const float2 c = __ldg(&((const float2 *)in)[ad]);
                    v = sqrtf(c.x * c.x + c.y * c.y);
                } else {
                    v = __ldg(&((const float *)in)[ad]);
                }
            }
            tile[a][pb * kPanel + jj] = v;
        }
    }
    __syncthreads();
    static_assert(H * kSwTile % NT == 0 && kSwTile * kSwTile % NT == 0, "whole rounds");
#pragma unroll
    for (int k = 0; k < H * kSwTile / NT; ++k) {
        const int e = t + k * NT;
        const int a = e / kSwTile, b = e % kSwTile;
        float acc = 0.f;
#pragma unroll
        for (int d = -cut; d <= cut; ++d) acc += g.w[d < 0 ? -d : d] * tile[a][b + 4 + d];
        rows[a][b] = acc;
    }
    __syncthreads();
    float m = -INFINITY;
#pragma unroll
    for (int k = 0; k < kSwTile * kSwTile / NT; ++k) {
        const int e = t + k * NT;
        const int jj = e % kPanel, a = (e / kPanel) % kSwTile, pb = e / (kPanel * kSwTile);
        const int b = pb * kPanel + jj;
        const int i = blockIdx.y * kSwTile + a, j = blockIdx.x * kSwTile + b;
        if (i < nx && j < ny) {
            float acc = 0.f;
#pragma unroll
            for (int d = -cut; d <= cut; ++d) acc += g.w[d < 0 ? -d : d] * rows[a + 4 + d][b];
            out[paddr(i, j, nx)] = acc;
            m = fmaxf(m, acc);
        }
    }
    // block maximum: warps by shuffles, then the 8 warp maxima
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    __shared__ float red[NT / 32];
    if ((t & 31) == 0) red[t >> 5] = m;
    __syncthreads();
    if (t == 0) {
        float r = red[0];
#pragma unroll
        for (int w = 1; w < NT / 32; ++w) r = fmaxf(r, red[w]);
        maxpart[blockIdx.y * gridDim.x + blockIdx.x] = r;
    }
}

// Square grids visit every element once in apply_threshold, so the values
// become 0/1 and their maximum is 1 when the largest blurred value passes
// its own threshold (max >= t*max) and 0 otherwise: threshold and the
// division by that maximum in one pass.
__global__ void k_threshold_divide_square(const float *in, float *out, size_t n, double t,
                                          const float *dmax)
{
    const double mx = (double)(*dmax);
    const double lim = t * mx;
    const float max2 = (mx >= lim) ? 1.f : 0.f;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x) {
        const float v = ((double)in[a] < lim) ? 0.f : 1.f;
        out[a] = v / max2;
    }
}

__global__ void k_max(const float *in, size_t n, float *maxpart)
{
    float m = -INFINITY;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x)
        m = fmaxf(m, in[a]);
    __shared__ float red[256];
    red[threadIdx.x] = m;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x == 0) maxpart[blockIdx.x] = red[0];
}

__global__ void k_max_final(float *maxpart, int nb)
{
    __shared__ float red[256];
    float m = -INFINITY;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) m = fmaxf(m, maxpart[b]);
    red[threadIdx.x] = m;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if (threadIdx.x < off) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + off]);
        __syncthreads();
    }
    if (threadIdx.x == 0) maxpart[nb] = red[0];
}

// BaseCDI::apply_threshold (BaseCDI.c++:477-492) with its loop bounds i < nx,
// j < nx over the row-major index L = i*ny + j; element (i, p) is visited once
// per pair (i', j' = L - i'*ny), 0 <= j' < nx, and reads 0 when j' > ny.
__global__ void k_threshold(float *a, int nx, int ny, double t, const float *dmax)
{
    const double lim = t * (double)(*dmax);
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int kk = (int)(e % kPanel);
        const size_t r = e / kPanel;
        const int i = (int)(r % nx);
        const int p = (int)(r / nx) * kPanel + kk;
        const long long L = (long long)i * ny + p;
        long long ilo = L - nx + 1 < 0 ? 0 : (L - nx + 1 + ny - 1) / ny;
        long long ihi = L / ny;
        if (ihi > nx - 1) ihi = nx - 1;
        if (ilo > ihi) continue;
        float cur = a[e];
        for (long long ii = ilo; ii <= ihi; ++ii) {
            const long long j = L - ii * ny;
            const float v = (j > ny) ? 0.f : cur;
            cur = ((double)v < lim) ? 0.f : 1.f;
        }
        a[e] = cur;
    }
}

__global__ void k_divide(const float *in, float *out, size_t n, const float *dmax)
{
    const float m = *dmax;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x)
        out[a] = in[a] / m;
}

// ESW = T*L - L (FresnelCDI.c++:253-283, with its `j < nx` bound) in panel layout
__global__ void k_fresnel_set_t(const float2 *t, const float2 *ill, float2 *esw, int nx, int ny)
{
    const size_t n = (size_t)nx * ny;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x) {
        const int kk = (int)(a % kPanel);
        const int p = (int)(a / kPanel / nx) * kPanel + kk;
        if (ny >= nx && p >= nx) continue;
        const float2 l = ill[a], tt = t[a];
        esw[a] = make_float2(l.x * tt.x - l.y * tt.y - l.x, l.x * tt.y + l.y * tt.x - l.y);
    }
}

// the constraint's per-pixel part over a whole panel-layout array (the
// transmission function FresnelCDI::get_transmission_function returns)
// per block and region: the sums of |ln|t|| and |arg t| over the region's
// pixels (FP64, each thread in pixel order, then the block's fixed tree);
// the region map streams as int4 (four pixels of a panel row)
__global__ void __launch_bounds__(kTcThreads) k_tc32_sums(const Slot *slot, int field,
                                                          const float2 *arr, size_t n)
{
    const Slot &S = *slot;
    const int R = S.tc_R;
    double lnA[kTcMaxRegions], ph[kTcMaxRegions];
#pragma unroll
    for (int r = 0; r < kTcMaxRegions; ++r) lnA[r] = ph[r] = 0.0;
    const int4 *reg4 = reinterpret_cast<const int4 *>(S.tc_region);
    for (size_t q = blockIdx.x * (size_t)kTcThreads + threadIdx.x; q < n / 4;
         q += (size_t)gridDim.x * kTcThreads) {
        const int4 rr = __ldg(&reg4[q]);
        const int rv[4] = {rr.x, rr.y, rr.z, rr.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int r = rv[c];
            if (r > 0) {
                const float2 t = tc_field(S, 4 * q + c, field, arr);
#pragma unroll
                for (int k = 0; k < kTcMaxRegions; ++k)
                    if (k == r - 1) {
                        ph[k] += fabs((double)atan2f(t.y, t.x));
                        lnA[k] += fabs((double)logf(sqrtf(t.x * t.x + t.y * t.y)));
                    }
            }
        }
    }
    for (int r = 0; r < R; ++r) {
        const double a = block_sum<kTcThreads>(lnA[r]);
        __syncthreads();
        const double b = block_sum<kTcThreads>(ph[r]);
        if (threadIdx.x == 0) {
            S.tc_part[2 * ((size_t)blockIdx.x * R + r)] = a;
            S.tc_part[2 * ((size_t)blockIdx.x * R + r) + 1] = b;
        }
        __syncthreads();
    }
}

// one block per region: the blocks' partials in a fixed order, then c_mean
// (the region's fixed value where one was set)
__global__ void __launch_bounds__(kTcThreads) k_tc32_cmean(const Slot *slot, int field, int nblocks)
{
    const Slot &S = *slot;
    const int R = S.tc_R, r = blockIdx.x;
    double a = 0.0, b = 0.0;
    for (int blk = threadIdx.x; blk < nblocks; blk += kTcThreads) {
        a += S.tc_part[2 * ((size_t)blk * R + r)];
        b += S.tc_part[2 * ((size_t)blk * R + r) + 1];
    }
    a = block_sum<kTcThreads>(a);
    __syncthreads();
    b = block_sum<kTcThreads>(b);
    if (threadIdx.x == 0)
        S.tc_cm[field * R + r] = S.tc_par[4 * r + 2] != 0.f ? S.tc_par[4 * r + 3] : (float)(a / b);
}

// the whole constraint on an array of transmission functions (or estimates)
// whose c_mean is field 2's (get_transmission_function, FresnelCDI.c++:352-353)
__global__ void k_tc32_apply_array(float2 *t, size_t n, const Slot *slot)
{
    const Slot &S = *slot;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x) {
        float2 v = t[a];
        const int r = S.tc_R > 0 ? S.tc_region[a] : 0;
        if (r > 0) v = tc_region_update(v, S.tc_par + 4 * (r - 1), S.tc_cm[2 * S.tc_R + r - 1]);
        t[a] = tc_pixel(v, S);
    }
}

__global__ void k_tc_pixels(float2 *t, size_t n, const Slot *slot)
{
    const Slot &S = *slot;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x)
        t[a] = tc_pixel(t[a], S);
}

// panel layout (float) <-> the reference's order (double), on the device
__global__ void k_panel_widen(const float2 *src, double2 *dst, int nx, int ny)
{
    const size_t n = (size_t)nx * ny;
    for (size_t d = blockIdx.x * (size_t)blockDim.x + threadIdx.x; d < n;
         d += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(d / ny), yy = (int)(d % ny);
        const float2 v = src[panel_index_dev(xx, yy, nx)];
        dst[d] = make_double2(v.x, v.y);
    }
}

__global__ void k_panel_narrow(const double2 *src, float2 *dst, int nx, int ny)
{
    const size_t n = (size_t)nx * ny;
    for (size_t d = blockIdx.x * (size_t)blockDim.x + threadIdx.x; d < n;
         d += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(d / ny), yy = (int)(d % ny);
        const double2 v = src[d];
        dst[panel_index_dev(xx, yy, nx)] = make_float2((float)v.x, (float)v.y);
    }
}

// T = (ESW + L) / L, 1 where L = 0 (FresnelCDI.c++:298-355)
__global__ void k_fresnel_get_t(const float2 *esw, const float2 *ill, float2 *out, size_t n)
{
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x) {
        const float2 l = ill[a];
        const float denom = l.x * l.x + l.y * l.y;
        if (denom != 0.f) {
            const float2 e = esw[a];
            const float rn = l.x * (e.x + l.x) + l.y * (e.y + l.y);
            const float in = l.x * (e.y + l.y) - l.y * (e.x + l.x);
            out[a] = make_float2(rn / denom, in / denom);
        } else {
            out[a] = make_float2(1.f, 0.f);
        }
    }
}

__global__ void k_support_apply(float2 *c, const float *sup, size_t n)
{
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x)
        c[a] = cscale(c[a], support_factor(sup[a]));
}

__global__ void k_scale32(float2 *c, float f, size_t n)
{
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x)
        c[a] = cscale(c[a], f);
}

// twiddle tables W[t] = exp(-2 pi i t / N) per device and length
const float2 *twiddle_table(int n)
{
    static std::mutex mu;
    static std::map<std::pair<int, int>, float2 *> tables;
    int dev = 0;
    NADIA_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    auto it = tables.find({dev, n});
    if (it != tables.end()) return it->second;
    std::vector<double2> w = twiddles(n);
    std::vector<float2> f(n);
    for (int t = 0; t < n; ++t) f[t] = make_float2((float)w[t].x, (float)w[t].y);
    float2 *d = nullptr;
    NADIA_CUDA(cudaMalloc(&d, n * sizeof(float2)));
    upload_now(d, f.data(), n * sizeof(float2));
    tables[{dev, n}] = d;
    return d;
}

inline int grid1(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }

int sm_count()
{
    static int n = [] {
        int dev = 0, v = 0;
        NADIA_CUDA(cudaGetDevice(&dev));
        NADIA_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        return v;
    }();
    return n;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda)
namespace {
using EncodeFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                              const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                              const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeFn encode_fn()
{
    static EncodeFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        NADIA_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        NADIA_REQUIRE(p && q == cudaDriverEntryPointSuccess, NADIA_ERR_CUDA,
                      "cuTensorMapEncodeTiled unavailable");
        return reinterpret_cast<EncodeFn>(p);
    }();
    return fn;
}

// panel-layout array (K, nx, ny/K) of 8- or 4-byte elements, box (K, rows, <=256)
void encode_one(CUtensorMap *m, void *base, bool complex8, int nx, int ny, int rows)
{
    const int npan = ny / kPanel;
    const cuuint64_t esz = complex8 ? 8 : 4;
    cuuint64_t dims[3] = {(cuuint64_t)kPanel, (cuuint64_t)nx, (cuuint64_t)npan};
    cuuint64_t strides[2] = {kPanel * esz, (cuuint64_t)nx * kPanel * esz};
    cuuint32_t box[3] = {(cuuint32_t)kPanel, (cuuint32_t)rows, (cuuint32_t)box_panels(npan)};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(m, complex8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                             3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    NADIA_REQUIRE(r == CUDA_SUCCESS, NADIA_ERR_CUDA,
                  "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}
} // namespace

// panel-layout array (K, nx, ny/K) viewed by the grouped column pass: box
// (cols of a panel, box_rows(nx) rows, 1 panel)
void encode_cols(CUtensorMap *m, void *base, bool complex8, int nx, int ny, int cols)
{
    const int npan = ny / kPanel;
    const cuuint64_t esz = complex8 ? 8 : 4;
    cuuint64_t dims[3] = {(cuuint64_t)kPanel, (cuuint64_t)nx, (cuuint64_t)npan};
    cuuint64_t strides[2] = {kPanel * esz, (cuuint64_t)nx * kPanel * esz};
    cuuint32_t box[3] = {(cuuint32_t)cols, (cuuint32_t)box_rows(nx), 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(m, complex8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                             3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    NADIA_REQUIRE(r == CUDA_SUCCESS, NADIA_ERR_CUDA,
                  "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

void encode_tensor_maps(Slot &s, int nx, int ny)
{
    encode_cols(&s.tc[0], s.P, true, nx, ny, 2);
    encode_cols(&s.tc[1], (void *)s.mI, false, nx, ny, 4);
    const int rows[5] = {1, 2, 4, 8, 16};
    for (int k = 0; k < 5; ++k) {
        if (nx % rows[k]) {
            std::memset(&s.tm[k][0], 0, sizeof(s.tm[k]));
            continue;
        }
        encode_one(&s.tm[k][0], s.P, true, nx, ny, rows[k]);
        encode_one(&s.tm[k][1], s.x, true, nx, ny, rows[k]);
        encode_one(&s.tm[k][2], (void *)s.sup, false, nx, ny, rows[k]);
    }
}

// ---------------------------------------------------------------- registry

void add_variants_256(std::vector<TileVariant> &);
void add_variants_512(std::vector<TileVariant> &);
void add_variants_768(std::vector<TileVariant> &);
void add_variants_1024(std::vector<TileVariant> &);
void add_variants_1536(std::vector<TileVariant> &);
void add_variants_2048(std::vector<TileVariant> &);
void add_variants_4096(std::vector<TileVariant> &);

const std::vector<TileVariant> &variants(int n)
{
    static const std::map<int, std::vector<TileVariant>> reg = [] {
        std::map<int, std::vector<TileVariant>> m;
        add_variants_256(m[256]);
        add_variants_512(m[512]);
        add_variants_768(m[768]);
        add_variants_1024(m[1024]);
        add_variants_1536(m[1536]);
        add_variants_2048(m[2048]);
        add_variants_4096(m[4096]);
        return m;
    }();
    static const std::vector<TileVariant> none;
    auto it = reg.find(n);
    return it == reg.end() ? none : it->second;
}

bool supported(int n) { return !variants(n).empty(); }

// ---------------------------------------------------------------- autotuner
//
// The first reconstruction of a given grid, kind and batch class times every
// compiled column variant (transform length nx) and row variant (length ny)
// on scratch buffers of that shape with CUDA events, and keeps the fastest.
// The scratch slots hold measured-everywhere data, so the timed work is the
// full iteration.  NADIA_TUNE=0 in the environment skips the timing and takes
// the first variant of each length; NADIA_TUNE_VERBOSE=1 prints the timings;
// NADIA_TUNE_FILE=<path> reads earlier choices from that file and appends new
// ones (lines "nx ny fresnel batch col_variant row_variant"), so a later run
// -- under a profiler, say -- reuses the variants an undisturbed run picked.

namespace {

struct TuneKey {
    int dev, nx, ny, fresnel, batch, plain_rows;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(dev, nx, ny, fresnel, batch, plain_rows) <
               std::tie(o.dev, o.nx, o.ny, o.fresnel, o.batch, o.plain_rows);
    }
};

// mean of `reps` back-to-back launches after two untimed ones; the best of
// two such rounds (the first round of a process can run at ramping clocks)
float time_launches(const std::function<void(cudaStream_t)> &f, cudaStream_t st, int reps)
{
    cudaEvent_t a, b;
    NADIA_CUDA(cudaEventCreate(&a));
    NADIA_CUDA(cudaEventCreate(&b));
    float best = 1e30f;
    for (int round = 0; round < 2; ++round) {
        f(st);
        f(st);
        NADIA_CUDA(cudaEventRecord(a, st));
        for (int i = 0; i < reps; ++i) f(st);
        NADIA_CUDA(cudaEventRecord(b, st));
        NADIA_CUDA(cudaEventSynchronize(b));
        float ms = 0;
        NADIA_CUDA(cudaEventElapsedTime(&ms, a, b));
        best = std::min(best, ms * 1000.f / reps);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

} // namespace

const Choice &choose(int nx, int ny, bool fresnel, int nslots, bool plain_rows, bool wf)
{
    static std::mutex mu;
    static std::map<TuneKey, Choice> cache;
    int dev = 0;
    NADIA_CUDA(cudaGetDevice(&dev));
    const int batch = nslots > 1 ? 4 : 1;
    const int kind = wf ? 2 : (fresnel ? 1 : 0);
    TuneKey key{dev, nx, ny, kind, batch, plain_rows ? 1 : 0};
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;

    const auto &cv = variants(nx), &rv = variants(ny);
    NADIA_REQUIRE(!cv.empty() && !rv.empty(), NADIA_ERR_UNSUPPORTED,
                  "the FP32 form supports 256, 512, 768, 1024, 1536, 2048 and 4096 per axis");
    for (const auto &v : cv) v.prepare();
    for (const auto &v : rv) v.prepare();
    Choice ch;
    const char *env = getenv("NADIA_TUNE");
    const bool tune = !(env && env[0] == '0');
    const bool verbose = getenv("NADIA_TUNE_VERBOSE") != nullptr;
    // pick the first variant whose tiles divide the grid (and tune among those)
    std::vector<const TileVariant *> cols, rows;
    for (const auto &v : cv)
        if ((wf ? v.wf_col != nullptr : v.col != nullptr) && ny % v.L == 0) cols.push_back(&v);
    for (const auto &v : rv)
        if ((wf ? v.wf_row != nullptr : v.row != nullptr) && nx % v.L == 0 &&
            !(plain_rows && v.persistent))
            rows.push_back(&v);
    NADIA_REQUIRE(!cols.empty() && !rows.empty(), NADIA_ERR_UNSUPPORTED,
                  "grid shape does not divide into the FP32 tiles");
    ch.col = cols[0];
    ch.row = rows[0];
    const char *tfile = plain_rows ? nullptr : getenv("NADIA_TUNE_FILE");
    if (tfile) {
        if (FILE *f = fopen(tfile, "r")) {
            int a, b, c, d, ci, ri;
            while (fscanf(f, "%d %d %d %d %d %d", &a, &b, &c, &d, &ci, &ri) == 6)
                if (a == nx && b == ny && c == kind && d == batch && ci >= 0 &&
                    ci < (int)cv.size() && ri >= 0 && ri < (int)rv.size() &&
                    (wf ? cv[ci].wf_col != nullptr : cv[ci].col != nullptr) &&
                    (wf ? rv[ri].wf_row != nullptr : rv[ri].row != nullptr) &&
                    ny % cv[ci].L == 0 && nx % rv[ri].L == 0) {
                    ch.col = &cv[ci];
                    ch.row = &rv[ri];
                    fclose(f);
                    return cache[key] = ch;
                }
            fclose(f);
        }
    }
    if (tune && (cols.size() > 1 || rows.size() > 1)) {
        const size_t n = (size_t)nx * ny;
        const int ns = batch;
        cudaStream_t st;
        NADIA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        std::vector<DevBuf<float2>> P(ns), X(ns);
        std::vector<DevBuf<float>> sup(ns), mI(ns);
        DevBuf<float2> W(n), tx(nx), ty(ny);
        int maxcol = 0; // error partials: one per column tile (per row tile for FresnelCDI_WF)
        for (auto *v : cols) maxcol = std::max(maxcol, ny / v->L);
        for (auto *v : rows) maxcol = std::max(maxcol, nx / v->L);
        DevBuf<double> part((size_t)maxcol * ns), err(ns), ring(ns * 4);
        DevBuf<long long> iter(ns);
        DevBuf<int> flag(1);
        NADIA_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
        std::vector<Slot> hs(ns);
        NADIA_CUDA(cudaMemsetAsync(W.p, 0, W.bytes(), st));
        NADIA_CUDA(cudaMemsetAsync(tx.p, 0, tx.bytes(), st));
        NADIA_CUDA(cudaMemsetAsync(ty.p, 0, ty.bytes(), st));
        NADIA_CUDA(cudaMemsetAsync(iter.p, 0, iter.bytes(), st));
        for (int i = 0; i < ns; ++i) {
            P[i].alloc(n); X[i].alloc(n); sup[i].alloc(n); mI[i].alloc(n);
            NADIA_CUDA(cudaMemsetAsync(P[i].p, 0, P[i].bytes(), st));
            NADIA_CUDA(cudaMemsetAsync(X[i].p, 0, X[i].bytes(), st));
            NADIA_CUDA(cudaMemsetAsync(sup[i].p, 0, sup[i].bytes(), st));
            NADIA_CUDA(cudaMemsetAsync(mI[i].p, 0, mI[i].bytes(), st));
            Slot &s = hs[i];
            s = Slot{};
            s.P = P[i].p; s.x = X[i].p; s.sup = sup[i].p; s.mI = mI[i].p;
            s.W = fresnel ? W.p : nullptr;
            s.tx = (fresnel || wf) ? tx.p : nullptr; // FresnelCDI_WF: the zone-plate factors
            s.ty = (fresnel || wf) ? ty.p : nullptr;
            s.partials = part.p + (size_t)i * maxcol; s.err = err.p + i; s.ring = ring.p + 4 * i;
            s.ring_len = 4; s.iter = iter.p + i; s.ncol = 1; s.w_id = 1; s.w_pf = -0.9f;
            s.w_ps = -1; s.w_psf = 1.9f; s.project = 1; s.s0 = 1.f; s.inv_norm2 = 1.0;
            s.flag = flag.p;
            encode_tensor_maps(s, nx, ny);
        }
        DevBuf<Slot> dslots(ns);
        DevBuf<Slot *> dptrs(ns);
        std::vector<Slot *> hp(ns);
        for (int i = 0; i < ns; ++i) hp[i] = dslots.p + i;
        NADIA_CUDA(cudaMemcpyAsync(dslots.p, hs.data(), ns * sizeof(Slot), cudaMemcpyHostToDevice, st));
        NADIA_CUDA(cudaMemcpyAsync(dptrs.p, hp.data(), ns * sizeof(Slot *), cudaMemcpyHostToDevice, st));
        NADIA_CUDA(cudaStreamSynchronize(st));
        const float2 *twx = twiddle_table(nx), *twy = twiddle_table(ny);
        // bring the clocks up before timing anything
        auto run_col = [&](const TileVariant *v, cudaStream_t s) {
            if (wf)
                v->wf_col(dptrs.p, ns, nx, ny, twx, s);
            else
                v->col(fresnel, dptrs.p, ns, nx, ny, twx, s);
        };
        for (int i = 0; i < 20; ++i) run_col(cols[0], st);
        NADIA_CUDA(cudaStreamSynchronize(st));
        float best = 1e30f;
        for (auto *v : cols) {
            float us = time_launches([&](cudaStream_t s) { run_col(v, s); }, st, 5);
            if (verbose)
                fprintf(stderr, "nadia tune: %scol n=%d NT=%d L=%d radices=%s%s batch=%d: %.2f us\n",
                        wf ? "FresnelCDI_WF " : "", nx, v->nt, v->L, v->radices,
                        v->single ? " persistent-1stage" : (v->persistent ? " persistent" : (v->ping ? " ping" : "")),
                        ns, us);
            if (us < best) { best = us; ch.col = v; ch.col_us = us; }
        }
        best = 1e30f;
        for (auto *v : rows) {
            float us = time_launches([&](cudaStream_t s) {
                if (wf)
                    v->wf_row(kRowFull, dptrs.p, ns, nx, ny, twy, s);
                else
                    v->row(kRowFull, dptrs.p, ns, nx, ny, twy, s);
            }, st, 5);
            if (verbose)
                fprintf(stderr, "nadia tune: %srow n=%d NT=%d L=%d G=%d radices=%s%s batch=%d: %.2f us\n",
                        wf ? "FresnelCDI_WF " : "", ny, v->nt, v->L, v->groups, v->radices,
                        v->persistent ? " persistent" : (v->ping ? " ping" : ""), ns, us);
            if (us < best) { best = us; ch.row = v; ch.row_us = us; }
        }
        NADIA_CUDA(cudaGetLastError());
        NADIA_CUDA(cudaStreamSynchronize(st));
        int fl = 0;
        NADIA_CUDA(cudaMemcpy(&fl, flag.p, sizeof(int), cudaMemcpyDeviceToHost));
        cudaStreamDestroy(st);
        NADIA_REQUIRE(fl == 0, NADIA_ERR_CUDA, "a device-side wait timed out while tuning");
    }
    if (tfile) {
        if (FILE *f = fopen(tfile, "a")) {
            fprintf(f, "%d %d %d %d %d %d\n", nx, ny, kind, batch,
                    (int)(ch.col - cv.data()), (int)(ch.row - rv.data()));
            fclose(f);
        }
    }
    return cache[key] = ch;
}

} // namespace f32

// =================================================================== host

using namespace f32;

Fused32::Fused32(Solver &s) : impl(new Impl(s)) {}
Fused32::~Fused32() { delete impl; }

Fused32::Impl::Impl(Solver &s) : S(s)
{
    nx = s.nx;
    ny = s.ny;
    n = s.n;
    const bool poly = s.kind == NADIA_POLY;
    const bool wf = s.kind == NADIA_FRESNEL_WF;
    if (poly) {
        // the transforms run on the padded grid, sized by set_spectrum
        NADIA_REQUIRE(nx % 8 == 0 && ny % 4 == 0, NADIA_ERR_UNSUPPORTED,
                      "the FP32 PolyCDI form needs nx a multiple of 8 and ny of 4");
    } else {
        NADIA_REQUIRE(supported(nx) && supported(ny), NADIA_ERR_UNSUPPORTED,
                      "the FP32 form supports grid sizes 256, 512, 768, 1024, 1536, 2048 and "
                      "4096 per axis; use NADIA_FP64 for other sizes");
        if (wf) {
            const Choice &c = choose(nx, ny, false, 1, false, true);
            wfc = c.col;
            wfr = c.row;
        } else {
            choice = &choose(nx, ny, s.kind == NADIA_FRESNEL, 1);
        }
    }
    P.alloc(n);
    x.alloc(n);
    sup.alloc(n);
    mI.alloc(n);
    // error partials: one per column tile (tiles of two columns at least), or
    // for FresnelCDI_WF one per row tile
    ncol = poly ? 0 : (wf ? nx / wfr->L : ny / choice->col->L);
    partials.alloc(wf ? nx : ny / 2);
    iter.alloc(1);
    flag.alloc(1);
    slot.alloc(1);
    slot_ptr.alloc(1);
    cudaStream_t st = s.st;
    NADIA_CUDA(cudaMemsetAsync(P.p, 0, P.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(x.p, 0, x.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(sup.p, 0, sup.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(mI.p, 0, mI.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(partials.p, 0, partials.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(iter.p, 0, iter.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(flag.p, 0, flag.bytes(), st));
    if (!poly) {
        twx = twiddle_table(nx);
        twy = twiddle_table(ny);
    }
    h_slot = Slot{};
    h_slot.P = P.p;
    h_slot.x = x.p;
    h_slot.sup = sup.p;
    h_slot.mI = mI.p;
    h_slot.partials = partials.p;
    h_slot.err = s.d_err.p;
    h_slot.ring = s.d_ring.p;
    h_slot.ring_len = Solver::kRing;
    h_slot.iter = iter.p;
    h_slot.ncol = ncol;
    h_slot.s0 = (float)(1.0 / sqrt((double)nx * (double)ny));
    h_slot.inv_norm2 = 0.0;
    h_slot.flag = flag.p;
    // test hook for the bounded-wait failure path (Slot::skip_first_load)
    if (const char *fw = getenv("NADIA_FAULT_WAIT")) {
        const long polls = strtol(fw, nullptr, 10);
        if (polls > 0) {
            h_slot.wait_polls = (unsigned)polls;
            h_slot.skip_first_load = 1;
        }
    }
    if (!poly) encode_tensor_maps(h_slot, nx, ny);
    Slot *sp = slot.p;
    NADIA_CUDA(cudaMemcpyAsync(slot_ptr.p, &sp, sizeof(Slot *), cudaMemcpyHostToDevice, st));
    push_slot();
}

Fused32::Impl::~Impl()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph_pfs) cudaGraphExecDestroy(graph_pfs);
}

void Fused32::Impl::use_choice(const f32::Choice *c)
{
    h_slot.ncol = ny / c->col->L;
}

void Fused32::Impl::push_slot()
{
    if (push_slot_async(S.st)) NADIA_CUDA(cudaStreamSynchronize(S.st));
}

// Uploads the descriptor only when it changed since the last upload: a copy
// from pageable memory may wait for the stream's queued work, which would
// stop the host from queueing further iterations while the device runs.
bool Fused32::Impl::push_slot_async(cudaStream_t st)
{
    flush_intensity();
    const double *w = S.w;
    h_slot.er = (S.algorithm == NADIA_ER);
    h_slot.w_id = (float)(1 + w[PI]);
    h_slot.w_pf = (float)w[PF];
    h_slot.w_ps = (float)w[PS];
    h_slot.w_psf = (float)w[PSF];
    h_slot.project = h_slot.er || w[PF] != 0 || w[PSF] != 0;
    h_slot.pfs = pfs_mode() ? 1 : 0;
    h_slot.w_pfs = (float)w[PFS];
    if (S.kind == NADIA_FRESNEL_WF) h_slot.project = 1; // its fixed iteration projects
    bool copied = false;
    if (h_slot.pfs && qslot) {
        // Q's column pass: the same reconstruction with Q as its work array
        Slot q = h_slot;
        q.P = Q.p;
        q.partials = qpartials.p;
        if (!qslot_uploaded || std::memcmp(&q, &qslot_on_device, sizeof(Slot)) != 0) {
            NADIA_CUDA(cudaMemcpyAsync(qslot.p, &q, sizeof(Slot), cudaMemcpyHostToDevice, st));
            qslot_on_device = q;
            qslot_uploaded = true;
            copied = true;
        }
    }
    if (slot_uploaded && std::memcmp(&h_slot, &slot_on_device, sizeof(Slot)) == 0) return copied;
    // pageable source: the copy is staged before this returns
    NADIA_CUDA(cudaMemcpyAsync(slot.p, &h_slot, sizeof(Slot), cudaMemcpyHostToDevice, st));
    slot_on_device = h_slot;
    slot_uploaded = true;
    return true;
}

bool Fused32::Impl::pfs_mode() const
{
    return S.kind != NADIA_FRESNEL_WF && S.algorithm != NADIA_ER && S.w[PFS] != 0;
}

// algorithms with a PfPs term: Q (rows of Ps x), its error partials and the
// descriptor of its column pass, allocated on first use; the row pass runs
// in a non-persistent variant (it carries two fields)
void Fused32::Impl::prepare_pfs()
{
    if (!Q) {
        Q.alloc(n);
        qpartials.alloc(ny / 2);
        qslot.alloc(1);
        qslot_ptr.alloc(1);
        NADIA_CUDA(cudaMemsetAsync(Q.p, 0, Q.bytes(), S.st));
        NADIA_CUDA(cudaMemsetAsync(qpartials.p, 0, qpartials.bytes(), S.st));
        Slot *qp = qslot.p;
        NADIA_CUDA(cudaMemcpyAsync(qslot_ptr.p, &qp, sizeof(Slot *), cudaMemcpyHostToDevice, S.st));
        NADIA_CUDA(cudaStreamSynchronize(S.st));
        h_slot.Q = Q.p;
        h_slot.qpartials = qpartials.p;
        q_valid = false;
    }
    if (!pfs_choice) pfs_choice = &choose(nx, ny, S.kind == NADIA_FRESNEL, 1, true);
}

// Host arrays are in the reference's order (element (x, y) at x*ny + y); the
// device arrays in the panel layout.  The host converts, so uploads and
// readbacks are plain copies: they run on the copy engines and never wait
// for SMs held by other reconstructions' passes.
namespace {
// host array (x*ny + y order, stride values per element, of type T) to the
// panel layout in FP32, converted in the same pass
template <class T>
void to_panel(const T *h, int stride, float *p, int nx, int ny, bool fold)
{
    // x outer, y inner: the source is read in order, and the panel rows a
    // column writes (16 bytes each) are the next column's neighbours
    for (int kx = 0; kx < nx; ++kx) {
        int dx = kx;
        if (fold) {
            dx = kx + nx / 2;
            dx = dx >= nx ? dx - nx : dx;
        }
        const T *src = h + (size_t)dx * ny * stride;
        for (int ky = 0; ky < ny; ++ky) {
            int dy = ky;
            if (fold) {
                dy = ky + ny / 2;
                dy = dy >= ny ? dy - ny : dy;
            }
            const size_t a = panel_index_dev(kx, ky, nx);
            for (int c = 0; c < stride; ++c) p[a * stride + c] = (float)src[(size_t)dy * stride + c];
        }
    }
}
} // namespace

// the host staging array of the conversions, kept between calls (a fresh
// one would be page-faulted in again on every upload and readback)
float *Fused32::Impl::staging(size_t count)
{
    if (stage.size() < count) stage.resize(count);
    return stage.data();
}

void Fused32::Impl::put_panel_f(const float *h, int stride, void *dst, bool fold)
{
    float *p = staging(n * stride);
    to_panel(h, stride, p, nx, ny, fold);
    NADIA_CUDA(cudaMemcpyAsync(dst, p, n * stride * sizeof(float), cudaMemcpyHostToDevice, S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
}

void Fused32::Impl::put_panel(const double *h, int stride, void *dst, bool fold)
{
    float *p = staging(n * stride);
    to_panel(h, stride, p, nx, ny, fold);
    NADIA_CUDA(cudaMemcpyAsync(dst, p, n * stride * sizeof(float), cudaMemcpyHostToDevice, S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
}

namespace {
// panel layout (FP32) to the reference's order, converted to T in the pass
template <class T>
void from_panel(const float *p, int stride, T *h, int nx, int ny)
{
    for (int xx = 0; xx < nx; ++xx)
        for (int yy = 0; yy < ny; ++yy) {
            const size_t a = panel_index_dev(xx, yy, nx), d = (size_t)xx * ny + yy;
            for (int c = 0; c < stride; ++c) h[d * stride + c] = (T)p[a * stride + c];
        }
}
} // namespace

void Fused32::Impl::get_panel_f(const void *src, int stride, float *h)
{
    float *p = staging(n * stride);
    NADIA_CUDA(cudaMemcpyAsync(p, src, n * stride * sizeof(float), cudaMemcpyDeviceToHost, S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
    from_panel(p, stride, h, nx, ny);
}

void Fused32::Impl::get_panel(const void *src, int stride, double *h)
{
    float *p = staging(n * stride);
    NADIA_CUDA(cudaMemcpyAsync(p, src, n * stride * sizeof(float), cudaMemcpyDeviceToHost, S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
    from_panel(p, stride, h, nx, ny);
}

// set_intensity and set_beam_stop mark sqrt(I) for conversion; it is formed
// once, when the reconstruction's estimate is set or before its descriptor
// goes to the device (every launch path pushes the descriptor first)
void Fused32::Impl::upload_intensity() { mI_dirty = true; }

// sqrt(I) in transform order with the unmeasured pixels marked -1; the
// normalisation sum of BaseCDI::scale_intensity over the measured pixels
void Fused32::Impl::flush_intensity()
{
    if (!mI_dirty) return;
    mI_dirty = false;
    std::vector<float> &m = mstage; // kept between calls, like the staging array
    m.resize(n);
    double norm2 = 0;
    for (size_t d = 0; d < n; ++d) {
        const bool measured = !S.has_beam_stop || h_bs[d] > 0;
        const float v = (float)S.h_isqrt[d];
        if (measured) norm2 += (double)v * (double)v;
        m[d] = measured ? v : -1.f;
    }
    // PlanarCDI's detector is centred (Complex_2D::invert): fold it into
    // transform order; Fresnel folds the swap into its phase factors, and
    // PolyCDI gathers in centred coordinates
    put_panel_f(m.data(), 1, mI.p, S.kind == NADIA_PLANAR);
    h_slot.inv_norm2 = 1.0 / norm2;
    push_slot();
}

void Fused32::upload_intensity() { impl->upload_intensity(); }

void Fused32::upload_beam_stop(const double *mask)
{
    impl->h_bs.assign(mask, mask + impl->n);
    impl->upload_intensity();
}

void Fused32::upload_support(const double *h)
{
    impl->put_panel(h, 1, impl->sup.p, false);
    impl->q_valid = false; // Q holds the rows of Ps x
}

void Fused32::soften_support()
{
    // BaseCDI::set_support's convolve(support, 3, 5), separably
    impl->blur(false, impl->sup.p, 3.0, 5);
    NADIA_CUDA(cudaMemcpyAsync(impl->sup.p, impl->tmp2.p, impl->n * sizeof(float),
                               cudaMemcpyDeviceToDevice, impl->S.st));
    impl->q_valid = false;
    impl->S.sync();
}


void Fused32::upload_illumination()
{
    Impl &I = *impl;
    I.W.alloc(I.n);
    I.ill.alloc(I.n);
    I.put_panel(I.S.h_illum.data(), 2, I.W.p, false);
    I.h_slot.W = I.W.p;
    I.push_slot();
}

// FresnelCDI::set_experimental_parameters (FresnelCDI.c++:57-95): the phase
// factor of multiply_factors becomes tx[kx]*ty[ky] with the quadrant-swap
// sign folded in; the sample-plane illumination is computed once in FP64
void Fused32::set_fresnel_geometry(double factor)
{
    Impl &I = *impl;
    Solver &S = I.S;
    auto make = [&](int m, DevBuf<float2> &buf) {
        std::vector<float2> t(m);
        double mid = (m - 1) / 2.0;
        for (int k = 0; k < m; ++k) {
            int k_ = (int)(mid - fabs(mid - k));
            double a = mid - k_;
            double ph = -factor * a * a; // conj(coef) along this axis
            double sg = (k % 2) ? -1.0 : 1.0;
            t[k] = make_float2((float)(sg * cos(ph)), (float)(sg * sin(ph)));
        }
        buf.alloc(m);
        upload_now(buf.p, t.data(), m * sizeof(float2));
    };
    make(I.nx, I.tx);
    make(I.ny, I.ty);
    I.h_slot.tx = I.tx.p;
    I.h_slot.ty = I.ty.p;
    I.push_slot();
    // illumination at the sample plane: FresnelCDI::propagate_from_detector
    // (FresnelCDI.c++:238-243) of the white field, in FP64
    const int qy = I.ny / 2;
    double x_mid = (I.nx - 1) / 2.0, y_mid = (I.ny - 1) / 2.0;
    std::vector<double2> hc((size_t)(I.nx / 2) * qy);
    for (int i = 0; i < I.nx / 2; i++)
        for (int j = 0; j < qy; j++) {
            double phi = factor * ((x_mid - i) * (x_mid - i) + (y_mid - j) * (y_mid - j));
            hc[(size_t)i * qy + j] = make_double2(cos(phi), sin(phi));
        }
    DevBuf<double2> coef(hc.size()), c(I.n);
    plain::Fft2d fft;
    fft.init(I.nx, I.ny);
    upload_now(coef.p, hc.data(), coef.bytes());
    upload_now(c.p, S.h_illum.data(), c.bytes());
    plain::multiply_factors(c.p, coef.p, I.nx, I.ny, +1, S.st);
    fft.exec(c.p, false, S.st);
    plain::invert(c.p, I.nx, I.ny, true, S.st);
    std::vector<double> h(2 * I.n);
    NADIA_CUDA(cudaMemcpyAsync(h.data(), c.p, c.bytes(), cudaMemcpyDeviceToHost, S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
    I.put_panel(h.data(), 2, I.ill.p, false);
}

// FresnelCDI_WF's coefficient (FresnelCDI_WF.c++:31-79): sin(phi) - i cos(phi)
// = -i e^{i phi} with phi = (rho_x^2 + rho_y^2)(1/z12 + 1/z23) pi / lambda,
// rho = scaling * (mid - k_) and k_ the reference's folded index; kept as
// b(k) = e^{i phi(k)} / m per axis of length m (the constant -i and the
// factor's 1/sqrt(N) with invert's 1/sqrt(N) are folded, see fused32_wf.cuh)
void Fused32::set_wf_geometry()
{
    Impl &I = *impl;
    Solver &S = I.S;
    auto make = [&](int m, double scaling, DevBuf<float2> &buf) {
        std::vector<float2> t(m);
        const double mid = (m - 1) / 2.0;
        for (int k = 0; k < m; ++k) {
            const int k_ = (int)(mid - fabs(mid - k));
            const double a = scaling * (mid - k_);
            const double r2 = a * a;
            const double ph = (r2 / S.z12 + r2 / S.z23) * (M_PI / S.wavelength);
            t[k] = make_float2((float)(cos(ph) / m), (float)(sin(ph) / m));
        }
        buf.alloc(m);
        upload_now(buf.p, t.data(), m * sizeof(float2));
    };
    make(I.nx, S.wavelength * S.z23 / (S.pixel * I.nx), I.tx);
    make(I.ny, S.wavelength * S.z23 / (S.pixel * I.ny), I.ty);
    I.h_slot.tx = I.tx.p;
    I.h_slot.ty = I.ty.p;
    I.push_slot();
}

void Fused32::scale_illumination(double f)
{
    Impl &I = *impl;
    k_scale32<<<grid1(I.n), 256, 0, I.S.st>>>(I.W.p, (float)f, I.n);
    k_scale32<<<grid1(I.n), 256, 0, I.S.st>>>(I.ill.p, (float)f, I.n);
    I.S.sync();
}

void Fused32::fresnel_initialise(const double *t)
{
    fresnel_set_transmission(t);
    Impl &I = *impl;
    k_support_apply<<<grid1(I.n), 256, 0, I.S.st>>>(I.x.p, I.sup.p, I.n);
    I.S.sync();
}

void Fused32::fresnel_set_transmission(const double *t)
{
    Impl &I = *impl;
    // the work array holds T for the moment; the next iteration rebuilds it
    I.p_valid = false;
    I.put_panel(t, 2, I.P.p, false);
    k_fresnel_set_t<<<grid1(I.n), 256, 0, I.S.st>>>(I.P.p, I.ill.p, I.x.p, I.nx, I.ny);
    I.S.sync();
}

void Fused32::set_constraint(bool on, bool unity, bool flip, int flip_sign, int nregions,
                             const int *map, const double *prm)
{
    Impl &I = *impl;
    NADIA_REQUIRE(!on || I.S.kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                  "a transmission constraint on PolyCDI runs in the FP64 form");
    NADIA_REQUIRE(nregions >= 0 && nregions <= kTcMaxRegions && (nregions == 0 || (map && prm)),
                  NADIA_ERR_INVALID, "between 0 and 16 complex-constraint regions");
    NADIA_CUDA(cudaStreamSynchronize(I.S.st)); // buffers of an earlier constraint may be replaced
    const int R = on ? nregions : 0;
    if (R > 0) {
        // the region map in the panel layout, the parameters as floats
        std::vector<int> pm(I.n);
        for (int kx = 0; kx < I.nx; ++kx)
            for (int ky = 0; ky < I.ny; ++ky)
                pm[panel_index_dev(kx, ky, I.nx)] = map[(size_t)kx * I.ny + ky];
        std::vector<float> pf(4 * (size_t)R);
        for (size_t k = 0; k < pf.size(); ++k) pf[k] = (float)prm[k];
        I.tc_region.alloc(I.n);
        I.tc_par.alloc(pf.size());
        I.tc_cm.alloc(3 * (size_t)R);
        I.tc_part.alloc(2 * (size_t)kTcBlocks * R);
        if (!I.Y) I.Y.alloc(I.n);
        upload_now(I.tc_region.p, pm.data(), I.n * sizeof(int));
        upload_now(I.tc_par.p, pf.data(), pf.size() * sizeof(float));
    }
    I.h_slot.tc_R = R;
    I.h_slot.tc_region = R > 0 ? I.tc_region.p : nullptr;
    I.h_slot.tc_par = R > 0 ? I.tc_par.p : nullptr;
    I.h_slot.tc_cm = R > 0 ? I.tc_cm.p : nullptr;
    I.h_slot.tc_part = R > 0 ? I.tc_part.p : nullptr;
    I.h_slot.Y = R > 0 ? I.Y.p : nullptr;
    I.h_slot.tc_on = on ? 1 : 0;
    I.h_slot.tc_unity = on && unity ? 1 : 0;
    I.h_slot.tc_flip = on && flip ? 1 : 0;
    I.h_slot.tc_sign = flip_sign > 0 ? 1.f : -1.f;
    I.h_slot.tc_ill = on && I.S.kind == NADIA_FRESNEL ? I.ill.p : nullptr;
    if (I.S.kind != NADIA_POLY) {
        NADIA_CUDA(cudaStreamSynchronize(I.S.st));
        I.choice = &choose(I.nx, I.ny, I.S.kind == NADIA_FRESNEL, 1, on);
        if (I.graph_exec) { // captured with the other variants
            cudaGraphExecDestroy(I.graph_exec);
            I.graph_exec = nullptr;
        }
        I.use_choice(I.choice);
    }
    I.push_slot();
}

bool Fused32::constrained() const { return impl->h_slot.tc_on != 0; }

// TransmissionConstraint::apply_constraint on a whole array (FresnelCDI's
// transmission function when it is read, FresnelCDI.c++:352-353): region
// sums and c_mean as field 2, then the update of every pixel
void Fused32::Impl::constrain_array(float2 *t)
{
    if (h_slot.tc_R > 0) {
        k_tc32_sums<<<kTcBlocks, kTcThreads, 0, S.st>>>(slot.p, 2, t, n);
        k_tc32_cmean<<<h_slot.tc_R, kTcThreads, 0, S.st>>>(slot.p, 2, kTcBlocks);
        k_tc32_apply_array<<<grid1(n), 256, 0, S.st>>>(t, n, slot.p);
    } else {
        k_tc_pixels<<<grid1(n), 256, 0, S.st>>>(t, n, slot.p);
    }
}

void Fused32::transmission_to_device(double2 *dst)
{
    Impl &I = *impl;
    const float2 *src = I.x.p;
    if (I.S.kind == NADIA_FRESNEL) {
        I.p_valid = false; // T is formed in the work array
        I.push_slot();
        k_fresnel_get_t<<<grid1(I.n), 256, 0, I.S.st>>>(I.x.p, I.ill.p, I.P.p, I.n);
        if (I.h_slot.tc_on) I.constrain_array(I.P.p);
        src = I.P.p;
    }
    k_panel_widen<<<grid1(I.n), 256, 0, I.S.st>>>(src, dst, I.nx, I.ny);
    NADIA_CUDA(cudaGetLastError());
}

void Fused32::transmission_from_device(const double2 *src)
{
    Impl &I = *impl;
    I.p_valid = false;
    if (I.S.kind == NADIA_FRESNEL) {
        k_panel_narrow<<<grid1(I.n), 256, 0, I.S.st>>>(src, I.P.p, I.nx, I.ny);
        k_fresnel_set_t<<<grid1(I.n), 256, 0, I.S.st>>>(I.P.p, I.ill.p, I.x.p, I.nx, I.ny);
    } else {
        k_panel_narrow<<<grid1(I.n), 256, 0, I.S.st>>>(src, I.x.p, I.nx, I.ny);
    }
    NADIA_CUDA(cudaGetLastError());
}

void Fused32::fresnel_get_transmission(double *t)
{
    Impl &I = *impl;
    I.p_valid = false; // T is formed in the work array
    I.push_slot();
    k_fresnel_get_t<<<grid1(I.n), 256, 0, I.S.st>>>(I.x.p, I.ill.p, I.P.p, I.n);
    if (I.h_slot.tc_on) I.constrain_array(I.P.p);
    I.get_panel(I.P.p, 2, t);
}

void Fused32::get_illumination_at_sample(double *h) { impl->get_panel(impl->ill.p, 2, h); }

void Fused32::set_x(const double *h)
{
    impl->put_panel(h, 2, impl->x.p, false);
    impl->p_valid = false;
    impl->flush_intensity();
}

void Fused32::get_x(double *h) { impl->get_panel(impl->x.p, 2, h); }

void Fused32::set_x_f32(const float *h)
{
    impl->put_panel_f(h, 2, impl->x.p, false);
    impl->p_valid = false;
    impl->flush_intensity();
}

void Fused32::get_x_f32(float *h) { impl->get_panel_f(impl->x.p, 2, h); }

// n-best copies are kept in the natural layout so get_best_result can
// download them directly
__global__ void k_unpanel(const float2 *src, float2 *dst, int nx, int ny)
{
    const size_t n = (size_t)nx * ny;
    for (size_t a = blockIdx.x * (size_t)blockDim.x + threadIdx.x; a < n;
         a += (size_t)gridDim.x * blockDim.x) {
        const int xx = (int)(a / ny), yy = (int)(a % ny);
        dst[a] = src[f32::panel_index_dev(xx, yy, nx)];
    }
}

void Fused32::copy_x_to(float2 *dst)
{
    Impl &I = *impl;
    k_unpanel<<<grid1(I.n), 256, 0, I.S.st>>>(I.x.p, dst, I.nx, I.ny);
}

void Fused32::Impl::check_algorithm() const
{
    if (!pfs_mode()) return;
    NADIA_REQUIRE(S.kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                  "PolyCDI algorithms with a PfPs term (DM, custom m1/m5/m6/m7) run in the FP64 form");
    NADIA_REQUIRE(!h_slot.tc_on, NADIA_ERR_UNSUPPORTED,
                  "algorithms with a PfPs term run with a transmission constraint in the FP64 form");
}

void Fused32::Impl::prime(cudaStream_t st)
{
    const Slot *const *sl = slot_ptr.p;
    if (S.kind == NADIA_FRESNEL_WF) {
        wfr->wf_row(kRowPrime, sl, 1, nx, ny, twy, st);
    } else if (S.kind == NADIA_POLY) {
        prow->row(kRowPrime, sl, 1, nx / prow->L, st, twy);
    } else if (pfs_mode()) {
        pfs_choice->row->row(kRowPrimePfs, sl, 1, nx, ny, twy, st);
        q_valid = true;
    } else {
        choice->row->row(kRowPrime, sl, 1, nx, ny, twy, st);
    }
    g_launches += 1;
    p_valid = true;
}

// FresnelCDI_WF::iterate (FresnelCDI_WF.c++:122-182): the column pass, the row
// pass, and the error metric of the row pass's modulus
void Fused32::Impl::launch_iteration_wf(cudaStream_t st)
{
    const Slot *const *sl = slot_ptr.p;
    wfc->wf_col(sl, 1, nx, ny, twx, st);
    wfr->wf_row(kRowFull, sl, 1, nx, ny, twy, st);
    k_wf_finish<256><<<1, 256, 0, st>>>(sl);
}

void Fused32::Impl::launch_iteration(cudaStream_t st)
{
    const Slot *const *sl = slot_ptr.p;
    if (h_slot.tc_R > 0) {
        // complex-constraint regions: the row pass in two halves around the
        // region sums of both projected fields (Ps x is summed for ER too,
        // so one captured graph serves every algorithm)
        choice->col->col(S.kind == NADIA_FRESNEL, sl, 1, nx, ny, twx, st);
        choice->row->tc_row(1, sl, 1, nx, ny, twy, st);
        for (int field = 0; field < 2; ++field) {
            k_tc32_sums<<<kTcBlocks, kTcThreads, 0, st>>>(slot.p, field, nullptr, n);
            k_tc32_cmean<<<h_slot.tc_R, kTcThreads, 0, st>>>(slot.p, field, kTcBlocks);
        }
        choice->row->tc_row(2, sl, 1, nx, ny, twy, st);
        return;
    }
    choice->col->col(S.kind == NADIA_FRESNEL, sl, 1, nx, ny, twx, st);
    choice->row->row(kRowFull, sl, 1, nx, ny, twy, st);
}

// BaseCDI::iterate's generic path with a PfPs term (BaseCDI.c++:313-383):
// the column pass projects both fields (x's rows in P, Ps x's rows in Q),
// then one row pass forms the combine and both fields' rows for the next
// iteration
void Fused32::Impl::launch_iteration_pfs(cudaStream_t st)
{
    const bool fr = S.kind == NADIA_FRESNEL;
    pfs_choice->col->col(fr, qslot_ptr.p, 1, nx, ny, twx, st);
    pfs_choice->col->col(fr, slot_ptr.p, 1, nx, ny, twx, st);
    pfs_choice->row->row(kRowPfs, slot_ptr.p, 1, nx, ny, twy, st);
}

void Fused32::iterate(int count)
{
    Impl &I = *impl;
    if (I.S.kind == NADIA_POLY) {
        iterate_poly(count);
        return;
    }
    const bool wf = I.S.kind == NADIA_FRESNEL_WF;
    I.check_algorithm();
    const bool pfs = I.pfs_mode();
    if (wf) {
        I.use_ncol(I.nx / I.wfr->L);
    } else if (pfs) {
        I.prepare_pfs();
        I.use_choice(I.pfs_choice);
    } else {
        I.use_choice(I.choice);
        I.q_valid = false; // Q is not carried by these iterations
    }
    I.push_slot();
    cudaStream_t st = I.S.st;
    if (!I.p_valid || (pfs && !I.q_valid)) I.prime(st);
    const int per_iter = (pfs || wf) ? 3 : (I.h_slot.tc_R > 0 ? 7 : 2);
    auto one = [&] {
        if (wf)
            I.launch_iteration_wf(st);
        else if (pfs)
            I.launch_iteration_pfs(st);
        else
            I.launch_iteration(st);
    };
    cudaGraphExec_t &exec = pfs ? I.graph_pfs : I.graph_exec;
    // replay a captured graph of kGraphIters iterations, then the remainder
    const int G = Impl::kGraphIters;
    int left = count;
    if (left >= G) {
        if (!exec) {
            cudaGraph_t g = nullptr;
            NADIA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            for (int i = 0; i < G; ++i) one();
            NADIA_CUDA(cudaStreamEndCapture(st, &g));
            NADIA_CUDA(cudaGraphInstantiate(&exec, g, 0));
            cudaGraphDestroy(g);
        }
        while (left >= G) {
            NADIA_CUDA(cudaGraphLaunch(exec, st));
            g_launches += per_iter * G;
            left -= G;
        }
    }
    for (; left > 0; --left) {
        one();
        g_launches += per_iter;
    }
    NADIA_CUDA(cudaGetLastError());
    I.S.iters += count;
}

// Blur into tmp2 and leave the maximum of the blurred values at
// maxpart[blur_blocks()]: one tiled kernel for the 4-pixel cut-off of
// apply_shrinkwrap, the two separable passes for wider ones (set_support's soften).
int Fused32::Impl::blur_blocks() const
{
    return ((nx + kSwTile - 1) / kSwTile) * ((ny + kSwTile - 1) / kSwTile);
}

void Fused32::Impl::blur(bool cplx, const void *in, double gauss_width, int cut)
{
    Gauss g{};
    g.cut = cut;
    for (int d = 0; d <= cut; ++d) g.w[d] = (float)exp(-(double)(d * d) / (2.0 * gauss_width * gauss_width));
    const int nb = blur_blocks();
    if (!tmp2) {
        tmp1.alloc(n);
        tmp2.alloc(n);
        maxpart.alloc(std::max(nb, (int)kMaxBlocks) + 2);
    }
    if (cut <= 4) {
        dim3 grid((ny + kSwTile - 1) / kSwTile, (nx + kSwTile - 1) / kSwTile),
            block(32, kSwThreads / 32);
        if (cplx && cut == 4)
            k_blur_tiles<true, 4><<<grid, block, 0, S.st>>>(in, tmp2.p, nx, ny, g, maxpart.p);
        else if (cplx)
            k_blur_tiles<true, 0><<<grid, block, 0, S.st>>>(in, tmp2.p, nx, ny, g, maxpart.p);
        else
            k_blur_tiles<false, 0><<<grid, block, 0, S.st>>>(in, tmp2.p, nx, ny, g, maxpart.p);
        k_max_final<<<1, 256, 0, S.st>>>(maxpart.p, nb);
        g_launches += 2;
        return;
    }
    const int gb = kMaxBlocks;
    if (cplx)
        k_blur_y<true><<<gb, 256, 0, S.st>>>(in, tmp1.p, nx, ny, g);
    else
        k_blur_y<false><<<gb, 256, 0, S.st>>>(in, tmp1.p, nx, ny, g);
    k_blur_x<<<gb, 256, 0, S.st>>>(tmp1.p, tmp2.p, nx, ny, g, maxpart.p);
    k_max_final<<<1, 256, 0, S.st>>>(maxpart.p, gb);
    // the maximum sits at maxpart[gb]; move it to where callers read it
    if (nb != gb)
        NADIA_CUDA(cudaMemcpyAsync(maxpart.p + nb, maxpart.p + gb, sizeof(float),
                                   cudaMemcpyDeviceToDevice, S.st));
    g_launches += 3;
}

// BaseCDI::apply_shrinkwrap (BaseCDI.c++:416-429): |x| blurred by the
// truncated Gaussian (exactly separable: square window, per-axis edge skip),
// thresholded at t*max, then divided by its own maximum
void Fused32::shrinkwrap(double gauss_width, double threshold)
{
    Impl &I = *impl;
    I.q_valid = false; // the support changes; Q holds the rows of Ps x
    I.blur(true, I.x.p, gauss_width, 4);
    const int nb = I.blur_blocks(), gb = Impl::kMaxBlocks;
    if (I.nx == I.ny) {
        k_threshold_divide_square<<<gb, 256, 0, I.S.st>>>(I.tmp2.p, I.sup.p, I.n, threshold,
                                                          I.maxpart.p + nb);
        g_launches += 1;
    } else {
        k_threshold<<<gb, 256, 0, I.S.st>>>(I.tmp2.p, I.nx, I.ny, threshold, I.maxpart.p + nb);
        k_max<<<gb, 256, 0, I.S.st>>>(I.tmp2.p, I.n, I.maxpart.p);
        k_max_final<<<1, 256, 0, I.S.st>>>(I.maxpart.p, gb);
        k_divide<<<gb, 256, 0, I.S.st>>>(I.tmp2.p, I.sup.p, I.n, I.maxpart.p + gb);
        g_launches += 4;
    }
    NADIA_CUDA(cudaGetLastError());
}

void Fused32::check_device_flag()
{
    int fl = 0;
    NADIA_CUDA(cudaMemcpyAsync(&fl, impl->flag.p, sizeof(int), cudaMemcpyDeviceToHost, impl->S.st));
    NADIA_CUDA(cudaStreamSynchronize(impl->S.st));
    if (fl) {
        NADIA_CUDA(cudaMemsetAsync(impl->flag.p, 0, sizeof(int), impl->S.st));
        throw Error(NADIA_ERR_CUDA, "a device-side wait timed out; the estimate is not valid");
    }
}

void Fused32::get_support(double *h) { impl->get_panel(impl->sup.p, 1, h); }

void Fused32::single_op(int, double *)
{
    throw Error(NADIA_ERR_UNSUPPORTED, "single operators run in the FP64 form");
}

void Fused32::autocorrelation(double *)
{
    throw Error(NADIA_ERR_UNSUPPORTED, "the autocorrelation runs in the FP64 form");
}

} // namespace nadia
