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
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "fft32.cuh"
#include "fused32_impl.h"
#include "solver.h"

namespace nadia {
namespace f32 {

// ------------------------------------------------------------ tile configs

// Column and row tile shapes per transform length.  K*L >= 16 keeps the row
// pass's panel segments at 128 bytes or more.
template <int N> struct Shape;
template <> struct Shape<256> {
    using Col = TileCfg<256, 256, 16, kColMap, Radices<16, 16>>;
    using Row = TileCfg<256, 256, 16, kRowMap, Radices<16, 16>>;
};
template <> struct Shape<512> {
    using Col = TileCfg<512, 256, 8, kColMap, Radices<16, 8, 4>>;
    using Row = TileCfg<512, 256, 8, kRowMap, Radices<16, 8, 4>>;
};
template <> struct Shape<768> {
    using Col = TileCfg<768, 256, 8, kColMap, Radices<8, 8, 4, 3>>;
    using Row = TileCfg<768, 256, 8, kRowMap, Radices<8, 8, 4, 3>>;
};
template <> struct Shape<1024> {
    using Col = TileCfg<1024, 256, 4, kColMap, Radices<16, 16, 4>>;
    using Row = TileCfg<1024, 256, 4, kRowMap, Radices<16, 16, 4>>;
};
template <> struct Shape<1536> {
    using Col = TileCfg<1536, 256, 4, kColMap, Radices<8, 8, 8, 3>>;
    using Row = TileCfg<1536, 256, 4, kRowMap, Radices<8, 8, 8, 3>>;
};
template <> struct Shape<2048> {
    using Col = TileCfg<2048, 512, 4, kColMap, Radices<16, 16, 8>>;
    using Row = TileCfg<2048, 512, 4, kRowMap, Radices<16, 16, 8>>;
};
template <> struct Shape<4096> {
    using Col = TileCfg<4096, 1024, 4, kColMap, Radices<16, 16, 16>>;
    using Row = TileCfg<4096, 1024, 4, kRowMap, Radices<16, 16, 16>>;
};

__device__ __forceinline__ size_t paddr(int i, int p, int nx)
{
    return ((size_t)(p / kPanel) * nx + i) * kPanel + (p % kPanel);
}

__device__ __forceinline__ float support_factor(float s)
{
    return s == 0.f ? 0.f : (s < 1.f ? s : 1.f);
}

// FP64 block sum; result valid in thread 0
template <int NT>
__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[NT / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < NT / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    }
    return t;
}

// -------------------------------------------------------------- column pass

template <class C, bool FRESNEL>
__global__ void __launch_bounds__(C::NT) k_col(const Slot *const *slots, int nx, int ny,
                                               const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    const float *__restrict__ mI = S.mI;
    const float s0 = S.s0;
    const int c0 = blockIdx.x * (C::L / kPanel);
    float2 v[C::E];

    for_each_slot<C, true, true>([&](int e, int s, int pos) {
        v[e] = P[paddr(pos, c0 * kPanel + s, nx)];
    });
    transform<C, true>(v, sm, tw);

    double diff = 0.0;
    for_each_slot<C, true, false>([&](int e, int s, int kx) {
        const int ky = c0 * kPanel + s;
        const size_t a = paddr(kx, ky, nx);
        const float m = __ldg(&mI[a]);
        float2 X = v[e];
        if (!FRESNEL) {
            if (!(m < 0.f)) {
                const float a2 = X.x * X.x + X.y * X.y;
                if (a2 > 0.f) {
                    const float inv = rsqrtf(a2);
                    const double d = (double)(a2 * inv * s0) - (double)m;
                    diff += d * d;
                    X = cscale(X, m * s0 * inv);
                } else {
                    diff += (double)m * (double)m;
                    X = make_float2(m * s0, 0.f);
                }
            } else {
                X = cscale(X, s0 * s0);
            }
        } else {
            const float2 cf = cmul(__ldg(&S.tx[kx]), __ldg(&S.ty[ky]));
            const float2 w = S.W[a];
            float2 u = cadd(cscale(cmul(cf, X), s0), w);
            if (!(m < 0.f)) {
                const float a2 = u.x * u.x + u.y * u.y;
                if (a2 > 0.f) {
                    const float inv = rsqrtf(a2);
                    const double d = (double)(a2 * inv) - (double)m;
                    diff += d * d;
                    u = cscale(u, m * inv);
                } else {
                    diff += (double)m * (double)m;
                    u = make_float2(m, 0.f);
                }
            }
            X = cscale(cmulc(csub(u, w), cf), s0);
        }
        v[e] = X;
    });
    const double tot = block_sum<C::NT>(diff);
    if (threadIdx.x == 0) S.partials[blockIdx.x] = tot;

    transform<C, false>(v, sm, tw);
    for_each_slot<C, false, false>([&](int e, int s, int pos) {
        P[paddr(pos, c0 * kPanel + s, nx)] = v[e];
    });
}

// ----------------------------------------------------------------- row pass

enum { kRowFull = 0, kRowPrime = 1 };

template <class C, int MODE>
__global__ void __launch_bounds__(C::NT) k_row(const Slot *const *slots, int nx, int ny,
                                               const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    float2 *__restrict__ x = S.x;
    const int i0 = blockIdx.x * C::L;
    float2 v[C::E];

    if (MODE == kRowFull) {
        // finish the error metric of the column pass that just ran
        if (blockIdx.x == 0 && S.project) {
            double t = 0.0;
            for (int b = threadIdx.x; b < S.ncol; b += C::NT) t += S.partials[b];
            t = block_sum<C::NT>(t);
            if (threadIdx.x == 0) {
                const double e = t * S.inv_norm2;
                long long it = *S.iter;
                *S.err = e;
                S.ring[it % S.ring_len] = e;
                *S.iter = it + 1;
            }
        } else if (blockIdx.x == 0 && threadIdx.x == 0) {
            long long it = *S.iter;
            S.ring[it % S.ring_len] = *S.err;
            *S.iter = it + 1;
        }
        for_each_slot<C, false, true>([&](int e, int s, int pos) {
            v[e] = P[paddr(i0 + s, pos, nx)];
        });
        transform<C, false>(v, sm, tw);
        const float *__restrict__ sup = S.sup;
        const float wid = S.w_id, wpf = S.w_pf, wps = S.w_ps, wpsf = S.w_psf;
        const bool er = S.er;
        for_each_slot<C, false, false>([&](int e, int s, int pos) {
            const size_t a = paddr(i0 + s, pos, nx);
            const float f = support_factor(__ldg(&sup[a]));
            const float2 y = v[e];
            float2 xn;
            if (er) {
                xn = cscale(y, f);
            } else {
                const float2 xk = x[a];
                xn = make_float2(wid * xk.x + wpf * y.x + wps * (f * xk.x) + wpsf * (f * y.x),
                                 wid * xk.y + wpf * y.y + wps * (f * xk.y) + wpsf * (f * y.y));
            }
            x[a] = xn;
            v[e] = xn;
        });
    } else {
        for_each_slot<C, true, true>([&](int e, int s, int pos) {
            v[e] = x[paddr(i0 + s, pos, nx)];
        });
    }
    transform<C, true>(v, sm, tw);
    for_each_slot<C, true, false>([&](int e, int s, int pos) {
        P[paddr(i0 + s, pos, nx)] = v[e];
    });
}

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

// ------------------------------------------------------------ dispatch

template <int N>
struct Kern {
    using Col = typename Shape<N>::Col;
    using Row = typename Shape<N>::Row;
};

template <class C>
size_t smem_bytes() { return (size_t)C::smem_words() * sizeof(float2); }

template <class C, class K>
void set_smem(K kernel)
{
    NADIA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_bytes<C>()));
}

template <int N>
void col_prepare_impl()
{
    using C = typename Kern<N>::Col;
    static std::once_flag once;
    std::call_once(once, [] {
        set_smem<C>(k_col<C, false>);
        set_smem<C>(k_col<C, true>);
    });
}

template <int N>
void row_prepare_impl()
{
    using C = typename Kern<N>::Row;
    static std::once_flag once;
    std::call_once(once, [] {
        set_smem<C>(k_row<C, kRowFull>);
        set_smem<C>(k_row<C, kRowPrime>);
    });
}

template <int N>
bool col_launch_impl(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                     const float2 *tw, cudaStream_t st)
{
    using C = typename Kern<N>::Col;
    dim3 grid(ny / C::L, nslots);
    if (fresnel)
        k_col<C, true><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    else
        k_col<C, false><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    return true;
}

template <int N>
bool row_launch_impl(int mode, const Slot *const *slots, int nslots, int nx, int ny,
                     const float2 *tw, cudaStream_t st)
{
    using C = typename Kern<N>::Row;
    dim3 grid(nx / C::L, nslots);
    if (mode == kRowFull)
        k_row<C, kRowFull><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    else
        k_row<C, kRowPrime><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    return true;
}

#define NADIA_SIZES(X) X(256) X(512) X(768) X(1024) X(1536) X(2048) X(4096)

bool supported(int n)
{
#define X(N) if (n == N) return true;
    NADIA_SIZES(X)
#undef X
    return false;
}

int col_tile(int n)
{
#define X(N) if (n == N) return Kern<N>::Col::L;
    NADIA_SIZES(X)
#undef X
    return 0;
}

int row_tile(int n)
{
#define X(N) if (n == N) return Kern<N>::Row::L;
    NADIA_SIZES(X)
#undef X
    return 0;
}

// Set the kernels' shared-memory limits (must happen before any stream capture).
void prepare(int nx, int ny)
{
#define X(N) if (nx == N) col_prepare_impl<N>();
    NADIA_SIZES(X)
#undef X
#define X(N) if (ny == N) row_prepare_impl<N>();
    NADIA_SIZES(X)
#undef X
}

void col_launch(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                const float2 *tw, cudaStream_t st)
{
#define X(N) if (nx == N) { col_launch_impl<N>(fresnel, slots, nslots, nx, ny, tw, st); return; }
    NADIA_SIZES(X)
#undef X
    throw Error(NADIA_ERR_UNSUPPORTED, "FP32 transform length not available");
}

void row_launch(int mode, const Slot *const *slots, int nslots, int nx, int ny, const float2 *tw,
                cudaStream_t st)
{
#define X(N) if (ny == N) { row_launch_impl<N>(mode, slots, nslots, nx, ny, tw, st); return; }
    NADIA_SIZES(X)
#undef X
    throw Error(NADIA_ERR_UNSUPPORTED, "FP32 transform length not available");
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

} // namespace f32

// =================================================================== host

using namespace f32;

namespace {
inline size_t panel_index(int x, int y, int nx)
{
    return ((size_t)(y / kPanel) * nx + x) * kPanel + (y % kPanel);
}
} // namespace

Fused32::Fused32(Solver &s) : impl(new Impl(s)) {}
Fused32::~Fused32() { delete impl; }

Fused32::Impl::Impl(Solver &s) : S(s)
{
    nx = s.nx;
    ny = s.ny;
    n = s.n;
    NADIA_REQUIRE(supported(nx) && supported(ny), NADIA_ERR_UNSUPPORTED,
                  "the FP32 form supports grid sizes 256, 512, 768, 1024, 1536, 2048 and 4096 "
                  "per axis; use NADIA_FP64 for other sizes");
    NADIA_REQUIRE(s.kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                  "PolyCDI runs in the FP64 form");
    NADIA_REQUIRE(ny % col_tile(nx) == 0 && nx % row_tile(ny) == 0, NADIA_ERR_UNSUPPORTED,
                  "grid shape does not divide into the FP32 tiles");
    prepare(nx, ny);
    P.alloc(n);
    x.alloc(n);
    sup.alloc(n);
    mI.alloc(n);
    ncol = ny / col_tile(nx);
    partials.alloc(ncol);
    iter.alloc(1);
    slot.alloc(1);
    slot_ptr.alloc(1);
    cudaStream_t st = s.st;
    NADIA_CUDA(cudaMemsetAsync(P.p, 0, P.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(x.p, 0, x.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(sup.p, 0, sup.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(mI.p, 0, mI.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(partials.p, 0, partials.bytes(), st));
    NADIA_CUDA(cudaMemsetAsync(iter.p, 0, iter.bytes(), st));
    twx = twiddle_table(nx);
    twy = twiddle_table(ny);
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
    Slot *sp = slot.p;
    NADIA_CUDA(cudaMemcpyAsync(slot_ptr.p, &sp, sizeof(Slot *), cudaMemcpyHostToDevice, st));
    push_slot();
}

Fused32::Impl::~Impl()
{
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
}

void Fused32::Impl::push_slot()
{
    const double *w = S.w;
    h_slot.er = (S.algorithm == NADIA_ER);
    h_slot.w_id = (float)(1 + w[PI]);
    h_slot.w_pf = (float)w[PF];
    h_slot.w_ps = (float)w[PS];
    h_slot.w_psf = (float)w[PSF];
    h_slot.project = h_slot.er || w[PF] != 0 || w[PSF] != 0;
    NADIA_CUDA(cudaMemcpyAsync(slot.p, &h_slot, sizeof(Slot), cudaMemcpyHostToDevice, S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
}

void Fused32::Impl::to_panel(const double *h, size_t stride, std::vector<float> &out) const
{
    out.resize(n * stride);
    for (int xx = 0; xx < nx; ++xx)
        for (int yy = 0; yy < ny; ++yy) {
            size_t a = panel_index(xx, yy, nx), b = (size_t)xx * ny + yy;
            for (size_t c = 0; c < stride; ++c) out[a * stride + c] = (float)h[b * stride + c];
        }
}

void Fused32::Impl::from_panel(const std::vector<float> &in, size_t stride, double *h) const
{
    for (int xx = 0; xx < nx; ++xx)
        for (int yy = 0; yy < ny; ++yy) {
            size_t a = panel_index(xx, yy, nx), b = (size_t)xx * ny + yy;
            for (size_t c = 0; c < stride; ++c) h[b * stride + c] = in[a * stride + c];
        }
}

void Fused32::Impl::upload(void *dst, const std::vector<float> &v)
{
    NADIA_CUDA(cudaMemcpyAsync(dst, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice,
                               S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
}

void Fused32::Impl::download(std::vector<float> &v, const void *src, size_t count)
{
    v.resize(count);
    NADIA_CUDA(cudaMemcpyAsync(v.data(), src, count * sizeof(float), cudaMemcpyDeviceToHost, S.st));
    NADIA_CUDA(cudaStreamSynchronize(S.st));
}

// sqrt(I) in transform order with the unmeasured pixels marked -1; the
// normalisation sum of BaseCDI::scale_intensity over the measured pixels
void Fused32::Impl::upload_intensity()
{
    std::vector<float> m(n);
    double norm2 = 0;
    const bool planar = S.kind == NADIA_PLANAR;
    for (int kx = 0; kx < nx; ++kx)
        for (int ky = 0; ky < ny; ++ky) {
            int dx = planar ? (kx + nx / 2) % nx : kx, dy = planar ? (ky + ny / 2) % ny : ky;
            size_t d = (size_t)dx * ny + dy;
            bool measured = !S.has_beam_stop || h_bs[d] > 0;
            float v = (float)S.h_isqrt[d];
            if (measured) norm2 += (double)v * (double)v;
            m[panel_index(kx, ky, nx)] = measured ? v : -1.f;
        }
    upload(mI.p, m);
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
    std::vector<float> f;
    impl->to_panel(h, 1, f);
    impl->upload(impl->sup.p, f);
}

void Fused32::soften_support()
{
    // BaseCDI::set_support's convolve(support, 3, 5), separably
    impl->blur(false, impl->sup.p, 3.0, 5);
    NADIA_CUDA(cudaMemcpyAsync(impl->sup.p, impl->tmp2.p, impl->n * sizeof(float),
                               cudaMemcpyDeviceToDevice, impl->S.st));
    impl->S.sync();
}

void Fused32::set_spectrum() { throw Error(NADIA_ERR_UNSUPPORTED, "PolyCDI runs in the FP64 form"); }

void Fused32::upload_illumination()
{
    Impl &I = *impl;
    I.W.alloc(I.n);
    I.ill.alloc(I.n);
    std::vector<float> f;
    I.to_panel(I.S.h_illum.data(), 2, f);
    I.upload(I.W.p, f);
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
    std::vector<float> f;
    I.to_panel(h.data(), 2, f);
    I.upload(I.ill.p, f);
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
    std::vector<float> f;
    I.to_panel(t, 2, f);
    DevBuf<float2> d(I.n);
    I.upload(d.p, f);
    k_fresnel_set_t<<<grid1(I.n), 256, 0, I.S.st>>>(d.p, I.ill.p, I.x.p, I.nx, I.ny);
    I.S.sync();
    I.p_valid = false;
}

void Fused32::fresnel_get_transmission(double *t)
{
    Impl &I = *impl;
    DevBuf<float2> d(I.n);
    k_fresnel_get_t<<<grid1(I.n), 256, 0, I.S.st>>>(I.x.p, I.ill.p, d.p, I.n);
    std::vector<float> f;
    I.download(f, d.p, 2 * I.n);
    I.from_panel(f, 2, t);
}

void Fused32::get_illumination_at_sample(double *h)
{
    std::vector<float> f;
    impl->download(f, impl->ill.p, 2 * impl->n);
    impl->from_panel(f, 2, h);
}

void Fused32::set_x(const double *h)
{
    std::vector<float> f;
    impl->to_panel(h, 2, f);
    impl->upload(impl->x.p, f);
    impl->p_valid = false;
}

void Fused32::get_x(double *h)
{
    std::vector<float> f;
    impl->download(f, impl->x.p, 2 * impl->n);
    impl->from_panel(f, 2, h);
}

void Fused32::set_x_f32(const float *h)
{
    Impl &I = *impl;
    std::vector<float> f(2 * I.n);
    for (int xx = 0; xx < I.nx; ++xx)
        for (int yy = 0; yy < I.ny; ++yy) {
            size_t a = panel_index(xx, yy, I.nx), b = (size_t)xx * I.ny + yy;
            f[2 * a] = h[2 * b];
            f[2 * a + 1] = h[2 * b + 1];
        }
    I.upload(I.x.p, f);
    I.p_valid = false;
}

void Fused32::get_x_f32(float *h)
{
    Impl &I = *impl;
    std::vector<float> f;
    I.download(f, I.x.p, 2 * I.n);
    for (int xx = 0; xx < I.nx; ++xx)
        for (int yy = 0; yy < I.ny; ++yy) {
            size_t a = panel_index(xx, yy, I.nx), b = (size_t)xx * I.ny + yy;
            h[2 * b] = f[2 * a];
            h[2 * b + 1] = f[2 * a + 1];
        }
}

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
    NADIA_REQUIRE(S.algorithm == NADIA_ER || S.w[PFS] == 0, NADIA_ERR_UNSUPPORTED,
                  "algorithms with a PfPs term (DM, custom m1/m5/m6/m7) run in the FP64 form");
}

void Fused32::Impl::prime(cudaStream_t st)
{
    const Slot *const *sl = slot_ptr.p;
    row_launch(kRowPrime, sl, 1, nx, ny, twy, st);
    p_valid = true;
}

void Fused32::Impl::launch_iteration(cudaStream_t st)
{
    const Slot *const *sl = slot_ptr.p;
    col_launch(S.kind == NADIA_FRESNEL, sl, 1, nx, ny, twx, st);
    row_launch(kRowFull, sl, 1, nx, ny, twy, st);
}

void Fused32::iterate(int count)
{
    Impl &I = *impl;
    I.check_algorithm();
    I.push_slot();
    cudaStream_t st = I.S.st;
    if (!I.p_valid) I.prime(st);
    // replay a captured graph of kGraphIters iterations, then the remainder
    const int G = Impl::kGraphIters;
    int left = count;
    if (left >= G) {
        if (!I.graph_exec) {
            cudaGraph_t g = nullptr;
            NADIA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            for (int i = 0; i < G; ++i) I.launch_iteration(st);
            NADIA_CUDA(cudaStreamEndCapture(st, &g));
            NADIA_CUDA(cudaGraphInstantiate(&I.graph_exec, g, 0));
            cudaGraphDestroy(g);
        }
        while (left >= G) {
            NADIA_CUDA(cudaGraphLaunch(I.graph_exec, st));
            left -= G;
        }
    }
    for (; left > 0; --left) I.launch_iteration(st);
    NADIA_CUDA(cudaGetLastError());
    I.S.iters += count;
}

void Fused32::Impl::blur(bool cplx, const void *in, double gauss_width, int cut)
{
    Gauss g{};
    g.cut = cut;
    for (int d = 0; d <= cut; ++d) g.w[d] = (float)exp(-(double)(d * d) / (2.0 * gauss_width * gauss_width));
    if (!tmp1) { tmp1.alloc(n); tmp2.alloc(n); maxpart.alloc(kMaxBlocks + 2); }
    const int gb = kMaxBlocks;
    if (cplx)
        k_blur_y<true><<<gb, 256, 0, S.st>>>(in, tmp1.p, nx, ny, g);
    else
        k_blur_y<false><<<gb, 256, 0, S.st>>>(in, tmp1.p, nx, ny, g);
    k_blur_x<<<gb, 256, 0, S.st>>>(tmp1.p, tmp2.p, nx, ny, g, maxpart.p);
    k_max_final<<<1, 256, 0, S.st>>>(maxpart.p, gb);
}

// BaseCDI::apply_shrinkwrap (BaseCDI.c++:416-429): |x| blurred by the
// truncated Gaussian (exactly separable: square window, per-axis edge skip),
// thresholded at t*max, then divided by its own maximum
void Fused32::shrinkwrap(double gauss_width, double threshold)
{
    Impl &I = *impl;
    I.blur(true, I.x.p, gauss_width, 4);
    const int gb = Impl::kMaxBlocks;
    k_threshold<<<gb, 256, 0, I.S.st>>>(I.tmp2.p, I.nx, I.ny, threshold, I.maxpart.p + gb);
    k_max<<<gb, 256, 0, I.S.st>>>(I.tmp2.p, I.n, I.maxpart.p);
    k_max_final<<<1, 256, 0, I.S.st>>>(I.maxpart.p, gb);
    k_divide<<<gb, 256, 0, I.S.st>>>(I.tmp2.p, I.sup.p, I.n, I.maxpart.p + gb);
    NADIA_CUDA(cudaGetLastError());
}

void Fused32::get_support(double *h)
{
    std::vector<float> f;
    impl->download(f, impl->sup.p, impl->n);
    impl->from_panel(f, 1, h);
}

void Fused32::single_op(int, double *)
{
    throw Error(NADIA_ERR_UNSUPPORTED, "single operators run in the FP64 form");
}

void Fused32::autocorrelation(double *)
{
    throw Error(NADIA_ERR_UNSUPPORTED, "the autocorrelation runs in the FP64 form");
}

} // namespace nadia
