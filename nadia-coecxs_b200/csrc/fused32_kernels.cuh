// fused32_kernels.cuh -- the column and row passes of the fused FP32
// iteration, templated on the tile shape (see fused32.cu for the design), and
// the glue that turns one tile shape into a launchable variant.
#pragma once

#include "fft32.cuh"
#include "fused32_impl.h"

namespace nadia {
namespace f32 {

__device__ __forceinline__ size_t paddr(int i, int p, int nx)
{
    return ((size_t)(p / kPanel) * nx + i) * kPanel + (p % kPanel);
}

__device__ __forceinline__ float support_factor(float s)
{
    return s == 0.f ? 0.f : (s < 1.f ? s : 1.f);
}

// 1/sqrt(a) for the magnitude ratios: PTX's approximate reciprocal square
// root (relative error below 2^-22.9) in its flush-to-zero form, on a raised
// to the smallest normal float, so no subnormal handling is emitted around
// it; a = 0 gives 2^63, finite, so a * rsqrt_normal(a) is 0.
__device__ __forceinline__ float rsqrt_normal(float a)
{
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(fmaxf(a, 1.17549435e-38f)));
    return r;
}

// Modulus projection of one transform value (BaseCDI::scale_intensity,
// BaseCDI.c++:163-189, with Complex_2D::set_mag, Complex_2D.h:205-215):
// u is the detector-plane value, m its sqrt(I) (-1 = unmeasured).  Returns
// the projected value and adds (|u| - m)^2 to diff for measured pixels.
// Written with selects rather than branches.
__device__ __forceinline__ float2 modulus(float2 u, float m, double &diff)
{
    const float a2 = u.x * u.x + u.y * u.y;
    const bool measured = !(m < 0.f);
    const bool zero = !(a2 > 0.f);
    const float inv = rsqrt_normal(a2);
    const float mag = a2 * inv;
    const float sc = measured ? m * inv : 1.f;
    float2 r = make_float2(u.x * sc, u.y * sc);
    if (measured && zero) r = make_float2(m, 0.f);
    const double d = (double)mag - (double)m;
    diff += measured ? d * d : 0.0;
    return r;
}

// The PlanarCDI column-pass projection of an unnormalised transform value X:
// Psi = s0 X goes through the modulus projection, and the value handed to
// the inverse transform is s0 times the projected Psi, that is X s0 m / |X|
// ((s0 m, 0) where X = 0); the 1/sqrt(N) factors are folded into the
// magnitude ratio; unmeasured pixels (m < 0) keep Psi, so they leave as
// s0^2 X.  Adds (|Psi| - m)^2 to diff for measured pixels (the difference
// formed in FP32, its square summed in FP64).
__device__ __forceinline__ float2 planar_modulus(float2 X, float m, float s0, double &diff)
{
    const float a2 = X.x * X.x + X.y * X.y;
    const bool measured = !(m < 0.f);
    const bool zero = !(a2 > 0.f);
    const float inv = rsqrt_normal(a2);
    const float sm = s0 * m;
    const float sc = measured ? sm * inv : s0 * s0; // unmeasured: Psi kept, s0 Psi = s0^2 X
    float2 r = make_float2(X.x * sc, X.y * sc);
    if (measured && zero) r = make_float2(sm, 0.f);
    const float mag = a2 * inv;
    const float d = measured ? fmaf(s0, mag, -m) : 0.f;
    diff = fma((double)d, (double)d, diff);
    return r;
}

// The combine of BaseCDI.c++:346-383 without a PfPs term, with the support
// factor f folded into two weights: x' = (1 + PI + PS f) x + (PF + PSF f) y
__device__ __forceinline__ float2 combine2(float2 xk, float2 y, float f, float wid, float wpf,
                                           float wps, float wpsf)
{
    const float a = fmaf(wps, f, wid), b = fmaf(wpsf, f, wpf);
    return make_float2(fmaf(a, xk.x, b * y.x), fmaf(a, xk.y, b * y.y));
}

// FP64 block sum; result valid in thread 0
// (NT that is not a multiple of 32: the last warp holds NT % 32 threads, a
// power of two, and sums over those lanes alone)
template <int NT>
__device__ __forceinline__ double block_sum(double v)
{
    constexpr int NW = (NT + 31) / 32, TAIL = NT % 32;
    static_assert(NT >= 32 && (TAIL & (TAIL - 1)) == 0, "last warp: a power of two of lanes");
    __shared__ double red[NW];
    if (TAIL == 0 || (int)(threadIdx.x >> 5) < NW - 1) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    } else {
#pragma unroll
        for (int off = TAIL / 2; off > 0; off >>= 1)
            v += __shfl_down_sync((1u << TAIL) - 1u, v, off);
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x < 32) {
        t = threadIdx.x < NW ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    }
    return t;
}

// FP64 block sum in the order of the persistent column pass (warp sums by
// shuffles, then warp 0's ... warp NT/32-1's added in turn); result valid in
// thread 0
template <int NT>
__device__ __forceinline__ double block_sum_seq(double v)
{
    __shared__ double red[NT / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
#pragma unroll
        for (int w = 0; w < NT / 32; ++w) t += red[w];
    return t;
}

// 16-byte asynchronous copies global -> shared (completion: cp_async_wait_all)
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}

// -------------------------------------------------------------- column pass

// STAGE: the tile's sqrt(I) (and, for FresnelCDI, white field) -- one
// contiguous run of N*L elements in the panel layout, like P's -- is copied
// into shared memory by cp.async when the tile starts, so those loads land
// during the forward transform instead of stalling the modulus after it.
template <class C, bool FRESNEL>
constexpr size_t col_stage_bytes()
{
    return (size_t)C::N * C::L * (FRESNEL ? 12 : 4);
}

template <class C, bool FRESNEL, bool STAGE = false>
__global__ void __launch_bounds__(C::NT, C::MINB) k_col(const Slot *const *slots, int nx, int ny,
                                               const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    const float *__restrict__ mI = S.mI;
    const float s0 = S.s0;
    const int c0 = blockIdx.x * (C::L / kPanel);
    float2 v[C::E];
    constexpr int TW = C::N * C::L;
    float *ms = reinterpret_cast<float *>(sm + C::smem_words());
    float2 *ws = reinterpret_cast<float2 *>(ms + TW);
    if constexpr (STAGE) {
        const size_t off = (size_t)c0 * kPanel * nx; // the tile's run (nx = N)
        for (int c = threadIdx.x; c < TW / 4; c += C::NT) cp_async16(ms + 4 * c, mI + off + 4 * c);
        if constexpr (FRESNEL)
            for (int c = threadIdx.x; c < TW / 2; c += C::NT) cp_async16(ws + 2 * c, S.W + off + 2 * c);
    }

    for_each_slot<C, true, true>([&](int e, int s, int pos) {
        v[e] = P[paddr(pos, c0 * kPanel + s, nx)];
    });
    transform<C, true>(v, sm, tw);
    if constexpr (STAGE) {
        cp_async_wait_all();
        __syncthreads();
    }

    double diff = 0.0;
    for_each_slot<C, true, false>([&](int e, int s, int kx) {
        const int ky = c0 * kPanel + s;
        const size_t a = paddr(kx, ky, nx);
        const int b = ((s / kPanel) * C::N + kx) * kPanel + s % kPanel; // staged index
        const float m = STAGE ? ms[b] : __ldg(&mI[a]);
        float2 X = v[e];
        if (!FRESNEL) {
            // Planar: Psi = X s0; back-propagated value = projected Psi * s0
            X = planar_modulus(X, m, s0, diff);
        } else {
            const float2 cf = cmul(__ldg(&S.tx[kx]), __ldg(&S.ty[ky]));
            const float2 w = STAGE ? ws[b] : S.W[a];
            const float2 u = modulus(cadd(cscale(cmul(cf, X), s0), w), m, diff);
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

// finish the error metric of the column pass that just ran (block 0 of a
// slot's row pass): from x's projection, or -- algorithms whose only
// projection is of Ps x (a PfPs term alone) -- from Q's
template <int NT>
__device__ __forceinline__ void finish_error_row(const Slot &S)
{
    const double *part = S.project ? S.partials : (S.pfs ? S.qpartials : nullptr);
    if (part) {
        double t = 0.0;
        for (int b = threadIdx.x; b < S.ncol; b += NT) t += part[b];
        t = block_sum<NT>(t);
        if (threadIdx.x == 0) {
            const double e = t * S.inv_norm2;
            long long it = *S.iter;
            *S.err = e;
            S.ring[it % S.ring_len] = e;
            *S.iter = it + 1;
        }
    } else if (threadIdx.x == 0) {
        long long it = *S.iter;
        S.ring[it % S.ring_len] = *S.err;
        *S.iter = it + 1;
    }
}

} // namespace f32
} // namespace nadia

#include "fused32_tc.cuh"

namespace nadia {
namespace f32 {

template <class C, int MODE>
__global__ void __launch_bounds__(C::NT, C::MINB) k_row(const Slot *const *slots, int nx, int ny,
                                               const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    float2 *__restrict__ x = S.x;
    const int i0 = blockIdx.x * C::L;
    float2 v[C::E];

    if (MODE == kRowFull) {
        if (blockIdx.x == 0) finish_error_row<C::NT>(S);
        for_each_slot<C, false, true>([&](int e, int s, int pos) {
            v[e] = P[paddr(i0 + s, pos, nx)];
        });
        transform<C, false>(v, sm, tw);
        const float *__restrict__ sup = S.sup;
        const float wid = S.w_id, wpf = S.w_pf, wps = S.w_ps, wpsf = S.w_psf;
        const bool er = S.er;
        const bool tc = S.tc_on != 0;
        for_each_slot<C, false, false>([&](int e, int s, int pos) {
            const size_t a = paddr(i0 + s, pos, nx);
            const float f = support_factor(__ldg(&sup[a]));
            const float2 y = v[e];
            float2 xn;
            if (er) {
                xn = cscale(y, f);
                if (tc) xn = tc_apply(xn, S, a, pos, nx, ny, 1);
            } else {
                const float2 xk = x[a];
                float2 ps = make_float2(f * xk.x, f * xk.y), psf = make_float2(f * y.x, f * y.y);
                if (tc) {
                    ps = tc_apply(ps, S, a, pos, nx, ny, 0);
                    psf = tc_apply(psf, S, a, pos, nx, ny, 1);
                }
                xn = make_float2(wid * xk.x + wpf * y.x + wps * ps.x + wpsf * psf.x,
                                 wid * xk.y + wpf * y.y + wps * ps.y + wpsf * psf.y);
            }
            x[a] = xn;
            v[e] = xn;
        });
    } else if (MODE == kRowPfs || MODE == kRowPrimePfs) {
        // algorithms with a PfPs term (BaseCDI.c++:313-383): y = Pf x from P,
        // z = Pf Ps x from Q, the five-term combine, then the rows of x' to P
        // and of Ps x' to Q
        float2 *__restrict__ Q = S.Q;
        const float *__restrict__ sup = S.sup;
        float2 w[C::E];
        if (MODE == kRowPfs) {
            if (blockIdx.x == 0) finish_error_row<C::NT>(S);
            for_each_slot<C, false, true>([&](int e, int s, int pos) {
                v[e] = P[paddr(i0 + s, pos, nx)];
                w[e] = Q[paddr(i0 + s, pos, nx)];
            });
            transform<C, false>(v, sm, tw);
            __syncthreads();
            transform<C, false>(w, sm, tw);
            const float wid = S.w_id, wpf = S.w_pf, wps = S.w_ps, wpsf = S.w_psf, wpfs = S.w_pfs;
            for_each_slot<C, false, false>([&](int e, int s, int pos) {
                const size_t a = paddr(i0 + s, pos, nx);
                const float f = support_factor(__ldg(&sup[a]));
                const float2 xk = x[a], y = v[e], z = w[e];
                const float2 xn = make_float2(
                    wid * xk.x + wpfs * z.x + wpf * y.x + wps * (f * xk.x) + wpsf * (f * y.x),
                    wid * xk.y + wpfs * z.y + wpf * y.y + wps * (f * xk.y) + wpsf * (f * y.y));
                x[a] = xn;
                v[e] = xn;
                w[e] = cscale(xn, f);
            });
        } else {
            for_each_slot<C, true, true>([&](int e, int s, int pos) {
                const size_t a = paddr(i0 + s, pos, nx);
                v[e] = x[a];
                w[e] = cscale(v[e], support_factor(__ldg(&sup[a])));
            });
        }
        transform<C, true>(v, sm, tw);
        for_each_slot<C, true, false>([&](int e, int s, int pos) {
            P[paddr(i0 + s, pos, nx)] = v[e];
        });
        __syncthreads();
        transform<C, true>(w, sm, tw);
        for_each_slot<C, true, false>([&](int e, int s, int pos) {
            Q[paddr(i0 + s, pos, nx)] = w[e];
        });
        return;
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


} // namespace f32
} // namespace nadia

#include "fused32_persist.cuh"
#include "fused32_wf.cuh"

namespace nadia {
namespace f32 {

// --------------------------------------------------------------- variants

template <class C>
constexpr size_t smem_bytes()
{
    return (size_t)C::smem_words() * sizeof(float2);
}

template <class C, class K>
void set_smem(K kernel)
{
    NADIA_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem_bytes<C>()));
}

template <class CC, class CR>
void prepare_variant()
{
    set_smem<CC>(k_col<CC, false>);
    set_smem<CC>(k_col<CC, true>);
    set_smem<CR>(k_row<CR, kRowFull>);
    set_smem<CR>(k_row<CR, kRowPrime>);
    set_smem<CR>(k_row<CR, kRowPfs>);
    set_smem<CR>(k_row<CR, kRowPrimePfs>);
    set_smem<CC>(k_wf_col<CC>);
    set_smem<CR>(k_wf_row<CR, kRowFull>);
    set_smem<CR>(k_wf_row<CR, kRowPrime>);
    set_smem<CR>(k_row_tc<CR, 1>);
    set_smem<CR>(k_row_tc<CR, 2>);
}

template <class C>
void launch_row_tc(int half, const Slot *const *slots, int nslots, int nx, int ny, const float2 *tw,
                   cudaStream_t st)
{
    const dim3 grid(nx / C::L, nslots);
    if (half == 1)
        k_row_tc<C, 1><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    else
        k_row_tc<C, 2><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
}

template <class C>
void launch_wf_col(const Slot *const *slots, int nslots, int nx, int ny, const float2 *tw,
                   cudaStream_t st)
{
    k_wf_col<C><<<dim3(ny / C::L, nslots), C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
}

template <class C>
void launch_wf_row(int mode, const Slot *const *slots, int nslots, int nx, int ny, const float2 *tw,
                   cudaStream_t st)
{
    const dim3 grid(nx / C::L, nslots);
    if (mode == kRowFull)
        k_wf_row<C, kRowFull><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    else
        k_wf_row<C, kRowPrime><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
}

template <class C>
void launch_col(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                const float2 *tw, cudaStream_t st)
{
    dim3 grid(ny / C::L, nslots);
    if (fresnel)
        k_col<C, true><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    else
        k_col<C, false><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
}

template <class C>
void launch_row(int mode, const Slot *const *slots, int nslots, int nx, int ny, const float2 *tw,
                cudaStream_t st)
{
    dim3 grid(nx / C::L, nslots);
    switch (mode) {
    case kRowFull:
        k_row<C, kRowFull><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
        break;
    case kRowPrime:
        k_row<C, kRowPrime><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
        break;
    case kRowPfs:
        k_row<C, kRowPfs><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
        break;
    default:
        k_row<C, kRowPrimePfs><<<grid, C::NT, smem_bytes<C>(), st>>>(slots, nx, ny, tw);
    }
}

// shared memory of the persistent passes: STAGES stages of P and sqrt(I)
// (column); two stages of P plus x and the support (row); and mbarriers
template <class C, int STAGES = 2, int MMODE = 0>
constexpr size_t persist_col_smem() { return persist_col_bytes<C, STAGES, MMODE>(); }
template <class C>
constexpr size_t persist_row_smem() { return (size_t)C::N * C::L * 28 + 24; }

// CTAs of a persistent kernel resident per SM (at most MINB), measured when
// the variant is prepared (before any launch, outside graph capture)
template <class K>
int resident_ctas(K kernel, int nt, size_t smem, int minb)
{
    int occ = 0;
    NADIA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, nt, smem));
    NADIA_REQUIRE(occ > 0, NADIA_ERR_CUDA, "a persistent pass does not fit on an SM");
    return occ < minb ? occ : minb;
}

template <class C, int STAGES, int MMODE>
struct PersistCol {
    static inline int per_sm = 1;
};
template <class C>
struct PersistRow {
    static inline int per_sm = 1;
};

template <class C, int STAGES, int MMODE = 0>
void prepare_persistent_col()
{
    constexpr int bytes = (int)persist_col_smem<C, STAGES, MMODE>();
    NADIA_CUDA(cudaFuncSetAttribute(kp_col<C, false, STAGES, MMODE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    NADIA_CUDA(cudaFuncSetAttribute(kp_col<C, true, STAGES, MMODE>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    PersistCol<C, STAGES, MMODE>::per_sm =
        resident_ctas(kp_col<C, false, STAGES, MMODE>, C::NT, bytes, C::MINB);
}

template <class C>
void prepare_persistent_row()
{
    set_smem<C>(k_row<C, kRowFull>);
    set_smem<C>(k_row<C, kRowPrime>);
    set_smem<C>(k_row<C, kRowPfs>);
    set_smem<C>(k_row<C, kRowPrimePfs>);
    NADIA_CUDA(cudaFuncSetAttribute(kp_row<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)persist_row_smem<C>()));
    PersistRow<C>::per_sm = resident_ctas(kp_row<C>, C::NT, persist_row_smem<C>(), C::MINB);
}

template <class CC, class CR>
void prepare_persistent()
{
    prepare_variant<CC, CR>();
    prepare_persistent_col<CC, 2>();
    prepare_persistent_row<CR>();
}

template <class C, int STAGES, int MMODE = 0>
void launch_col_persistent(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                           const float2 *tw, cudaStream_t st)
{
    constexpr size_t bytes = persist_col_smem<C, STAGES, MMODE>();
    const int ntiles = (ny / C::L) * nslots;
    const int cap = sm_count() * PersistCol<C, STAGES, MMODE>::per_sm;
    const int grid = ntiles < cap ? ntiles : cap;
    if (fresnel)
        kp_col<C, true, STAGES, MMODE><<<grid, C::NT, bytes, st>>>(slots, nslots, nx, ny, tw);
    else
        kp_col<C, false, STAGES, MMODE><<<grid, C::NT, bytes, st>>>(slots, nslots, nx, ny, tw);
}

template <class C>
void launch_row_persistent(int mode, const Slot *const *slots, int nslots, int nx, int ny,
                           const float2 *tw, cudaStream_t st)
{
    if (mode != kRowFull) {
        launch_row<C>(mode, slots, nslots, nx, ny, tw, st);
        return;
    }
    const int ntiles = (nx / C::L) * nslots;
    const int cap = sm_count() * PersistRow<C>::per_sm;
    const int grid = ntiles < cap ? ntiles : cap;
    kp_row<C><<<grid, C::NT, persist_row_smem<C>(), st>>>(slots, nslots, nx, ny, tw);
}

// One tile shape (N, NT threads, L signals per block, radices, swizzle, min
// blocks per SM) as a column-pass and a row-pass variant.
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_variant(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB>;
    using CR = TileCfg<N, NT, L, kRowMap, Radices<Rs...>, SW, MINB>;
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.radices = radices;
    t.prepare = &prepare_variant<CC, CR>;
    t.col = &launch_col<CC>;
    t.row = &launch_row<CR>;
    t.wf_col = &launch_wf_col<CC>;
    t.wf_row = &launch_wf_row<CR>;
    t.tc_row = &launch_row_tc<CR>;
    return t;
}

// Column-pass-only variants whose tiles stage sqrt(I) (and the white field)
// by cp.async at the start (k_col's STAGE), plain or with ping-pong exchanges.
template <class C>
void prepare_staged()
{
    NADIA_CUDA(cudaFuncSetAttribute(k_col<C, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(smem_bytes<C>() + col_stage_bytes<C, false>())));
    NADIA_CUDA(cudaFuncSetAttribute(k_col<C, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(smem_bytes<C>() + col_stage_bytes<C, true>())));
}

template <class C>
void launch_col_staged(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                       const float2 *tw, cudaStream_t st)
{
    dim3 grid(ny / C::L, nslots);
    if (fresnel)
        k_col<C, true, true><<<grid, C::NT, smem_bytes<C>() + col_stage_bytes<C, true>(), st>>>(
            slots, nx, ny, tw);
    else
        k_col<C, false, true><<<grid, C::NT, smem_bytes<C>() + col_stage_bytes<C, false>(), st>>>(
            slots, nx, ny, tw);
}

template <int N, int NT, int L, int MINB, class SW, bool PING, int... Rs>
TileVariant make_staged_col(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB, PING>;
    static_assert(smem_bytes<CC>() + col_stage_bytes<CC, true>() <= 227 * 1024, "stage too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.ping = PING;
    t.radices = radices;
    t.prepare = &prepare_staged<CC>;
    t.col = &launch_col_staged<CC>; // column pass only (no row, FresnelCDI_WF or constraint pass)
    return t;
}
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_staged(const char *radices)
{
    return make_staged_col<N, NT, L, MINB, SW, false, Rs...>(radices);
}
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_staged_ping(const char *radices)
{
    return make_staged_col<N, NT, L, MINB, SW, true, Rs...>(radices);
}

// The same tile shape with ping-pong exchange buffers (twice the shared memory).
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_ping(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB, true>;
    using CR = TileCfg<N, NT, L, kRowMap, Radices<Rs...>, SW, MINB, true>;
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.ping = true;
    t.radices = radices;
    t.prepare = &prepare_variant<CC, CR>;
    t.col = &launch_col<CC>;
    t.row = &launch_row<CR>;
    t.tc_row = &launch_row_tc<CR>;
    return t;
}

// The same tile shape as persistent, TMA-pipelined passes (tiles of at most
// 8192 elements, so both stages fit in shared memory); MINB CTAs per SM where
// shared memory allows.  RL: the radix list type (Radices or RadicesTW).
template <int N, int NT, int L, int MINB, class SW, class RL>
TileVariant make_persistent_rl(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, RL, SW, MINB>;
    using CR = TileCfg<N, NT, L, kRowMap, RL, SW, MINB>;
    static_assert(persist_row_smem<CR>() <= 227 * 1024, "persistent row tile too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.persistent = true;
    t.radices = radices;
    t.prepare = &prepare_persistent<CC, CR>;
    t.col = &launch_col_persistent<CC, 2>;
    t.row = &launch_row_persistent<CR>;
    return t;
}

template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent(const char *radices)
{
    return make_persistent_rl<N, NT, L, MINB, SW, Radices<Rs...>>(radices);
}
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent_tw(const char *radices)
{
    return make_persistent_rl<N, NT, L, MINB, SW, RadicesTW<Rs...>>(radices);
}

// A persistent column pass with one stage per CTA (MINB CTAs share an SM);
// no row pass.
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent_single(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB>;
    static_assert(persist_col_smem<CC, 1>() * MINB <= 226 * 1024, "stages too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.persistent = true;
    t.single = true;
    t.radices = radices;
    t.prepare = &prepare_persistent_col<CC, 1>;
    t.col = &launch_col_persistent<CC, 1>;
    return t;
}

// A persistent column pass reading sqrt(I) straight from global memory:
// STAGES stages of P, and with PING a second exchange buffer (one barrier per
// exchange); no row pass.
template <int STAGES, bool PING, int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent_direct_t(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB, PING>;
    static_assert(persist_col_smem<CC, STAGES, 1>() * MINB <= 226 * 1024, "stages too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.persistent = true;
    t.single = STAGES == 1;
    t.ping = PING;
    t.direct = true;
    t.radices = radices;
    t.prepare = &prepare_persistent_col<CC, STAGES, 1>;
    t.col = &launch_col_persistent<CC, STAGES, 1>;
    return t;
}
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent_direct(const char *radices)
{
    return make_persistent_direct_t<1, false, N, NT, L, MINB, SW, Rs...>(radices);
}
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent_ping(const char *radices)
{
    return make_persistent_direct_t<2, true, N, NT, L, MINB, SW, Rs...>(radices);
}

// The row pass in G independent groups of NT threads a CTA (tiles of L rows
// per group); no column pass.
template <class C>
void prepare_grouped_row()
{
    set_smem<C>(k_row<C, kRowFull>);
    set_smem<C>(k_row<C, kRowPrime>);
    set_smem<C>(k_row<C, kRowPfs>);
    set_smem<C>(k_row<C, kRowPrimePfs>);
    NADIA_CUDA(cudaFuncSetAttribute(kg_row<C>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)grouped_row_smem<C>()));
}

template <class C>
void launch_row_grouped(int mode, const Slot *const *slots, int nslots, int nx, int ny,
                        const float2 *tw, cudaStream_t st)
{
    if (mode != kRowFull) {
        launch_row<C>(mode, slots, nslots, nx, ny, tw, st);
        return;
    }
    const int ntiles = (nx / C::L) * nslots;
    const int ctas = (ntiles + C::GROUPS - 1) / C::GROUPS;
    const int grid = ctas < sm_count() ? ctas : sm_count();
    kg_row<C><<<grid, C::NT * C::GROUPS, grouped_row_smem<C>(), st>>>(slots, nslots, nx, ny, tw);
}

template <class C>
void prepare_grouped_col()
{
    NADIA_CUDA(cudaFuncSetAttribute(kg_col<C, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)grouped_col_smem<C>()));
    NADIA_CUDA(cudaFuncSetAttribute(kg_col<C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)grouped_col_smem<C>()));
}

template <class C>
void launch_col_grouped(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                        const float2 *tw, cudaStream_t st)
{
    const int ntiles = (ny / C::L) * nslots;
    const int ctas = (ntiles + C::GROUPS - 1) / C::GROUPS;
    const int grid = ctas < sm_count() ? ctas : sm_count();
    if (fresnel)
        kg_col<C, true><<<grid, C::NT * C::GROUPS, grouped_col_smem<C>(), st>>>(slots, nslots, nx, ny, tw);
    else
        kg_col<C, false><<<grid, C::NT * C::GROUPS, grouped_col_smem<C>(), st>>>(slots, nslots, nx, ny, tw);
}

// The column pass in G independent groups of NT threads a CTA, each on half
// panels (two columns); no row pass.
template <int N, int NT, int L, int G, class SW, int... Rs>
TileVariant make_grouped_col(const char *radices)
{
    static_assert(L == 2, "half-panel tiles");
    using CC = TileCfg<N, NT, 2, kRowMap, Radices<Rs...>, SW, 1, false, G>;
    static_assert(grouped_col_smem<CC>() <= 227 * 1024, "grouped column stages too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = 2;
    t.minb = 1;
    t.persistent = true;
    t.groups = G;
    t.radices = radices;
    t.prepare = &prepare_grouped_col<CC>;
    t.col = &launch_col_grouped<CC>;
    return t;
}

template <int N, int NT, int L, int G, class SW, class RL>
TileVariant make_grouped_row_rl(const char *radices)
{
    using CR = TileCfg<N, NT, L, kRowMap, RL, SW, 1, false, G>;
    static_assert(grouped_row_smem<CR>() <= 227 * 1024, "grouped row stages too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = 1;
    t.persistent = true;
    t.groups = G;
    t.radices = radices;
    t.prepare = &prepare_grouped_row<CR>;
    t.row = &launch_row_grouped<CR>;
    return t;
}

template <int N, int NT, int L, int G, class SW, int... Rs>
TileVariant make_grouped_row(const char *radices)
{
    return make_grouped_row_rl<N, NT, L, G, SW, Radices<Rs...>>(radices);
}
template <int N, int NT, int L, int G, class SW, int... Rs>
TileVariant make_grouped_row_tw(const char *radices)
{
    return make_grouped_row_rl<N, NT, L, G, SW, RadicesTW<Rs...>>(radices);
}

// A persistent column pass with two stages of P, one stage of sqrt(I)
// refilled after each modulus, and ping-pong exchanges; no row pass.
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent_mstage(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB, true>;
    static_assert(persist_col_smem<CC, 2, 2>() <= 227 * 1024, "stages too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.persistent = true;
    t.ping = true;
    t.radices = radices;
    t.prepare = &prepare_persistent_col<CC, 2, 2>;
    t.col = &launch_col_persistent<CC, 2, 2>;
    return t;
}

// A persistent row pass only: tiles of L rows (L = 2 allowed, below the
// panel width a column tile needs), MINB CTAs per SM.
template <int N, int NT, int L, int MINB, class SW, int... Rs>
TileVariant make_persistent_row(const char *radices)
{
    using CR = TileCfg<N, NT, L, kRowMap, Radices<Rs...>, SW, MINB>;
    static_assert(persist_row_smem<CR>() * MINB <= 226 * 1024, "row stages too large");
    TileVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.minb = MINB;
    t.persistent = true;
    t.radices = radices;
    t.prepare = &prepare_persistent_row<CR>;
    t.row = &launch_row_persistent<CR>;
    return t;
}

} // namespace f32
} // namespace nadia
