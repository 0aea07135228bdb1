// fused32_poly.cuh -- the FP32 PolyCDI iteration (PolyCDI::iterate,
// PolyCDI.c++:130-250) as three passes over the padded grid.
//
// The estimate x (nx x ny) is zero-padded to mx x my = (nx + 2 px) x
// (ny + 2 py) around each projection (get_padded / get_unpadded).  The work
// array P holds the padded grid in the panel layout; only its rows
// px..px+nx-1 ever carry the estimate, so the forward column transform reads
// those rows and takes the others as zero, and the inverse column transform
// writes back only those rows.
//
//   column pass 1: forward column transforms; Psi (transform order) back to P,
//                  |Psi|^2 of the centred detector field (propagate_to_detector:
//                  FFT then Complex_2D::invert(true)) to q
//   expansion:     for every measured pixel of the detector window, the
//                  wavelength-expanded intensity of expand_wl (PolyCDI.c++:296-334)
//                  gathered from q, the modulus ratio of PolyCDI::scale_intensity
//                  (PolyCDI.c++:255-292) to `ratio`, and the FP64 error partials
//                  (a light kernel at full occupancy: the gathers are latency-bound)
//   column pass 2: Psi times the ratio, inverse column transforms; the
//                  estimate's rows to P
//   row pass:      inverse row transforms of those rows, the window
//                  py..py+ny-1 combined with x and the support (the generic
//                  combine of PolyCDI.c++:201-237, or ER), x written, forward
//                  row transforms of the zero-padded rows to P
//
// The passes are separate launches because every expanded pixel reads
// |Psi|^2 from other columns (q stays in L2: 4 bytes per padded pixel).
#pragma once

#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

// centred coordinate of transform index k on an axis of even length m
__device__ __forceinline__ int centred(int k, int m)
{
    const int c = k + m / 2;
    return c >= m ? c - m : c;
}

template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) k_poly_col_fwd(const Slot *const *slots,
                                                                   const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    const int mx = S.mx, my = S.my, r0 = S.px, r1 = S.mx - S.px; // the estimate's rows
    const int c0 = blockIdx.x * (C::L / kPanel);
    float2 v[C::E];
    for_each_slot<C, true, true>([&](int e, int s, int pos) {
        v[e] = (pos >= r0 && pos < r1) ? P[paddr(pos, c0 * kPanel + s, mx)]
                                       : make_float2(0.f, 0.f);
    });
    transform<C, true>(v, sm, tw);
    const float s02 = S.s0 * S.s0;
    float *__restrict__ q = S.q;
    for_each_slot<C, true, false>([&](int e, int s, int kx) {
        const int ky = c0 * kPanel + s;
        const float2 X = v[e];
        P[paddr(kx, ky, mx)] = X;
        q[paddr(centred(kx, mx), centred(ky, my), mx)] = s02 * (X.x * X.x + X.y * X.y);
    });
}

constexpr int kExpandThreads = 256;
constexpr int kExpandBlocks = 1184; // 8 per SM
constexpr int kNoSample = -(1 << 30); // offset of a sample outside the padded grid

// One thread per pixel of the detector window in the panel layout (lanes
// cover 4 columns x 8 rows, so the gathered q addresses of a warp are nearly
// contiguous; 32-bit index arithmetic, one division per pixel).  S.gx[l][i]
// and S.gy[l][j] hold the parts of q's panel address of the sample that
// wavelength l takes for row i and column j (row part 4 ga, column part
// (gb/4) 4 mx + gb%4, kNoSample when outside the grid), so a sample's address
// is their sum and it exists when that sum is not negative.
// ratio = sqrt(I)/sqrt(I_calc) (0 when I_calc = 0) for measured pixels, 1
// elsewhere; partials[block] = sum of (sqrt(I) - sqrt(I_calc))^2.
__global__ void __launch_bounds__(kExpandThreads) k_poly_expand(const Slot *const *slots)
{
    const Slot &S = *slots[blockIdx.y];
    const int mx = S.mx, px = S.px, py = S.py;
    const int nx = mx - 2 * px, ny = S.my - 2 * py;
    const int nl = S.nl;
    const float *__restrict__ q = S.q;
    const float *__restrict__ mI = S.mI;
    const int *__restrict__ gx = S.gx;
    const int *__restrict__ gy = S.gy;
    const float *__restrict__ wl = S.wl;
    float *__restrict__ ratio = S.ratio;
    const unsigned n = (unsigned)nx * (unsigned)ny;
    double diff = 0.0;
    for (unsigned a = blockIdx.x * kExpandThreads + threadIdx.x; a < n;
         a += gridDim.x * kExpandThreads) {
        const unsigned t = a / kPanel, jp = t / (unsigned)nx;
        const int i = (int)(t - jp * (unsigned)nx), j = (int)(jp * kPanel + a % kPanel);
        const float m = __ldg(&mI[a]);
        float r = 1.f;
        if (!(m < 0.f)) {
            // groups of four wavelengths: their loads issue together (a whole
            // spectrum's loads at once measured slower)
            float acc = 0.f;
            int l = 0;
            for (; l + 4 <= nl; l += 4) {
                int off[4];
                float qv[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    off[u] = __ldg(&gx[(l + u) * nx + i]) + __ldg(&gy[(l + u) * ny + j]);
#pragma unroll
                for (int u = 0; u < 4; ++u) qv[u] = off[u] >= 0 ? __ldg(&q[off[u]]) : 0.f;
#pragma unroll
                for (int u = 0; u < 4; ++u) acc += __ldg(&wl[l + u]) * qv[u];
            }
            for (; l < nl; ++l) {
                const int o = __ldg(&gx[l * nx + i]) + __ldg(&gy[l * ny + j]);
                acc += __ldg(&wl[l]) * (o >= 0 ? __ldg(&q[o]) : 0.f);
            }
            const float calc = sqrtf(acc);
            r = calc == 0.f ? 0.f : m / calc;
            const double d = (double)m - (double)calc;
            diff += d * d;
        }
        ratio[a] = r;
    }
    const double tot = block_sum<kExpandThreads>(diff);
    if (threadIdx.x == 0) S.partials[blockIdx.x] = tot;
}

template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) k_poly_col_inv(const Slot *const *slots,
                                                                   const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    const int mx = S.mx, my = S.my, px = S.px, py = S.py;
    const int nx = mx - 2 * px, ny = my - 2 * py;
    const float *__restrict__ ratio = S.ratio;
    const int c0 = blockIdx.x * (C::L / kPanel);
    const float s02 = S.s0 * S.s0;
    float2 v[C::E];
    for_each_slot<C, true, false>([&](int e, int s, int kx) {
        const int ky = c0 * kPanel + s;
        const int i = centred(kx, mx) - px, j = centred(ky, my) - py;
        float r = 1.f;
        if (i >= 0 && i < nx && j >= 0 && j < ny) r = __ldg(&ratio[paddr(i, j, nx)]);
        v[e] = cscale(P[paddr(kx, ky, mx)], s02 * r);
    });
    transform<C, false>(v, sm, tw);
    for_each_slot<C, false, false>([&](int e, int s, int pos) {
        if (pos >= px && pos < px + nx) P[paddr(pos, c0 * kPanel + s, mx)] = v[e];
    });
}

template <class C, int MODE>
__global__ void __launch_bounds__(C::NT, C::MINB) k_poly_row(const Slot *const *slots,
                                                               const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    float2 *__restrict__ x = S.x;
    const int mx = S.mx, my = S.my, px = S.px, py = S.py;
    const int nx = mx - 2 * px, ny = my - 2 * py;
    const int i0 = blockIdx.x * C::L; // unpadded row of the tile's first signal
    float2 v[C::E];

    if (MODE == kRowFull) {
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
            v[e] = P[paddr(px + i0 + s, pos, mx)];
        });
        transform<C, false>(v, sm, tw);
        const float *__restrict__ sup = S.sup;
        const float wid = S.w_id, wpf = S.w_pf, wps = S.w_ps, wpsf = S.w_psf;
        const bool er = S.er;
        for_each_slot<C, false, false>([&](int e, int s, int pos) {
            const int j = pos - py;
            float2 xn = make_float2(0.f, 0.f);
            if (j >= 0 && j < ny) {
                const size_t a = paddr(i0 + s, j, nx);
                const float f = support_factor(__ldg(&sup[a]));
                const float2 y = v[e];
                if (er) {
                    xn = cscale(y, f);
                } else {
                    const float2 xk = x[a];
                    xn = combine2(xk, y, f, wid, wpf, wps, wpsf);
                }
                x[a] = xn;
            }
            v[e] = xn;
        });
    } else {
        for_each_slot<C, true, true>([&](int e, int s, int pos) {
            const int j = pos - py;
            v[e] = (j >= 0 && j < ny) ? x[paddr(i0 + s, j, nx)] : make_float2(0.f, 0.f);
        });
    }
    transform<C, true>(v, sm, tw);
    for_each_slot<C, true, false>([&](int e, int s, int pos) {
        P[paddr(px + i0 + s, pos, mx)] = v[e];
    });
}

template <class CC, class CR>
void prepare_poly()
{
    set_smem<CC>(k_poly_col_fwd<CC>);
    set_smem<CC>(k_poly_col_inv<CC>);
    set_smem<CR>(k_poly_row<CR, kRowFull>);
    set_smem<CR>(k_poly_row<CR, kRowPrime>);
}

// column passes: tiles = my / L column tiles; row pass: tiles = nx / L row tiles
template <class C>
void launch_poly_col_fwd(const Slot *const *slots, int nslots, int tiles, cudaStream_t st,
                         const float2 *tw)
{
    k_poly_col_fwd<C><<<dim3(tiles, nslots), C::NT, smem_bytes<C>(), st>>>(slots, tw);
}

template <class C>
void launch_poly_col_inv(const Slot *const *slots, int nslots, int tiles, cudaStream_t st,
                         const float2 *tw)
{
    k_poly_expand<<<dim3(kExpandBlocks, nslots), kExpandThreads, 0, st>>>(slots);
    k_poly_col_inv<C><<<dim3(tiles, nslots), C::NT, smem_bytes<C>(), st>>>(slots, tw);
}

template <class C>
void launch_poly_row(int mode, const Slot *const *slots, int nslots, int tiles, cudaStream_t st,
                     const float2 *tw)
{
    if (mode == kRowFull)
        k_poly_row<C, kRowFull><<<dim3(tiles, nslots), C::NT, smem_bytes<C>(), st>>>(slots, tw);
    else
        k_poly_row<C, kRowPrime><<<dim3(tiles, nslots), C::NT, smem_bytes<C>(), st>>>(slots, tw);
}

template <int N, int NT, int L, int MINB, class SW, int... Rs>
PolyVariant make_poly(const char *radices)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB>;
    using CR = TileCfg<N, NT, L, kRowMap, Radices<Rs...>, SW, MINB>;
    PolyVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.radices = radices;
    t.prepare = &prepare_poly<CC, CR>;
    t.col_fwd = &launch_poly_col_fwd<CC>;
    t.col_inv = &launch_poly_col_inv<CC>;
    t.row = &launch_poly_row<CR>;
    return t;
}

} // namespace f32
} // namespace nadia
