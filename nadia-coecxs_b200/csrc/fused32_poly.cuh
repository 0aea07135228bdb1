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
    if ((ny & 3) == 0) {
        // whole panels: a thread takes the four pixels (i, 4 jp .. 4 jp + 3),
        // sixteen contiguous bytes of sqrt(I) and of the ratio, and reads each
        // wavelength's row part once and its four column parts as one vector
        // (lanes run along i, so the column parts are one broadcast); each
        // pixel's sum runs over the wavelengths in the same order as below
        const float4 *__restrict__ mI4 = reinterpret_cast<const float4 *>(mI);
        float4 *__restrict__ ratio4 = reinterpret_cast<float4 *>(ratio);
        const unsigned cells = n / kPanel;
        for (unsigned u = blockIdx.x * kExpandThreads + threadIdx.x; u < cells;
             u += gridDim.x * kExpandThreads) {
            const unsigned jp = u / (unsigned)nx;
            const int i = (int)(u - jp * (unsigned)nx);
            const float4 m4 = __ldg(&mI4[u]);
            const float m[4] = {m4.x, m4.y, m4.z, m4.w};
            float r[4] = {1.f, 1.f, 1.f, 1.f};
            if (!(m[0] < 0.f) || !(m[1] < 0.f) || !(m[2] < 0.f) || !(m[3] < 0.f)) {
                const int4 *__restrict__ gy4 = reinterpret_cast<const int4 *>(gy + jp * kPanel);
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                int l = 0;
                for (; l + 2 <= nl; l += 2) {
                    float qv[2][4];
#pragma unroll
                    for (int u2 = 0; u2 < 2; ++u2) {
                        const int ox = __ldg(&gx[(l + u2) * nx + i]);
                        const int4 oy = __ldg(&gy4[(l + u2) * (ny / kPanel)]);
                        const int o[4] = {ox + oy.x, ox + oy.y, ox + oy.z, ox + oy.w};
#pragma unroll
                        for (int k = 0; k < 4; ++k) qv[u2][k] = o[k] >= 0 ? __ldg(&q[o[k]]) : 0.f;
                    }
#pragma unroll
                    for (int u2 = 0; u2 < 2; ++u2) {
                        const float w = __ldg(&wl[l + u2]);
#pragma unroll
                        for (int k = 0; k < 4; ++k) acc[k] += w * qv[u2][k];
                    }
                }
                for (; l < nl; ++l) {
                    const int ox = __ldg(&gx[l * nx + i]);
                    const int4 oy = __ldg(&gy4[l * (ny / kPanel)]);
                    const int o[4] = {ox + oy.x, ox + oy.y, ox + oy.z, ox + oy.w};
                    const float w = __ldg(&wl[l]);
#pragma unroll
                    for (int k = 0; k < 4; ++k) acc[k] += w * (o[k] >= 0 ? __ldg(&q[o[k]]) : 0.f);
                }
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    if (m[k] < 0.f) continue;
                    // sqrt(I_calc) and the ratio from one approximate reciprocal
                    // square root (no IEEE square-root or division sequence)
                    const float inv = rsqrt_normal(acc[k]);
                    const float calc = acc[k] * inv;
                    r[k] = calc == 0.f ? 0.f : m[k] * inv;
                    const double d = (double)m[k] - (double)calc;
                    diff += d * d;
                }
            }
            ratio4[u] = make_float4(r[0], r[1], r[2], r[3]);
        }
    } else {
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

// Shared memory of the row pass: the exchange tile, then (PREF) the tile's
// rows of x and of the support, staged in their panel order [ny/4][L][4]
template <class C, bool PREF>
constexpr size_t poly_row_smem()
{
    return (size_t)C::smem_words() * sizeof(float2) + (PREF ? (size_t)C::N * C::L * 12 : 0);
}

// PREF: when the window's width is a multiple of the panel (always for the
// padded grids in use), the tile's rows of x and of the support are copied
// into shared memory by cp.async at the start, so those loads run during the
// inverse row transform instead of stalling the combine after it.  The tile's
// rows of a panel are one contiguous run of L*4 elements.
template <class C, int MODE, bool PREF>
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
    float2 *xs = sm + C::smem_words();
    float *ss = reinterpret_cast<float *>(xs + C::N * C::L);
    const bool staged = PREF && MODE == kRowFull && (ny & 3) == 0;
    if (staged) {
        constexpr int SEG = C::L * kPanel; // elements of one panel's run
        const int nseg = ny / kPanel;
        const bool need_x = !S.er;
        const float2 *__restrict__ xg = x + (size_t)i0 * kPanel;
        const float *__restrict__ sg = S.sup + (size_t)i0 * kPanel;
        // x: SEG/2 chunks of 16 bytes a run; the support: SEG/4
        for (int c = threadIdx.x; c < nseg * (SEG / 2); c += C::NT) {
            if (!need_x) break;
            const int jp = c / (SEG / 2), k = c % (SEG / 2);
            cp_async16(xs + jp * SEG + 2 * k, xg + (size_t)jp * nx * kPanel + 2 * k);
        }
        for (int c = threadIdx.x; c < nseg * (SEG / 4); c += C::NT) {
            const int jp = c / (SEG / 4), k = c % (SEG / 4);
            cp_async16(ss + jp * SEG + 4 * k, sg + (size_t)jp * nx * kPanel + 4 * k);
        }
    }

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
        if (staged) {
            cp_async_wait_all();
            __syncthreads();
        }
        const float *__restrict__ sup = S.sup;
        const float wid = S.w_id, wpf = S.w_pf, wps = S.w_ps, wpsf = S.w_psf;
        const bool er = S.er;
        for_each_slot<C, false, false>([&](int e, int s, int pos) {
            const int j = pos - py;
            float2 xn = make_float2(0.f, 0.f);
            if (j >= 0 && j < ny) {
                const size_t a = paddr(i0 + s, j, nx);
                const int b = ((j / kPanel) * C::L + s) * kPanel + j % kPanel; // staged index
                const float f = support_factor(staged ? ss[b] : __ldg(&sup[a]));
                const float2 y = v[e];
                if (er) {
                    xn = cscale(y, f);
                } else {
                    const float2 xk = staged ? xs[b] : x[a];
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

template <class CC, class CR, bool PREF>
void prepare_poly()
{
    set_smem<CC>(k_poly_col_fwd<CC>);
    set_smem<CC>(k_poly_col_inv<CC>);
    NADIA_CUDA(cudaFuncSetAttribute(k_poly_row<CR, kRowFull, PREF>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)poly_row_smem<CR, PREF>()));
    set_smem<CR>(k_poly_row<CR, kRowPrime, PREF>);
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

template <class C, bool PREF>
void launch_poly_row(int mode, const Slot *const *slots, int nslots, int tiles, cudaStream_t st,
                     const float2 *tw)
{
    if (mode == kRowFull)
        k_poly_row<C, kRowFull, PREF>
            <<<dim3(tiles, nslots), C::NT, poly_row_smem<C, PREF>(), st>>>(slots, tw);
    else
        k_poly_row<C, kRowPrime, PREF><<<dim3(tiles, nslots), C::NT, smem_bytes<C>(), st>>>(slots, tw);
}

template <int N, int NT, int L, int MINB, class SW, int... Rs>
PolyVariant make_poly(const char *radices, bool prefetch = true)
{
    using CC = TileCfg<N, NT, L, kColMap, Radices<Rs...>, SW, MINB>;
    using CR = TileCfg<N, NT, L, kRowMap, Radices<Rs...>, SW, MINB>;
    PolyVariant t;
    t.n = N;
    t.nt = NT;
    t.L = L;
    t.radices = radices;
    t.prepare = prefetch ? &prepare_poly<CC, CR, true> : &prepare_poly<CC, CR, false>;
    t.col_fwd = &launch_poly_col_fwd<CC>;
    t.col_inv = &launch_poly_col_inv<CC>;
    t.row = prefetch ? &launch_poly_row<CR, true> : &launch_poly_row<CR, false>;
    return t;
}

} // namespace f32
} // namespace nadia
