// fused32_mixed.cuh -- one persistent launch per pass over reconstructions of
// several grid sizes (nadia_iterate_many's batched path).
//
// A launch walks a work list of items (reconstruction, tile, length class).
// Every length class is a tile configuration of the same thread count, so
// one kernel holds the code of all of them and picks the class per item; the
// shared-memory stages are sized for the largest tile.  The list is ordered
// by class and each CTA takes one contiguous range of it, cut so that the
// ranges carry equal estimated work: a CTA runs one class (two where its range
// crosses a class boundary), so its instruction working set stays that of one
// tile shape.  The TMA pipeline brings item i+1 (whatever its class) while
// item i is transformed, as in the single-length persistent passes.
//
// The per-tile arithmetic is that of the single-length persistent passes
// (fused32_persist.cuh) for the class's tile configuration: a reconstruction's
// result depends on its own grid only, never on the other items of the list.
#pragma once

#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

// twiddle tables of the classes, by value in the launch parameters
constexpr int kMixMaxClasses = 8;
struct MixTw {
    const float2 *t[kMixMaxClasses];
};

// A class list: tile configurations (TileCfg) of one thread count, each of a
// different transform length.
template <class... Cs>
struct MixFamily {
    static constexpr int K = sizeof...(Cs);
    static_assert(K >= 1 && K <= kMixMaxClasses, "1 to 8 classes");
    static constexpr int NT = [] {
        constexpr int a[] = {Cs::NT...};
        for (int i = 1; i < K; ++i)
            if (a[i] != a[0]) return -1;
        return a[0];
    }();
    static_assert(NT > 0, "every class runs on the same thread count");
    static constexpr int maxTW()
    {
        constexpr int a[] = {(Cs::N * Cs::L)...};
        int m = 0;
        for (int i = 0; i < K; ++i) m = a[i] > m ? a[i] : m;
        return m;
    }
    static constexpr int TW = maxTW();
    static constexpr int len(int c)
    {
        constexpr int a[] = {Cs::N...};
        return a[c];
    }
    static constexpr int tile(int c)
    {
        constexpr int a[] = {Cs::L...};
        return a[c];
    }
    // the class of transform length n, or -1
    static constexpr int class_of(int n)
    {
        for (int c = 0; c < K; ++c)
            if (len(c) == n) return c;
        return -1;
    }
};

template <class T>
struct Tag {
    using type = T;
};

// call f(Tag<C_cls>{}) for the class `cls` of the pack
template <class C0, class... Cs, class Fn>
__device__ __forceinline__ void mix_dispatch(int cls, Fn &&f)
{
    if (cls == 0) {
        f(Tag<C0>{});
    } else if constexpr (sizeof...(Cs) > 0) {
        mix_dispatch<Cs...>(cls - 1, f);
    }
}

template <class... Cs>
struct MixDispatch;
template <class... Cs>
struct MixDispatch<MixFamily<Cs...>> {
    template <class Fn>
    static __device__ __forceinline__ void run(int cls, Fn &&f)
    {
        mix_dispatch<Cs...>(cls, f);
    }
};

template <class F>
constexpr size_t mix_col_smem() { return (size_t)F::TW * 24 + 16; }
template <class F>
constexpr size_t mix_row_smem() { return (size_t)F::TW * 28 + 24; }

// Column pass over a work list (classes: column-map tile configurations).
// Stages: two of P and sqrt(I), as in kp_col<C, FRESNEL, 2, false>; FresnelCDI
// items (a slot with phase factors) add the white field and the factors.
template <class F, bool FRESNEL>
__global__ void __launch_bounds__(F::NT, 1)
    kp_colm(const MixItem *__restrict__ items, const int *__restrict__ bounds,
            const Slot *const *slots, MixTw tws)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    constexpr int TW = F::TW;
    float2 *Pb0 = reinterpret_cast<float2 *>(smraw);
    float2 *Pb1 = Pb0 + TW;
    float *Mb0 = reinterpret_cast<float *>(Pb1 + TW);
    float *Mb1 = Mb0 + TW;
    uint64_t *bar = reinterpret_cast<uint64_t *>(Mb1 + TW);

    if (threadIdx.x == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();

    // this CTA's items: [t0, t1) of the list (ordered by class)
    const int t0 = bounds[blockIdx.x], t1 = bounds[blockIdx.x + 1];
    const MixItem first = items[t0 < t1 ? t0 : 0];
    const Slot &S0 = *slots[first.slot];
    const uint32_t polls = S0.wait_polls ? S0.wait_polls : kWaitPolls;
    const bool skip0 = S0.skip_first_load != 0;
    auto issue = [&](const MixItem &m, int b, bool skip) {
        const Slot &S = *slots[m.slot];
        MixDispatch<F>::run(m.cls, [&](auto tag) {
            using C = typename decltype(tag)::type;
            constexpr int tw = C::N * C::L;
            const size_t off = (size_t)m.tile * C::L * C::N;
            tma::mbar_arrive_expect_tx(&bar[b], tw * 12);
            if (skip) return;
            tma::bulk_load(b ? (void *)Pb1 : (void *)Pb0, S.P + off, tw * 8, &bar[b]);
            tma::bulk_load(b ? (void *)Mb1 : (void *)Mb0, S.mI + off, tw * 4, &bar[b]);
        });
    };
    int t = t0;
    if (threadIdx.x == 0 && t < t1) issue(items[t], 0, skip0);

    for (int it = 0; t < t1; ++it, ++t) {
        const int b = it & 1;
        const uint32_t par = (it >> 1) & 1;
        float2 *Pb = b ? Pb1 : Pb0;
        const float *Mb = b ? Mb1 : Mb0;
        const MixItem m = items[t];
        const Slot &S = *slots[m.slot];
        const int tn = t + 1;
        if (threadIdx.x == 0 && tn < t1) {
            tma::bulk_wait_read_all();
            issue(items[tn], b ^ 1, false);
        }
        const bool ok = tma::mbar_wait(&bar[b], par, polls);
        if (__syncthreads_or(!ok)) {
            // every copy issued so far lands before the CTA leaves
            if (threadIdx.x == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[b], par, polls);
                if (tn < t1) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        MixDispatch<F>::run(m.cls, [&](auto tag) {
            using C = typename decltype(tag)::type;
            constexpr int nx = C::N;
            const float2 *__restrict__ tw = tws.t[m.cls];
            const int c0 = m.tile * (C::L / kPanel);
            float2 v[C::E];
            for_each_slot<C, true, true>([&](int e, int s, int pos) { v[e] = Pb[raw_col<C>(s, pos)]; });
            __syncthreads();
            transform<C, true>(v, Pb, tw);
            const float s0 = S.s0;
            double diff = 0.0;
            for_each_slot<C, true, false>([&](int e, int s, int kx) {
                const float mm = Mb[raw_col<C>(s, kx)];
                float2 X = v[e];
                if (!FRESNEL) {
                    X = planar_modulus(X, mm, s0, diff);
                } else {
                    const int ky = c0 * kPanel + s;
                    const float2 cf = cmul(__ldg(&S.tx[kx]), __ldg(&S.ty[ky]));
                    const float2 w = __ldg(&S.W[paddr(kx, ky, nx)]);
                    const float2 u = modulus(cadd(cscale(cmul(cf, X), s0), w), mm, diff);
                    X = cscale(cmulc(csub(u, w), cf), s0);
                }
                v[e] = X;
            });
            const double tot = block_sum_seq<C::NT>(diff); // the order of kp_col
            if (threadIdx.x == 0) S.partials[m.tile] = tot;
            transform<C, false>(v, Pb, tw);
            for_each_slot<C, false, false>([&](int e, int s, int pos) { Pb[raw_col<C>(s, pos)] = v[e]; });
            tma::fence_async_shared();
            __syncthreads();
            if (threadIdx.x == 0) {
                tma::bulk_store(S.P + (size_t)m.tile * C::L * C::N, Pb, C::N * C::L * 8);
                tma::bulk_commit();
            }
        });
    }
    if (threadIdx.x == 0) tma::bulk_wait_all();
}

// Row pass over a work list (classes: row-map tile configurations; a row
// tile of class C holds C::L rows of length C::N = the grid's ny), as
// kp_row<C>: P through the reconstruction's tensor maps for C::L-row boxes,
// x and the support on their own barrier, the combine, x and P stored back.
// CTAs first finish the error metrics of the reconstructions in `slots`.
template <class F>
__global__ void __launch_bounds__(F::NT, 1)
    kp_rowm(const MixItem *__restrict__ items, const int *__restrict__ bounds,
            const Slot *const *slots, int nslots, MixTw tws)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    constexpr int TW = F::TW;
    float2 *Pb0 = reinterpret_cast<float2 *>(smraw);
    float2 *Pb1 = Pb0 + TW;
    float2 *Xb = Pb1 + TW;
    float *Sb = reinterpret_cast<float *>(Xb + TW);
    uint64_t *bar = reinterpret_cast<uint64_t *>(Sb + TW);

    if (threadIdx.x == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::mbar_init(&bar[2], 1);
        tma::fence_barrier_init();
    }
    for (int sl = blockIdx.x; sl < nslots; sl += gridDim.x) finish_error<F::NT>(*slots[sl]);
    __syncthreads();

    const int t0 = bounds[blockIdx.x], t1 = bounds[blockIdx.x + 1];
    const MixItem first = items[t0 < t1 ? t0 : 0];
    const Slot &S0 = *slots[first.slot];
    const uint32_t polls = S0.wait_polls ? S0.wait_polls : kWaitPolls;
    const bool skip0 = S0.skip_first_load != 0;
    auto issue_p = [&](const MixItem &m, int b, bool skip) {
        const Slot &S = *slots[m.slot];
        MixDispatch<F>::run(m.cls, [&](auto tag) {
            using C = typename decltype(tag)::type;
            constexpr int TM = tmap_index<C::L>();
            constexpr int npan = C::N / kPanel;
            const int boxp = box_panels(npan);
            float2 *dst = b ? Pb1 : Pb0;
            tma::mbar_arrive_expect_tx(&bar[b], C::N * C::L * 8);
            if (skip) return;
            for (int c = 0; c < npan; c += boxp)
                tma::tensor_load_3d(dst + (size_t)c * C::L * kPanel, &S.tm[TM][0], 0, m.tile * C::L,
                                    c, &bar[b]);
        });
    };
    auto issue_xs = [&](const MixItem &m) {
        const Slot &S = *slots[m.slot];
        MixDispatch<F>::run(m.cls, [&](auto tag) {
            using C = typename decltype(tag)::type;
            constexpr int TM = tmap_index<C::L>();
            constexpr int npan = C::N / kPanel;
            const int boxp = box_panels(npan);
            tma::mbar_arrive_expect_tx(&bar[2], C::N * C::L * 12);
            for (int c = 0; c < npan; c += boxp) {
                tma::tensor_load_3d(Xb + (size_t)c * C::L * kPanel, &S.tm[TM][1], 0, m.tile * C::L,
                                    c, &bar[2]);
                tma::tensor_load_3d(Sb + (size_t)c * C::L * kPanel, &S.tm[TM][2], 0, m.tile * C::L,
                                    c, &bar[2]);
            }
        });
    };
    int t = t0;
    if (threadIdx.x == 0 && t < t1) issue_p(items[t], 0, skip0);

    for (int it = 0; t < t1; ++it, ++t) {
        const int b = it & 1;
        float2 *Pb = b ? Pb1 : Pb0;
        const MixItem m = items[t];
        const Slot &S = *slots[m.slot];
        const int tn = t + 1;
        if (threadIdx.x == 0) {
            tma::bulk_wait_read_all();
            issue_xs(m);
            if (tn < t1) issue_p(items[tn], b ^ 1, false);
        }
        bool ok = tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
        if (__syncthreads_or(!ok)) {
            // every copy issued so far lands before the CTA leaves
            if (threadIdx.x == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
                tma::mbar_wait(&bar[2], it & 1, polls);
                if (tn < t1) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        bool failed = false;
        MixDispatch<F>::run(m.cls, [&](auto tag) {
            using C = typename decltype(tag)::type;
            constexpr int TM = tmap_index<C::L>();
            constexpr int npan = C::N / kPanel;
            const int boxp = box_panels(npan);
            const float2 *__restrict__ tw = tws.t[m.cls];
            float2 v[C::E];
            for_each_slot<C, false, true>([&](int e, int s, int pos) { v[e] = Pb[raw_row<C>(s, pos)]; });
            __syncthreads();
            transform<C, false>(v, Pb, tw);
            const bool ok2 = tma::mbar_wait(&bar[2], it & 1, polls);
            if (__syncthreads_or(!ok2)) {
                if (threadIdx.x == 0) {
                    raise_flag(S);
                    tma::mbar_wait(&bar[2], it & 1, polls);
                    if (tn < t1) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
                }
                failed = true;
                return;
            }
            const float wid = S.w_id, wpf = S.w_pf, wps = S.w_ps, wpsf = S.w_psf;
            const bool er = S.er;
            for_each_slot<C, false, false>([&](int e, int s, int pos) {
                const int a = raw_row<C>(s, pos);
                const float f = support_factor(Sb[a]);
                const float2 y = v[e];
                float2 xn;
                if (er) {
                    xn = cscale(y, f);
                } else {
                    const float2 xk = Xb[a];
                    xn = combine2(xk, y, f, wid, wpf, wps, wpsf);
                }
                Xb[a] = xn;
                v[e] = xn;
            });
            transform<C, true>(v, Pb, tw);
            for_each_slot<C, true, false>([&](int e, int s, int pos) { Pb[raw_row<C>(s, pos)] = v[e]; });
            tma::fence_async_shared();
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int c = 0; c < npan; c += boxp) {
                    tma::tensor_store_3d(&S.tm[TM][0], 0, m.tile * C::L, c, Pb + (size_t)c * C::L * kPanel);
                    tma::tensor_store_3d(&S.tm[TM][1], 0, m.tile * C::L, c, Xb + (size_t)c * C::L * kPanel);
                }
                tma::bulk_commit();
            }
        });
        if (failed) break;
    }
    if (threadIdx.x == 0) tma::bulk_wait_all();
}

} // namespace f32
} // namespace nadia
