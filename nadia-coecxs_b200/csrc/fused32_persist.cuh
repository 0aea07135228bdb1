// fused32_persist.cuh -- persistent, TMA-pipelined forms of the column and
// row passes.
//
// One CTA per SM loops over tiles.  While it transforms tile i, the tensor
// memory accelerator brings tile i+1 into the other shared-memory stage
// (cp.async.bulk completing on an mbarrier) and writes tile i-1 back
// (cp.async.bulk bulk-group stores), so HBM traffic overlaps the arithmetic.
//
//   column pass: a tile of L columns is one contiguous run of the panel
//     layout (N*L elements of P plus N*L of sqrt(I)): two plain bulk copies.
//   row pass: a tile of L rows is ny/K segments of K*L elements spaced nx*K
//     apart: a 3-D tensor map (K, nx, ny/K) with box (K, L, <=256) fetches it
//     in a few tensor copies; x and the support arrive the same way, on their
//     own barrier, while the inverse row transform runs.
//
// Every mbarrier wait is bounded (Slot::wait_polls, default kWaitPolls); on
// a timeout the CTA raises the slot's error flag, waits (bounded) for its
// copies in flight and leaves.
#pragma once

#include "tma.cuh"

namespace nadia {
namespace f32 {

constexpr uint32_t kWaitPolls = 1u << 24;

// raw shared-memory index of element (signal s, position pos) as the bulk
// copies lay a tile out: column tiles [panel][pos][kk], row tiles [panel][row][kk]
template <class C>
__device__ __forceinline__ int raw_col(int s, int pos)
{
    return ((s / kPanel) * C::N + pos) * kPanel + (s % kPanel);
}
template <class C>
__device__ __forceinline__ int raw_row(int s, int pos)
{
    return ((pos / kPanel) * C::L + s) * kPanel + (pos % kPanel);
}

__device__ __forceinline__ void raise_flag(const Slot &S)
{
    if (S.flag) atomicExch(S.flag, 1);
}

// STAGES = 2: tile i+1 loads while tile i is transformed.  STAGES = 1: one
// buffer per CTA (less shared memory, so two CTAs share an SM and each one's
// load overlaps the other's arithmetic); the next load is issued once the
// previous tile's store has read the buffer.
// MMODE (how sqrt(I) reaches the modulus):
//   0  staged with P in every stage;
//   1  not staged: each thread reads its values straight from global memory
//      (a warp reads 128 contiguous bytes), issued before the last pass of
//      the forward transform so that the loads overlap that pass;
//   2  one stage of its own (on mbarrier 2), refilled with the next tile's
//      values as soon as the current tile's modulus has read it, so that the
//      load overlaps the inverse transform and the next forward transform.
// C::PING: the exchanges alternate between the stage and one more tile
// buffer, one barrier per exchange instead of two.
// Shared memory: STAGES x P, sqrt(I) (STAGES, 0 or 1 tiles), [exchange
// buffer], 3 mbarriers.
template <class C, int STAGES, int MMODE>
constexpr size_t persist_col_bytes()
{
    return (size_t)C::N * C::L *
               (8 * STAGES + (MMODE == 0 ? 4 * STAGES : (MMODE == 2 ? 4 : 0)) + (C::PING ? 8 : 0)) +
           24;
}

template <class C, bool FRESNEL, int STAGES, int MMODE>
__global__ void __launch_bounds__(C::NT, C::MINB)
    kp_col(const Slot *const *slots, int nslots, int nx, int ny, const float2 *__restrict__ tw)
{
    static_assert(STAGES == 1 || STAGES == 2, "one or two stages");
    static_assert(MMODE != 2 || STAGES == 2, "a sqrt(I) stage of its own pairs with two P stages");
    constexpr bool MDIRECT = MMODE == 1;
    constexpr bool MSTAGE = MMODE == 2;
    extern __shared__ __align__(1024) unsigned char smraw[];
    __shared__ double wsum[C::NT / 32];
    constexpr int TW = C::N * C::L;
    float2 *Pb0 = reinterpret_cast<float2 *>(smraw);
    float2 *Pb1 = Pb0 + TW * (STAGES - 1);
    float *Mb0 = reinterpret_cast<float *>(Pb1 + TW);
    float *Mb1 = Mb0 + (MMODE == 0 ? TW * (STAGES - 1) : 0);
    float2 *Xb = reinterpret_cast<float2 *>(Mb1 + (MMODE == 1 ? 0 : TW)); // PING only
    uint64_t *bar = reinterpret_cast<uint64_t *>(Xb + (C::PING ? TW : 0));
    const int tps = ny / C::L;
    const int ntiles = tps * nslots;
    constexpr uint32_t kBytes = TW * (MMODE == 0 ? 12 : 8);

    if (threadIdx.x == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::mbar_init(&bar[2], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();

    // the first tile's reconstruction sets the wait limit (and the test hook
    // that leaves the first tile's copy unissued, see Slot::skip_first_load)
    const Slot &S0 = *slots[blockIdx.x / tps];
    const uint32_t polls = S0.wait_polls ? S0.wait_polls : kWaitPolls;
    const bool skip0 = S0.skip_first_load != 0;
    auto issue = [&](int tile, int b, bool skip) {
        const Slot &S = *slots[tile / tps];
        const size_t off = (size_t)(tile % tps) * C::L * nx;
        tma::mbar_arrive_expect_tx(&bar[b], kBytes);
        if (skip) return;
        tma::bulk_load(b ? (void *)Pb1 : (void *)Pb0, S.P + off, TW * 8, &bar[b]);
        if (MMODE == 0)
            tma::bulk_load(b ? (void *)Mb1 : (void *)Mb0, S.mI + off, TW * 4, &bar[b]);
    };
    auto issue_m = [&](int tile) { // MSTAGE: sqrt(I) of `tile` into its stage
        const Slot &S = *slots[tile / tps];
        tma::mbar_arrive_expect_tx(&bar[2], TW * 4);
        tma::bulk_load(Mb0, S.mI + (size_t)(tile % tps) * C::L * nx, TW * 4, &bar[2]);
    };
    int t = blockIdx.x;
    if (STAGES == 2 && threadIdx.x == 0 && t < ntiles) {
        issue(t, 0, skip0);
        if (MSTAGE) issue_m(t);
    }

    for (int it = 0; t < ntiles; ++it, t += gridDim.x) {
        const int b = STAGES == 2 ? (it & 1) : 0;
        const uint32_t par = STAGES == 2 ? ((it >> 1) & 1) : (it & 1);
        float2 *Pb = b ? Pb1 : Pb0;
        const float *Mb = b ? Mb1 : Mb0;
        const Slot &S = *slots[t / tps];
        const int c0 = (t % tps) * (C::L / kPanel);
        const int tn = t + gridDim.x;
        if (threadIdx.x == 0) {
            if (STAGES == 1) {
                tma::bulk_wait_read_all();
                issue(t, 0, it == 0 && skip0);
            } else if (tn < ntiles) {
                tma::bulk_wait_read_all();
                issue(tn, b ^ 1, false);
            }
        }
        const bool ok = tma::mbar_wait(&bar[b], par, polls);
        float2 v[C::E];
        float m[C::E];
        // (where the wait gave up these are stale values; the tile is dropped)
        for_each_slot<C, true, true>([&](int e, int s, int pos) { v[e] = Pb[raw_col<C>(s, pos)]; });
        // one barrier: the stage has been read (the first exchange writes it)
        // and every thread knows whether the wait gave up
        if (__syncthreads_or(!ok)) {
            // every copy issued so far lands before the CTA leaves
            if (threadIdx.x == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[b], par, polls);
                if (STAGES == 2 && tn < ntiles)
                    tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
                if (MSTAGE) tma::mbar_wait(&bar[2], it & 1, polls);
            }
            break;
        }
        const float *mg = S.mI + (size_t)(t % tps) * C::L * nx;
        transform_h<C, true>(v, Pb, Xb, tw, [&] {
            if (MDIRECT)
                for_each_slot<C, true, false>(
                    [&](int e, int s, int kx) { m[e] = __ldg(&mg[raw_col<C>(s, kx)]); });
        });

        if (MSTAGE) {
            const bool okm = tma::mbar_wait(&bar[2], it & 1, polls);
            if (__syncthreads_or(!okm)) {
                if (threadIdx.x == 0) {
                    raise_flag(S);
                    tma::mbar_wait(&bar[2], it & 1, polls);
                    if (tn < ntiles) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
                }
                break;
            }
        }
        const float s0 = S.s0;
        double diff = 0.0;
        for_each_slot<C, true, false>([&](int e, int s, int kx) {
            const float mm = MDIRECT ? m[e] : (MSTAGE ? Mb0 : Mb)[raw_col<C>(s, kx)];
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
        if (MSTAGE) {
            const double tot = block_sum<C::NT>(diff); // every thread has read sqrt(I)
            if (threadIdx.x == 0) {
                S.partials[t % tps] = tot;
                if (tn < ntiles) {
                    tma::fence_async_shared();
                    issue_m(tn);
                }
            }
        } else {
            // warp sums now; thread 0 adds them up after the barrier that
            // precedes the tile's store (no barrier of its own)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) diff += __shfl_down_sync(0xffffffffu, diff, off);
            if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = diff;
        }

        transform_h<C, false>(v, Pb, Xb, tw, [] {});
        for_each_slot<C, false, false>([&](int e, int s, int pos) { Pb[raw_col<C>(s, pos)] = v[e]; });
        tma::fence_async_shared();
        __syncthreads();
        if (threadIdx.x == 0) {
            tma::bulk_store(S.P + (size_t)(t % tps) * C::L * nx, Pb, TW * 8);
            tma::bulk_commit();
            if (!MSTAGE) {
                // the warps' sums in a fixed order; the next tile's writes
                // come after its first barrier, which thread 0 reaches later
                double tot = 0.0;
#pragma unroll
                for (int w = 0; w < C::NT / 32; ++w) tot += wsum[w];
                S.partials[t % tps] = tot;
            }
        }
    }
    if (threadIdx.x == 0) tma::bulk_wait_all();
}

// finish the error metric of the column pass for one slot (all threads)
template <int NT>
__device__ __forceinline__ void finish_error(const Slot &S)
{
    finish_error_row<NT>(S);
    __syncthreads();
}

template <int L>
__host__ __device__ constexpr int tmap_index()
{
    return L == 1 ? 0 : (L == 2 ? 1 : (L == 4 ? 2 : (L == 8 ? 3 : 4)));
}

template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB)
    kp_row(const Slot *const *slots, int nslots, int nx, int ny, const float2 *__restrict__ tw)
{
    extern __shared__ __align__(1024) unsigned char smraw[];
    constexpr int TW = C::N * C::L;
    constexpr int TM = tmap_index<C::L>();
    float2 *Pb0 = reinterpret_cast<float2 *>(smraw);
    float2 *Pb1 = Pb0 + TW;
    float2 *Xb = Pb1 + TW;
    float *Sb = reinterpret_cast<float *>(Xb + TW);
    uint64_t *bar = reinterpret_cast<uint64_t *>(Sb + TW);
    const int tps = nx / C::L;
    const int ntiles = tps * nslots;
    const int npan = ny / kPanel;
    const int boxp = box_panels(npan);

    if (threadIdx.x == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::mbar_init(&bar[2], 1);
        tma::fence_barrier_init();
    }
    // slots whose error this CTA finishes (the column pass ran before)
    for (int sl = blockIdx.x; sl < nslots; sl += gridDim.x) finish_error<C::NT>(*slots[sl]);
    __syncthreads();

    const Slot &S0 = *slots[blockIdx.x / tps];
    const uint32_t polls = S0.wait_polls ? S0.wait_polls : kWaitPolls;
    const bool skip0 = S0.skip_first_load != 0;
    auto issue_p = [&](int tile, int b, bool skip) {
        const Slot &S = *slots[tile / tps];
        const int i0 = (tile % tps) * C::L;
        float2 *dst = b ? Pb1 : Pb0;
        tma::mbar_arrive_expect_tx(&bar[b], TW * 8);
        if (skip) return;
        for (int c = 0; c < npan; c += boxp)
            tma::tensor_load_3d(dst + (size_t)c * C::L * kPanel, &S.tm[TM][0], 0, i0, c, &bar[b]);
    };
    auto issue_xs = [&](int tile) {
        const Slot &S = *slots[tile / tps];
        const int i0 = (tile % tps) * C::L;
        tma::mbar_arrive_expect_tx(&bar[2], TW * 12);
        for (int c = 0; c < npan; c += boxp) {
            tma::tensor_load_3d(Xb + (size_t)c * C::L * kPanel, &S.tm[TM][1], 0, i0, c, &bar[2]);
            tma::tensor_load_3d(Sb + (size_t)c * C::L * kPanel, &S.tm[TM][2], 0, i0, c, &bar[2]);
        }
    };
    int t = blockIdx.x;
    if (threadIdx.x == 0 && t < ntiles) issue_p(t, 0, skip0);

    for (int it = 0; t < ntiles; ++it, t += gridDim.x) {
        const int b = it & 1;
        float2 *Pb = b ? Pb1 : Pb0;
        const Slot &S = *slots[t / tps];
        const int i0 = (t % tps) * C::L;
        const int tn = t + gridDim.x;
        if (threadIdx.x == 0) {
            tma::bulk_wait_read_all();
            issue_xs(t);
            if (tn < ntiles) issue_p(tn, b ^ 1, false);
        }
        const bool ok = tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
        float2 v[C::E];
        // (where the wait gave up these are stale values; the tile is dropped)
        for_each_slot<C, false, true>([&](int e, int s, int pos) { v[e] = Pb[raw_row<C>(s, pos)]; });
        // one barrier: the stage has been read (the first exchange writes it)
        // and every thread knows whether the wait gave up
        if (__syncthreads_or(!ok)) {
            // every copy issued so far lands before the CTA leaves
            if (threadIdx.x == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
                tma::mbar_wait(&bar[2], it & 1, polls);
                if (tn < ntiles) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        transform<C, false>(v, Pb, tw);

        // x and the support; a wait that gave up is acted on at the barrier
        // before the store (the tile's values are dropped there)
        const bool okx = tma::mbar_wait(&bar[2], it & 1, polls);
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
        if (__syncthreads_or(!okx)) {
            if (threadIdx.x == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[2], it & 1, polls);
                if (tn < ntiles) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        if (threadIdx.x == 0) {
            for (int c = 0; c < npan; c += boxp) {
                tma::tensor_store_3d(&S.tm[TM][0], 0, i0, c, Pb + (size_t)c * C::L * kPanel);
                tma::tensor_store_3d(&S.tm[TM][1], 0, i0, c, Xb + (size_t)c * C::L * kPanel);
            }
            tma::bulk_commit();
        }
    }
    if (threadIdx.x == 0) tma::bulk_wait_all();
}

// OR of a predicate over the thread's group (the CTA when C::GROUPS == 1),
// which also synchronises the group
template <class C>
__device__ __forceinline__ bool group_or(bool v)
{
    if constexpr (C::GROUPS > 1) {
        uint32_t out;
        asm volatile("{\n\t.reg .pred p, q;\n\t"
                     "setp.ne.u32 p, %1, 0;\n\t"
                     "bar.red.or.pred q, %2, %3, p;\n\t"
                     "selp.u32 %0, 1, 0, q;\n\t}"
                     : "=r"(out)
                     : "r"((uint32_t)v), "r"(1 + (int)(threadIdx.x / C::NT)), "n"(C::NT)
                     : "memory");
        return out != 0;
    } else {
        return __syncthreads_or(v);
    }
}

// The row pass in C::GROUPS independent groups of C::NT threads.  Each group
// owns a quarter (or half) of the shared memory and runs the pipeline of
// kp_row on its own: its tiles of C::L rows (tile g, g + G, ... of the CTA's
// share), its own mbarriers, its own TMA issue thread (the group's first),
// and exchanges behind its own named barrier.  Nothing synchronises the
// groups after the error metrics are finished, so one group's barrier and
// load waits overlap the others' arithmetic.
template <class C>
constexpr size_t grouped_row_smem()
{
    return (size_t)C::GROUPS * ((size_t)C::N * C::L * 28 + 24);
}

template <class C>
__global__ void __launch_bounds__(C::NT * C::GROUPS, 1)
    kg_row(const Slot *const *slots, int nslots, int nx, int ny, const float2 *__restrict__ tw)
{
    static_assert(C::GROUPS > 1, "grouped tiles");
    constexpr int G = C::GROUPS;
    extern __shared__ __align__(1024) unsigned char smraw[];
    constexpr int TW = C::N * C::L;
    constexpr int TM = tmap_index<C::L>();
    const int g = threadIdx.x / C::NT, u = threadIdx.x % C::NT;
    float2 *Pb0 = reinterpret_cast<float2 *>(smraw + (size_t)g * TW * 28);
    float2 *Pb1 = Pb0 + TW;
    float2 *Xb = Pb1 + TW;
    float *Sb = reinterpret_cast<float *>(Xb + TW);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + (size_t)G * TW * 28) + 3 * g;
    const int tps = nx / C::L;
    const int ntiles = tps * nslots;
    const int npan = ny / kPanel;
    const int boxp = box_panels(npan);

    if (u == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::mbar_init(&bar[2], 1);
        tma::fence_barrier_init();
    }
    // slots whose error this CTA finishes (the column pass ran before)
    for (int sl = blockIdx.x; sl < nslots; sl += gridDim.x) finish_error<C::NT * G>(*slots[sl]);
    __syncthreads();

    int t = blockIdx.x * G + g;
    const int stride = gridDim.x * G;
    if (t >= ntiles) return; // a group without tiles (no CTA-wide barrier follows)
    const Slot &S0 = *slots[t / tps];
    const uint32_t polls = S0.wait_polls ? S0.wait_polls : kWaitPolls;
    const bool skip0 = S0.skip_first_load != 0;
    auto issue_p = [&](int tile, int b, bool skip) {
        const Slot &S = *slots[tile / tps];
        const int i0 = (tile % tps) * C::L;
        float2 *dst = b ? Pb1 : Pb0;
        tma::mbar_arrive_expect_tx(&bar[b], TW * 8);
        if (skip) return;
        for (int c = 0; c < npan; c += boxp)
            tma::tensor_load_3d(dst + (size_t)c * C::L * kPanel, &S.tm[TM][0], 0, i0, c, &bar[b]);
    };
    auto issue_xs = [&](int tile) {
        const Slot &S = *slots[tile / tps];
        const int i0 = (tile % tps) * C::L;
        tma::mbar_arrive_expect_tx(&bar[2], TW * 12);
        for (int c = 0; c < npan; c += boxp) {
            tma::tensor_load_3d(Xb + (size_t)c * C::L * kPanel, &S.tm[TM][1], 0, i0, c, &bar[2]);
            tma::tensor_load_3d(Sb + (size_t)c * C::L * kPanel, &S.tm[TM][2], 0, i0, c, &bar[2]);
        }
    };
    if (u == 0) issue_p(t, 0, skip0);

    for (int it = 0; t < ntiles; ++it, t += stride) {
        const int b = it & 1;
        float2 *Pb = b ? Pb1 : Pb0;
        const Slot &S = *slots[t / tps];
        const int i0 = (t % tps) * C::L;
        const int tn = t + stride;
        if (u == 0) {
            tma::bulk_wait_read_all();
            issue_xs(t);
            if (tn < ntiles) issue_p(tn, b ^ 1, false);
        }
        const bool ok = tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
        float2 v[C::E];
        // (where the wait gave up these are stale values; the tile is dropped)
        for_each_slot<C, false, true>([&](int e, int s, int pos) { v[e] = Pb[raw_row<C>(s, pos)]; });
        // one group barrier: the stage has been read (the first exchange
        // writes it) and the group knows whether the wait gave up
        if (group_or<C>(!ok)) {
            // every copy issued so far lands before the group leaves
            if (u == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
                tma::mbar_wait(&bar[2], it & 1, polls);
                if (tn < ntiles) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        transform<C, false>(v, Pb, tw);

        // x and the support; a wait that gave up is acted on at the barrier
        // before the store (the tile's values are dropped there)
        const bool okx = tma::mbar_wait(&bar[2], it & 1, polls);
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
        if (group_or<C>(!okx)) {
            if (u == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[2], it & 1, polls);
                if (tn < ntiles) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        if (u == 0) {
            for (int c = 0; c < npan; c += boxp) {
                tma::tensor_store_3d(&S.tm[TM][0], 0, i0, c, Pb + (size_t)c * C::L * kPanel);
                tma::tensor_store_3d(&S.tm[TM][1], 0, i0, c, Xb + (size_t)c * C::L * kPanel);
            }
            tma::bulk_commit();
        }
    }
    if (u == 0) tma::bulk_wait_all();
}

// FP64 sum over the thread's group; the result is valid in the group's
// first thread.  Synchronises the group.
template <class C>
__device__ __forceinline__ double group_sum(double v)
{
    __shared__ double red[C::GROUPS][C::NT / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int g = threadIdx.x / C::NT, u = threadIdx.x % C::NT;
    if ((u & 31) == 0) red[g][u >> 5] = v;
    C::sync();
    double t = 0;
    if (u == 0)
        for (int w = 0; w < C::NT / 32; ++w) t += red[g][w];
    return t;
}

// The column pass in C::GROUPS independent groups of C::NT threads: a group's
// tile is half a panel (two whole columns of length nx = C::N, C::L == 2).
// Per group: two stages of P (column pairs through the tensor map tc[0]),
// one stage of sqrt(I) (the tile's whole panel through tc[1], refilled for
// the next tile as soon as the modulus has read it), its own mbarriers, its
// own TMA issue thread and named-barrier exchanges.  Error partials are kept
// per half panel.
template <class C>
constexpr size_t grouped_col_smem()
{
    return (size_t)C::GROUPS * ((size_t)C::N * C::L * 16 + (size_t)C::N * 16) + 24 * C::GROUPS;
}

template <class C, bool FRESNEL>
__global__ void __launch_bounds__(C::NT * C::GROUPS, 1)
    kg_col(const Slot *const *slots, int nslots, int nx, int ny, const float2 *__restrict__ tw)
{
    static_assert(C::GROUPS > 1 && C::L == 2, "grouped tiles of two columns");
    constexpr int G = C::GROUPS;
    constexpr int TW = C::N * C::L;
    constexpr size_t GB = (size_t)TW * 16 + (size_t)C::N * 16;
    extern __shared__ __align__(1024) unsigned char smraw[];
    const int g = threadIdx.x / C::NT, u = threadIdx.x % C::NT;
    float2 *Pb0 = reinterpret_cast<float2 *>(smraw + (size_t)g * GB);
    float2 *Pb1 = Pb0 + TW;
    float *Mb = reinterpret_cast<float *>(Pb1 + TW);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smraw + (size_t)G * GB) + 3 * g;
    const int tps = ny / C::L; // half-panel tiles per reconstruction
    const int ntiles = tps * nslots;
    const int bx = box_rows(nx);

    if (u == 0) {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::mbar_init(&bar[2], 1);
        tma::fence_barrier_init();
    }
    __syncthreads();

    int t = blockIdx.x * G + g;
    const int stride = gridDim.x * G;
    if (t >= ntiles) return; // a group without tiles (no CTA-wide barrier follows)
    const Slot &S0 = *slots[t / tps];
    const uint32_t polls = S0.wait_polls ? S0.wait_polls : kWaitPolls;
    const bool skip0 = S0.skip_first_load != 0;
    auto issue_p = [&](int tile, int b, bool skip) {
        const Slot &S = *slots[tile / tps];
        const int tt = tile % tps, panel = tt >> 1, half = tt & 1;
        float2 *dst = b ? Pb1 : Pb0;
        tma::mbar_arrive_expect_tx(&bar[b], TW * 8);
        if (skip) return;
        for (int x0 = 0; x0 < nx; x0 += bx)
            tma::tensor_load_3d(dst + (size_t)x0 * 2, &S.tc[0], 2 * half, x0, panel, &bar[b]);
    };
    auto issue_m = [&](int tile) {
        const Slot &S = *slots[tile / tps];
        const int panel = (tile % tps) >> 1;
        tma::mbar_arrive_expect_tx(&bar[2], C::N * 16);
        for (int x0 = 0; x0 < nx; x0 += bx)
            tma::tensor_load_3d(Mb + (size_t)x0 * 4, &S.tc[1], 0, x0, panel, &bar[2]);
    };
    if (u == 0) {
        issue_p(t, 0, skip0);
        issue_m(t);
    }

    for (int it = 0; t < ntiles; ++it, t += stride) {
        const int b = it & 1;
        float2 *Pb = b ? Pb1 : Pb0;
        const Slot &S = *slots[t / tps];
        const int tt = t % tps, panel = tt >> 1, half = tt & 1;
        const int tn = t + stride;
        if (u == 0 && tn < ntiles) {
            tma::bulk_wait_read_all();
            issue_p(tn, b ^ 1, false);
        }
        bool ok = tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
        if (group_or<C>(!ok)) {
            // every copy issued so far lands before the group leaves
            if (u == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[b], (it >> 1) & 1, polls);
                tma::mbar_wait(&bar[2], it & 1, polls);
                if (tn < ntiles) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        float2 v[C::E];
        for_each_slot<C, true, true>([&](int e, int s, int pos) { v[e] = Pb[pos * 2 + s]; });
        C::sync();
        transform<C, true>(v, Pb, tw);

        ok = tma::mbar_wait(&bar[2], it & 1, polls);
        if (group_or<C>(!ok)) {
            if (u == 0) {
                raise_flag(S);
                tma::mbar_wait(&bar[2], it & 1, polls);
                if (tn < ntiles) tma::mbar_wait(&bar[b ^ 1], ((it + 1) >> 1) & 1, polls);
            }
            break;
        }
        const float s0 = S.s0;
        double diff = 0.0;
        for_each_slot<C, true, false>([&](int e, int s, int kx) {
            const float mm = Mb[kx * 4 + 2 * half + s];
            float2 X = v[e];
            if (!FRESNEL) {
                X = planar_modulus(X, mm, s0, diff);
            } else {
                const int ky = panel * kPanel + 2 * half + s;
                const float2 cf = cmul(__ldg(&S.tx[kx]), __ldg(&S.ty[ky]));
                const float2 w = __ldg(&S.W[paddr(kx, ky, nx)]);
                const float2 uu = modulus(cadd(cscale(cmul(cf, X), s0), w), mm, diff);
                X = cscale(cmulc(csub(uu, w), cf), s0);
            }
            v[e] = X;
        });
        const double tot = group_sum<C>(diff); // the group has read sqrt(I)
        if (u == 0) {
            S.partials[tt] = tot;
            if (tn < ntiles) {
                tma::fence_async_shared();
                issue_m(tn);
            }
        }
        transform<C, false>(v, Pb, tw);
        for_each_slot<C, false, false>([&](int e, int s, int pos) { Pb[pos * 2 + s] = v[e]; });
        tma::fence_async_shared();
        C::sync();
        if (u == 0) {
            for (int x0 = 0; x0 < nx; x0 += bx)
                tma::tensor_store_3d(&S.tc[0], 2 * half, x0, panel, Pb + (size_t)x0 * 2);
            tma::bulk_commit();
        }
    }
    if (u == 0) tma::bulk_wait_all();
}

} // namespace f32
} // namespace nadia
