// fused32_wf.cuh -- the FP32 form of FresnelCDI_WF::iterate
// (FresnelCDI_WF.c++:122-182) as one column pass and one row pass.
//
// One reference iteration takes the detector-plane field c through four
// unnormalised 2-D transforms:
//
//   c1 = IDFT2(c); c2 = swap(c1) s; c3 = c2 B          propagate_from_detector
//   c4 = IDFT2(c3); c5 = c4 support                     apply_support
//   c6 = DFT2(c5); c7 = c6 F; c8 = swap(c7) s; c9 = DFT2(c8)   propagate_to_detector
//   c10 = c9 with |c9| set to sqrt(I) (measured pixels)  scale_intensity
//
// with s = 1/sqrt(nx ny), swap the quadrant swap of Complex_2D::invert and
// B = -i s e^{i phi}, F = +i s e^{-i phi} (multiply_factors, BACKWARD and
// FORWARD), phi = phi_x(i) + phi_y(j) separable.  So:
//   * the constant phases -i and +i cancel within an iteration (the support
//     and the modulus commute with a constant phase) and are left out;
//   * each factor splits into per-axis tables b_x(k) = e^{i phi_x(k)} / nx and
//     b_y(k) = e^{i phi_y(k)} / ny (Slot::tx, ty), F's being their conjugates;
//   * the swaps become signs: swapping after a transform is the transform of
//     the (-1)^n-modulated input, swapping before it modulates the output by
//     (-1)^k.  Both swaps of an iteration then meet at the modulus as the one
//     sign (-1)^(i+j): the passes carry c' = (-1)^(i+j) c, the modulus keeps
//     the magnitude (and writes sg (sqrt(I), 0) where c' = 0), and the
//     estimate x is written back as (-1)^(i+j) c';
//   * transforms along one axis commute with factors and signs of the other,
//     so an iteration is a column pass (x axis: inverse, b_x, inverse,
//     support, forward, conj(b_x), forward) and a row pass (y axis: forward,
//     conj(b_y), forward, modulus, inverse, b_y, inverse).  The row pass ends
//     one iteration and starts the next one; P carries the field between the
//     passes, and a prime (the second half of the row pass, from x) starts it.
//
// Consecutive transforms of one pass alternate in direction as the register
// tiles need them (a forward transform leaves each thread holding the inputs
// of an inverse one and vice versa); a transform of the other direction is
// taken as conj(T(conj v)), so every factor step is v <- conj(v) b, and the
// stored field is the true one.
#pragma once

namespace nadia {
namespace f32 {

// conj(v) * b
__device__ __forceinline__ float2 conj_mul(float2 v, float2 b) { return cmulc(b, v); }

// BaseCDI::scale_intensity (BaseCDI.c++:163-189) with Complex_2D::set_mag
// (Complex_2D.h:205-215) on c' = sg c: the magnitude ratio is sign-blind,
// the zero case writes sg (m, 0); (|c| - m)^2 of measured pixels to diff
__device__ __forceinline__ float2 wf_modulus(float2 c, float m, float sg, double &diff)
{
    if (m < 0.f) return c; // unmeasured: kept
    const float a2 = c.x * c.x + c.y * c.y;
    const bool zero = !(a2 > 0.f);
    const float inv = rsqrt_normal(a2);
    const float mag = a2 * inv;
    const float d = mag - m;
    diff = fma((double)d, (double)d, diff);
    if (zero) return make_float2(sg * m, 0.f);
    const float sc = m * inv;
    return make_float2(c.x * sc, c.y * sc);
}

// column pass: tiles of L columns (y = blockIdx.x*L + s), signals along x
template <class C>
__global__ void __launch_bounds__(C::NT, C::MINB) k_wf_col(const Slot *const *slots, int nx, int ny,
                                                  const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    const float2 *__restrict__ bx = S.tx;
    const float *__restrict__ sup = S.sup;
    const int y0 = blockIdx.x * C::L;
    float2 v[C::E];
    // inverse transform as conj(F(conj v))
    for_each_slot<C, true, true>([&](int e, int s, int i) {
        const float2 a = P[paddr(i, y0 + s, nx)];
        v[e] = make_float2(a.x, -a.y);
    });
    transform<C, true>(v, sm, tw);
    for_each_slot<C, true, false>([&](int e, int, int k) { v[e] = conj_mul(v[e], __ldg(&bx[k])); });
    transform<C, false>(v, sm, tw);
    // c4 -> c5: BaseCDI::support_constraint (BaseCDI.c++:136-154)
    for_each_slot<C, false, false>([&](int e, int s, int i) {
        v[e] = cscale(v[e], support_factor(__ldg(&sup[paddr(i, y0 + s, nx)])));
    });
    transform<C, true>(v, sm, tw);
    // times conj(b_x), then the forward transform as conj(I(conj v))
    for_each_slot<C, true, false>([&](int e, int, int k) { v[e] = conj_mul(v[e], __ldg(&bx[k])); });
    transform<C, false>(v, sm, tw);
    for_each_slot<C, false, false>([&](int e, int s, int i) {
        P[paddr(i, y0 + s, nx)] = make_float2(v[e].x, -v[e].y);
    });
}

// row pass: tiles of L rows (x = blockIdx.x*L + s), signals along y.
// kRowFull: the end of an iteration (the y-axis half of propagate_to_detector,
// the modulus, x written, error partial per tile) and the y-axis half of the
// next propagate_from_detector; kRowPrime: that second half only, from x.
template <class C, int MODE>
__global__ void __launch_bounds__(C::NT, C::MINB) k_wf_row(const Slot *const *slots, int nx, int ny,
                                                  const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    float2 *__restrict__ x = S.x;
    const float2 *__restrict__ by = S.ty;
    const int i0 = blockIdx.x * C::L;
    float2 v[C::E];
    if (MODE == kRowFull) {
        for_each_slot<C, true, true>([&](int e, int s, int j) { v[e] = P[paddr(i0 + s, j, nx)]; });
        transform<C, true>(v, sm, tw);
        for_each_slot<C, true, false>([&](int e, int, int k) { v[e] = conj_mul(v[e], __ldg(&by[k])); });
        transform<C, false>(v, sm, tw);
        const float *__restrict__ mI = S.mI;
        double diff = 0.0;
        for_each_slot<C, false, false>([&](int e, int s, int j) {
            const size_t a = paddr(i0 + s, j, nx);
            const float sg = ((i0 + s + j) & 1) ? -1.f : 1.f;
            const float2 c = wf_modulus(make_float2(v[e].x, -v[e].y), __ldg(&mI[a]), sg, diff);
            x[a] = make_float2(sg * c.x, sg * c.y);
            v[e] = make_float2(c.x, -c.y); // the next inverse transform as conj(F(conj v))
        });
        const double tot = block_sum<C::NT>(diff);
        if (threadIdx.x == 0) S.partials[blockIdx.x] = tot;
    } else {
        for_each_slot<C, true, true>([&](int e, int s, int j) {
            const float2 c = x[paddr(i0 + s, j, nx)];
            const float sg = ((i0 + s + j) & 1) ? -1.f : 1.f;
            v[e] = make_float2(sg * c.x, -sg * c.y);
        });
    }
    transform<C, true>(v, sm, tw);
    for_each_slot<C, true, false>([&](int e, int, int k) { v[e] = conj_mul(v[e], __ldg(&by[k])); });
    transform<C, false>(v, sm, tw);
    for_each_slot<C, false, false>([&](int e, int s, int j) { P[paddr(i0 + s, j, nx)] = v[e]; });
}

// the error metric of the row pass that just ran, one block per slot
// (S.ncol = the row tiles whose partials it sums)
template <int NT>
__global__ void __launch_bounds__(NT) k_wf_finish(const Slot *const *slots)
{
    finish_error_row<NT>(*slots[blockIdx.x]);
}

} // namespace f32
} // namespace nadia
