// fused32_tc.cuh -- TransmissionConstraint's complex-constraint regions
// (TransmissionConstraint.c++:76-172) in the FP32 form.
//
// A region's update needs c_mean = sum |ln|t|| / sum |arg t| over the region
// of the very field it updates, so the row pass splits in two around the
// sums: the first half inverse-transforms the rows into Y; the sums kernel
// reads the support-projected fields (Ps x, and Ps Y for the projection)
// and writes fixed-order FP64 partials per block and region; a one-block-
// per-region kernel forms c_mean; the second half applies region update,
// charge flipping and unit magnitude to each projected field inside the
// combine, writes x and forward-transforms the rows.  FresnelCDI's fields
// are transmission functions T = (z + L) / L of the projected z.  The sums
// and c_mean kernels (one instance, in fused32.cu) follow the same plan.
#pragma once

namespace nadia {
namespace f32 {

constexpr int kTcBlocks = 296;  // sums blocks per field (2 per SM)
constexpr int kTcThreads = 256;
constexpr int kTcMaxRegions = 16;

// FresnelCDI::get_transmission_function's T = (z + L)/L (1 where L = 0)
__device__ __forceinline__ float2 tc_to_t(float2 z, float2 l)
{
    const float denom = l.x * l.x + l.y * l.y;
    if (denom == 0.f) return make_float2(1.f, 0.f);
    const float rn = l.x * (z.x + l.x) + l.y * (z.y + l.y);
    const float in = l.x * (z.y + l.y) - l.y * (z.x + l.x);
    return make_float2(rn / denom, in / denom);
}

// ComplexConstraint's update of one pixel (TransmissionConstraint.c++:136-150):
// new magnitude exp((1-a1) ln|t| + a1 c arg t), new phase (1-a2) arg t +
// a2 ln|t| / c, set as Complex_2D::set_mag then set_phase (which keeps the
// magnitude just set)
__device__ __forceinline__ float2 tc_region_update(float2 v, const float *par, float cm)
{
    const float mag_old = sqrtf(v.x * v.x + v.y * v.y);
    const float phase_old = atan2f(v.y, v.x);
    const float lm = logf(mag_old);
    const float mag_new = expf((1.f - par[0]) * lm + par[0] * cm * phase_old);
    const float phase_new = (1.f - par[1]) * phase_old + par[1] * lm / cm;
    if (mag_old == 0.f) {
        v = make_float2(mag_new, 0.f);
    } else {
        const float q = mag_new / mag_old;
        v = make_float2(v.x * q, v.y * q);
    }
    const float m = sqrtf(v.x * v.x + v.y * v.y);
    float sn, cs;
    sincosf(phase_new, &sn, &cs);
    return make_float2(m * cs, m * sn);
}

// the constraint on a support-projected value z at panel address a, column
// yy, as field `field` (its c_mean): on z itself, or for FresnelCDI on its
// transmission function, written back as L T - L for columns below nx
// (set_transmission_function's bound, FresnelCDI.c++:271)
__device__ __forceinline__ float2 tc_apply(float2 z, const Slot &S, size_t a, int yy, int nx,
                                           int ny, int field)
{
    const int r = S.tc_R > 0 ? S.tc_region[a] : 0;
    if (!S.tc_ill) {
        if (r > 0) z = tc_region_update(z, S.tc_par + 4 * (r - 1), S.tc_cm[field * S.tc_R + r - 1]);
        return tc_pixel(z, S);
    }
    if (ny >= nx && yy >= nx) return z;
    const float2 l = S.tc_ill[a];
    float2 t = tc_to_t(z, l);
    if (r > 0) t = tc_region_update(t, S.tc_par + 4 * (r - 1), S.tc_cm[field * S.tc_R + r - 1]);
    t = tc_pixel(t, S);
    return make_float2(l.x * t.x - l.y * t.y - l.x, l.x * t.y + l.y * t.x - l.y);
}

// the value field `field` holds at panel address a: 0 = Ps x, 1 = Ps Y (the
// projection's rows inverse-transformed), as transmission functions for
// FresnelCDI (no column bound: the reference forms T everywhere); 2 = arr[a]
__device__ __forceinline__ float2 tc_field(const Slot &S, size_t a, int field, const float2 *arr)
{
    if (field == 2) return arr[a];
    const float f = support_factor(__ldg(&S.sup[a]));
    const float2 v = field == 0 ? S.x[a] : S.Y[a];
    const float2 z = make_float2(f * v.x, f * v.y);
    return S.tc_ill ? tc_to_t(z, S.tc_ill[a]) : z;
}

// The row pass in two halves around the region sums.  HALF 1: the column
// pass's error metric (block 0 of each slot), then the inverse row
// transforms into Y.  HALF 2: Y back into the same registers, the combine of
// k_row with the whole constraint on each support-projected field (Ps x as
// field 0, Ps Pf x as field 1), x written, forward row transforms to P.
template <class C, int HALF>
__global__ void __launch_bounds__(C::NT, C::MINB) k_row_tc(const Slot *const *slots, int nx, int ny,
                                                  const float2 *__restrict__ tw)
{
    extern __shared__ float2 sm[];
    const Slot &S = *slots[blockIdx.y];
    float2 *__restrict__ P = S.P;
    float2 *__restrict__ Y = S.Y;
    const int i0 = blockIdx.x * C::L;
    float2 v[C::E];
    if (HALF == 1) {
        if (blockIdx.x == 0) finish_error_row<C::NT>(S);
        for_each_slot<C, false, true>([&](int e, int s, int pos) {
            v[e] = P[paddr(i0 + s, pos, nx)];
        });
        transform<C, false>(v, sm, tw);
        for_each_slot<C, false, false>([&](int e, int s, int pos) {
            Y[paddr(i0 + s, pos, nx)] = v[e];
        });
        return;
    }
    float2 *__restrict__ x = S.x;
    const float *__restrict__ sup = S.sup;
    const float wid = S.w_id, wpf = S.w_pf, wps = S.w_ps, wpsf = S.w_psf;
    const bool er = S.er;
    for_each_slot<C, false, false>([&](int e, int s, int pos) {
        const size_t a = paddr(i0 + s, pos, nx);
        const float f = support_factor(__ldg(&sup[a]));
        const float2 y = Y[a];
        float2 xn;
        if (er) {
            xn = tc_apply(cscale(y, f), S, a, pos, nx, ny, 1);
        } else {
            const float2 xk = x[a];
            const float2 ps = tc_apply(cscale(xk, f), S, a, pos, nx, ny, 0);
            const float2 psf = tc_apply(cscale(y, f), S, a, pos, nx, ny, 1);
            xn = make_float2(wid * xk.x + wpf * y.x + wps * ps.x + wpsf * psf.x,
                             wid * xk.y + wpf * y.y + wps * ps.y + wpsf * psf.y);
        }
        x[a] = xn;
        v[e] = xn;
    });
    transform<C, true>(v, sm, tw);
    for_each_slot<C, true, false>([&](int e, int s, int pos) {
        P[paddr(i0 + s, pos, nx)] = v[e];
    });
}

} // namespace f32
} // namespace nadia
