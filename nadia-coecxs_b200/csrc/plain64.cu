// plain64.cu -- kernels of the plain FP64 path (see plain64.h).  Compiled
// with --fmad=false: every product and sum below rounds separately, as in
// the reference's double build compiled without contraction.
#include "plain64.h"

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace nadia {
namespace plain {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(size_t n, int per = kThreads)
{
    size_t b = (n + per - 1) / per;
    return (int)std::min<size_t>(std::max<size_t>(b, 1), 1u << 30);
}

__device__ __forceinline__ double2 cmul(double2 a, double2 w)
{
    return make_double2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}

__device__ __forceinline__ void bf4(double2 *v, bool fwd)
{
    double2 a, b, c, d;
    a.x = v[0].x + v[2].x; a.y = v[0].y + v[2].y;
    b.x = v[0].x - v[2].x; b.y = v[0].y - v[2].y;
    c.x = v[1].x + v[3].x; c.y = v[1].y + v[3].y;
    d.x = v[1].x - v[3].x; d.y = v[1].y - v[3].y;
    v[0].x = a.x + c.x; v[0].y = a.y + c.y;
    v[2].x = a.x - c.x; v[2].y = a.y - c.y;
    if (fwd) {
        v[1].x = b.x + d.y; v[1].y = b.y - d.x;
        v[3].x = b.x - d.y; v[3].y = b.y + d.x;
    } else {
        v[1].x = b.x - d.y; v[1].y = b.y + d.x;
        v[3].x = b.x + d.y; v[3].y = b.y - d.x;
    }
}

__device__ __forceinline__ void bf8(double2 *v, bool fwd)
{
    const double c8 = 0.70710678118654752440;
    double2 a[4], b[4], t;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        a[r].x = v[r].x + v[r + 4].x; a[r].y = v[r].y + v[r + 4].y;
        b[r].x = v[r].x - v[r + 4].x; b[r].y = v[r].y - v[r + 4].y;
    }
    if (fwd) {
        t = b[1]; b[1].x = (t.x + t.y) * c8; b[1].y = (t.y - t.x) * c8;
        t = b[2]; b[2].x = t.y;              b[2].y = -t.x;
        t = b[3]; b[3].x = (t.y - t.x) * c8; b[3].y = -((t.x + t.y) * c8);
    } else {
        t = b[1]; b[1].x = (t.x - t.y) * c8; b[1].y = (t.y + t.x) * c8;
        t = b[2]; b[2].x = -t.y;             b[2].y = t.x;
        t = b[3]; b[3].x = -((t.x + t.y) * c8); b[3].y = (t.x - t.y) * c8;
    }
    bf4(a, fwd);
    bf4(b, fwd);
#pragma unroll
    for (int r = 0; r < 4; ++r) { v[2 * r] = a[r]; v[2 * r + 1] = b[r]; }
}

// One Stockham pass of radix R (compile-time for 2/4/8) over L signals of
// length n held in shared memory (signal stride n).
template <int R>
__device__ void pass_fixed(const double2 *src, double2 *dst, int n, int L, int Ns,
                           const double2 *__restrict__ W, bool fwd)
{
    const int m = n / R;
    const int tstep = n / (Ns * R);
    for (int b = threadIdx.x; b < L * m; b += blockDim.x) {
        const int sig = b / m, j = b - sig * m;
        const double2 *s = src + (size_t)sig * n;
        double2 *d = dst + (size_t)sig * n;
        const int k = j % Ns;
        double2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = s[j + r * m];
        if (k > 0) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                double2 w = __ldg(&W[k * r * tstep]);
                if (!fwd) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        if (R == 2) {
            double2 a = v[0], c = v[1];
            v[0].x = a.x + c.x; v[0].y = a.y + c.y;
            v[1].x = a.x - c.x; v[1].y = a.y - c.y;
        } else if (R == 4) {
            bf4(v, fwd);
        } else {
            bf8(v, fwd);
        }
        const int base = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) d[base + r * Ns] = v[r];
    }
}

// Generic (prime) radix: direct sum in increasing r.
__device__ void pass_generic(const double2 *src, double2 *dst, int n, int L, int R, int Ns,
                             const double2 *__restrict__ W, bool fwd)
{
    const int m = n / R;
    const int tstep = n / (Ns * R);
    const int q = n / R;
    for (int b = threadIdx.x; b < L * m; b += blockDim.x) {
        const int sig = b / m, j = b - sig * m;
        const double2 *s = src + (size_t)sig * n;
        double2 *d = dst + (size_t)sig * n;
        const int k = j % Ns;
        if (R > kMaxRadix) {
            // large primes: the same sums, each twiddled input formed again
            // from shared memory where it is used (identical arithmetic)
            auto in = [&](int r) {
                double2 x = s[j + r * m];
                if (k > 0 && r > 0) {
                    double2 w = __ldg(&W[k * r * tstep]);
                    if (!fwd) w.y = -w.y;
                    x = cmul(x, w);
                }
                return x;
            };
            const int base = (j / Ns) * Ns * R + k;
            double2 y0 = in(0);
            for (int r = 1; r < R; ++r) {
                const double2 x = in(r);
                y0.x = y0.x + x.x;
                y0.y = y0.y + x.y;
            }
            double2 *out0 = d + base;
            for (int sidx = 1; sidx < R; ++sidx) {
                double2 acc = in(0);
                for (int r = 1; r < R; ++r) {
                    double2 w = __ldg(&W[((r * sidx) % R) * q]);
                    if (!fwd) w.y = -w.y;
                    double2 pp = cmul(in(r), w);
                    acc.x = acc.x + pp.x;
                    acc.y = acc.y + pp.y;
                }
                out0[sidx * Ns] = acc;
            }
            out0[0] = y0;
            continue;
        }
        double2 v[kMaxRadix];
        for (int r = 0; r < R; ++r) v[r] = s[j + r * m];
        if (k > 0) {
            for (int r = 1; r < R; ++r) {
                double2 w = __ldg(&W[k * r * tstep]);
                if (!fwd) w.y = -w.y;
                v[r] = cmul(v[r], w);
            }
        }
        const int base = (j / Ns) * Ns * R + k;
        double2 y0 = v[0];
        for (int r = 1; r < R; ++r) { y0.x = y0.x + v[r].x; y0.y = y0.y + v[r].y; }
        d[base] = y0;
        for (int sidx = 1; sidx < R; ++sidx) {
            double2 acc = v[0];
            for (int r = 1; r < R; ++r) {
                double2 w = __ldg(&W[((r * sidx) % R) * q]);
                if (!fwd) w.y = -w.y;
                double2 p = cmul(v[r], w);
                acc.x = acc.x + p.x; acc.y = acc.y + p.y;
            }
            d[base + sidx * Ns] = acc;
        }
    }
}

// All passes of a plan; returns the buffer holding the result.
__device__ double2 *run_passes(double2 *a, double2 *b, int L, const FftPlan &p,
                               const double2 *__restrict__ W, bool fwd)
{
    int Ns = 1;
    for (int ip = 0; ip < p.np; ++ip) {
        const int R = p.radix[ip];
        if (R == 8)
            pass_fixed<8>(a, b, p.n, L, Ns, W, fwd);
        else if (R == 4)
            pass_fixed<4>(a, b, p.n, L, Ns, W, fwd);
        else if (R == 2)
            pass_fixed<2>(a, b, p.n, L, Ns, W, fwd);
        else
            pass_generic(a, b, p.n, L, R, Ns, W, fwd);
        __syncthreads();
        Ns *= R;
        double2 *t = a; a = b; b = t;
    }
    return a;
}

__global__ void k_fft_rows(double2 *data, int nx, int ny, int rows, FftPlan p,
                           const double2 *__restrict__ W, bool fwd)
{
    extern __shared__ double2 sm[];
    double2 *a = sm, *b = sm + (size_t)rows * ny;
    const int r0 = blockIdx.x * rows;
    const int nr = min(rows, nx - r0);
    double2 *g = data + (size_t)r0 * ny;
    for (int e = threadIdx.x; e < nr * ny; e += blockDim.x) a[e] = g[e];
    __syncthreads();
    double2 *res = run_passes(a, b, nr, p, W, fwd);
    for (int e = threadIdx.x; e < nr * ny; e += blockDim.x) g[e] = res[e];
}

__global__ void k_fft_cols(double2 *data, int nx, int ny, int cols, FftPlan p,
                           const double2 *__restrict__ W, bool fwd)
{
    extern __shared__ double2 sm[];
    double2 *a = sm, *b = sm + (size_t)cols * nx;
    const int c0 = blockIdx.x * cols;
    const int nc = min(cols, ny - c0);
    for (int e = threadIdx.x; e < nc * nx; e += blockDim.x) {
        int i = e / nc, c = e - i * nc;
        a[(size_t)c * nx + i] = data[(size_t)i * ny + c0 + c];
    }
    __syncthreads();
    double2 *res = run_passes(a, b, nc, p, W, fwd);
    for (int e = threadIdx.x; e < nc * nx; e += blockDim.x) {
        int i = e / nc, c = e - i * nc;
        data[(size_t)i * ny + c0 + c] = res[(size_t)c * nx + i];
    }
}

__global__ void k_invert(double2 *a, int nx, int ny, double s)
{
    const int mx = nx / 2, my = ny / 2;
    const size_t total = (size_t)nx * my;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e / my), j = (int)(e - (size_t)i * my);
        int jn = j + my, in = i + mx;
        if (i >= mx) in = in - 2 * mx;
        double2 *pp = a + (size_t)in * ny + jn, *qq = a + (size_t)i * ny + j;
        double2 t = *pp, u = *qq;
        *pp = make_double2(u.x * s, u.y * s);
        *qq = make_double2(t.x * s, t.y * s);
    }
}

// Block sum of two doubles with a fixed tree; thread 0 gets the result.
__device__ void block_sum2(double &a, double &b)
{
    __shared__ double sa[kThreads], sb[kThreads];
    sa[threadIdx.x] = a;
    sb[threadIdx.x] = b;
    __syncthreads();
    for (int off = kThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            sa[threadIdx.x] += sa[threadIdx.x + off];
            sb[threadIdx.x] += sb[threadIdx.x + off];
        }
        __syncthreads();
    }
    a = sa[0];
    b = sb[0];
}

__device__ __forceinline__ double mag_of(double2 c) { return sqrt(c.x * c.x + c.y * c.y); }

__device__ __forceinline__ double2 set_mag(double2 c, double value)
{
    double mag = mag_of(c);
    if (mag == 0) return make_double2(value, 0.0);
    double q = value / mag;
    return make_double2(c.x * q, c.y * q);
}

__global__ void k_scale_intensity(double2 *c, const double *__restrict__ isqrt,
                                  const double *__restrict__ bs, size_t n, double *partials)
{
    double diff = 0, mag = 0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        if (bs == nullptr || bs[k] > 0) {
            double cis = isqrt[k];
            double2 v = c[k];
            double cm = mag_of(v);
            c[k] = set_mag(v, cis);
            mag += cis * cis;
            diff += (cm - cis) * (cm - cis);
        }
    }
    block_sum2(diff, mag);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = diff;
        partials[2 * blockIdx.x + 1] = mag;
    }
}

__global__ void k_finish_error(const double *partials, int nblocks, double *err)
{
    double diff = 0, mag = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        diff += partials[2 * b];
        mag += partials[2 * b + 1];
    }
    block_sum2(diff, mag);
    if (threadIdx.x == 0) *err = (diff / mag);
}

__global__ void k_support(double2 *c, const double *__restrict__ sup, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double sv = sup[k];
        if (sv == 0) {
            c[k] = make_double2(0.0, 0.0);
        } else if (sv < 1) {
            double2 v = c[k];
            c[k] = make_double2(v.x * sv, v.y * sv);
        }
    }
}

struct Weights { double w[5]; double id; };

__global__ void k_combine(double2 *x, const double2 *__restrict__ pfs,
                          const double2 *__restrict__ pf, const double2 *__restrict__ ps,
                          const double2 *__restrict__ psf, Weights W, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double2 v = x[k];
        double vr = W.id * v.x, vi = W.id * v.y;
        if (pfs) { double2 t = pfs[k]; vr += W.w[1] * t.x; vi += W.w[1] * t.y; }
        if (pf) { double2 t = pf[k]; vr += W.w[3] * t.x; vi += W.w[3] * t.y; }
        if (ps) { double2 t = ps[k]; vr += W.w[2] * t.x; vi += W.w[2] * t.y; }
        if (psf) { double2 t = psf[k]; vr += W.w[0] * t.x; vi += W.w[0] * t.y; }
        x[k] = make_double2(vr, vi);
    }
}

// k_support's operation on one value
__device__ __forceinline__ double2 supported(double2 v, double sv)
{
    if (sv == 0) return make_double2(0.0, 0.0);
    if (sv < 1) return make_double2(v.x * sv, v.y * sv);
    return v;
}

// The combine loop with the support projections formed on the fly (no
// transmission constraint, no PfPs term): Ps x = support(x), PsPf x =
// support(Pf x); the same sums in the same order as copying, projecting and
// combining separately.
__global__ void k_combine_support(double2 *x, const double2 *__restrict__ pf,
                                  const double *__restrict__ sup, int use_ps, int use_psf,
                                  Weights W, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const double2 v = x[k];
        const double sv = sup[k];
        double vr = W.id * v.x, vi = W.id * v.y;
        double2 f = make_double2(0.0, 0.0);
        if (pf) {
            f = pf[k];
            vr += W.w[3] * f.x;
            vi += W.w[3] * f.y;
        }
        if (use_ps) {
            const double2 t = supported(v, sv);
            vr += W.w[2] * t.x;
            vi += W.w[2] * t.y;
        }
        if (use_psf) {
            const double2 t = supported(f, sv);
            vr += W.w[0] * t.x;
            vi += W.w[0] * t.y;
        }
        x[k] = make_double2(vr, vi);
    }
}

// PlanarCDI's detector side of project_intensity (PlanarCDI.c++:65-73 around
// BaseCDI::scale_intensity, BaseCDI.c++:163-189) between the two transforms:
// invert(scale) -> scale_intensity -> invert(scale).  The quadrant swap pairs
// q with p(q), so per element out[q] = s * set_mag(s * a[q], sqrt(I)[p(q)])
// (measured pixels; s * (s * a[q]) otherwise) -- the same operations.
__global__ void k_detector_planar(double2 *c, const double *__restrict__ isqrt,
                                  const double *__restrict__ bs, int nx, int ny, double s,
                                  double *partials)
{
    double diff = 0, mag = 0;
    const int mx = nx / 2, my = ny / 2;
    const size_t n = (size_t)nx * ny;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n;
         q += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(q / ny), j = (int)(q - (size_t)i * ny);
        const int ip = i < mx ? i + mx : i - mx, jp = j < my ? j + my : j - my;
        const size_t d = (size_t)ip * ny + jp;
        const double2 u = c[q];
        double2 v = make_double2(u.x * s, u.y * s);
        if (bs == nullptr || bs[d] > 0) {
            const double cis = isqrt[d];
            const double cm = mag_of(v);
            v = set_mag(v, cis);
            mag += cis * cis;
            diff += (cm - cis) * (cm - cis);
        }
        c[q] = make_double2(v.x * s, v.y * s);
    }
    block_sum2(diff, mag);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = diff;
        partials[2 * blockIdx.x + 1] = mag;
    }
}

// FresnelCDI's detector side between the two transforms (FresnelCDI.c++:217-250):
// multiply_factors(-1) -> add(illumination) -> scale_intensity ->
// add(-illumination) -> multiply_factors(+1), all at the same element.
__global__ void k_detector_fresnel(double2 *c, const double2 *__restrict__ coef,
                                   const double2 *__restrict__ ill,
                                   const double *__restrict__ isqrt,
                                   const double *__restrict__ bs, int nx, int ny,
                                   double *partials)
{
    double diff = 0, mag = 0;
    const double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    const int qy = ny / 2;
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / ny), j = (int)(e - (size_t)i * ny);
        const int i_ = (int)(x_mid - fabs(x_mid - i));
        const int j_ = (int)(y_mid - fabs(y_mid - j));
        const double2 cf = coef[(size_t)i_ * qy + j_];
        const double2 t = ill[e];
        double2 o = c[e];
        double cr = cf.x, ci = -1 * cf.y;
        double2 v = make_double2(o.x * cr - o.y * ci, o.y * cr + o.x * ci);
        v = make_double2(v.x + 1.0 * t.x, v.y + 1.0 * t.y);
        if (bs == nullptr || bs[e] > 0) {
            const double cis = isqrt[e];
            const double cm = mag_of(v);
            v = set_mag(v, cis);
            mag += cis * cis;
            diff += (cm - cis) * (cm - cis);
        }
        v = make_double2(v.x + -1.0 * t.x, v.y + -1.0 * t.y);
        ci = 1 * cf.y;
        c[e] = make_double2(v.x * cr - v.y * ci, v.y * cr + v.x * ci);
    }
    block_sum2(diff, mag);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = diff;
        partials[2 * blockIdx.x + 1] = mag;
    }
}

// multiply_factors' operation on element (i, j)
__device__ __forceinline__ double2 factor_at(double2 o, const double2 *__restrict__ coef, int i,
                                             int j, int nx, int ny, int direction)
{
    const double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    const int i_ = (int)(x_mid - fabs(x_mid - i));
    const int j_ = (int)(y_mid - fabs(y_mid - j));
    const double2 cf = coef[(size_t)i_ * (ny / 2) + j_];
    const double cr = cf.x, ci = direction * cf.y;
    return make_double2(o.x * cr - o.y * ci, o.y * cr + o.x * ci);
}

// invert(scale) and multiply_factors in one pass (FresnelCDI_WF.c++:165-182):
// each thread takes a swap pair (q, p(q)); factors_first multiplies before
// the swap (propagate_to_detector), otherwise after it (propagate_from)
__global__ void k_invert_factors(double2 *a, const double2 *__restrict__ coef, int nx, int ny,
                                 double s, int direction, int factors_first)
{
    const int mx = nx / 2, my = ny / 2;
    const size_t total = (size_t)nx * my;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
         e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / my), j = (int)(e - (size_t)i * my);
        const int jn = j + my;
        int in = i + mx;
        if (i >= mx) in = in - 2 * mx;
        double2 *pp = a + (size_t)in * ny + jn, *qq = a + (size_t)i * ny + j;
        double2 t = *pp, u = *qq;
        if (factors_first) {
            t = factor_at(t, coef, in, jn, nx, ny, direction);
            u = factor_at(u, coef, i, j, nx, ny, direction);
        }
        double2 np = make_double2(u.x * s, u.y * s), nq = make_double2(t.x * s, t.y * s);
        if (!factors_first) {
            np = factor_at(np, coef, in, jn, nx, ny, direction);
            nq = factor_at(nq, coef, i, j, nx, ny, direction);
        }
        *pp = np;
        *qq = nq;
    }
}

__global__ void k_multiply_factors(double2 *c, const double2 *__restrict__ coef, int nx, int ny,
                                   int direction)
{
    const double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    const int qy = ny / 2;
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e / ny), j = (int)(e - (size_t)i * ny);
        double2 o = c[e];
        int i_ = (int)(x_mid - fabs(x_mid - i));
        int j_ = (int)(y_mid - fabs(y_mid - j));
        double2 cf = coef[(size_t)i_ * qy + j_];
        double cr = cf.x, ci = direction * cf.y;
        c[e] = make_double2(o.x * cr - o.y * ci, o.y * cr + o.x * ci);
    }
}

__global__ void k_add_scaled(double2 *c, const double2 *__restrict__ b, double sc, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double2 v = c[k], t = b[k];
        c[k] = make_double2(v.x + sc * t.x, v.y + sc * t.y);
    }
}

__global__ void k_scale(double2 *c, double f, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double2 v = c[k];
        c[k] = make_double2(v.x * f, v.y * f);
    }
}

__global__ void k_pad(const double2 *__restrict__ x, int nx, int ny, double2 *p, int px, int py)
{
    const int mx = nx + 2 * px, my = ny + 2 * py;
    const size_t n = (size_t)mx * my;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e / my) - px, j = (int)(e % my) - py;
        p[e] = (i >= 0 && i < nx && j >= 0 && j < ny) ? x[(size_t)i * ny + j]
                                                      : make_double2(0.0, 0.0);
    }
}

__global__ void k_unpad(const double2 *__restrict__ p, int nx, int ny, int px, int py,
                        double2 *x)
{
    const int my = ny + 2 * py;
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e / ny), j = (int)(e - (size_t)i * ny);
        x[e] = p[(size_t)(i + px) * my + j + py];
    }
}

__global__ void k_poly_expand(const double2 *__restrict__ c, const double *__restrict__ spec,
                              int nl, double lambdac, int nx, int ny, int px, int py,
                              double *isc)
{
    const int mx = nx + 2 * px, my = ny + 2 * py;
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e / ny) + px, j = (int)(e % ny) + py; // padded coordinates
        double acc = 0.0;
        for (int sn = 0; sn < nl; ++sn) {
            double lambda = spec[2 * sn], weightl = spec[2 * sn + 1];
            double lf = lambda / lambdac;
            double xval = lf * (i - nx / 2.0) + nx / 2.0;
            double yval = lf * (j - ny / 2.0) + ny / 2.0;
            if (((xval >= 0) && (xval < mx)) && ((yval >= 0) && (yval < my))) {
                double m = mag_of(c[(size_t)(int)xval * my + (int)yval]);
                acc = acc + weightl * (m * m);
            }
        }
        isc[e] = sqrt(acc);
    }
}

__global__ void k_poly_scale(double2 *c, const double *__restrict__ isc,
                             const double *__restrict__ isqrt, const double *__restrict__ bs,
                             int nx, int ny, int px, int py, double *partials)
{
    const int my = ny + 2 * py;
    const size_t n = (size_t)nx * ny;
    double diff = 0, mag = 0;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        if (bs == nullptr || bs[e] > 0) {
            int i = (int)(e / ny), j = (int)(e - (size_t)i * ny);
            double calc = isc[e], meas = isqrt[e], scaled;
            double2 *pp = c + (size_t)(i + px) * my + j + py;
            double2 v = *pp;
            if (calc == 0.0)
                scaled = 0.0;
            else
                scaled = mag_of(v) * meas / calc;
            *pp = set_mag(v, scaled);
            mag += meas * meas;
            diff += (meas - calc) * (meas - calc);
        }
    }
    block_sum2(diff, mag);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = diff;
        partials[2 * blockIdx.x + 1] = mag;
    }
}

__global__ void k_magnitude(const double2 *__restrict__ c, double *out, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        out[k] = mag_of(c[k]);
}

__global__ void k_convolve(const double *__restrict__ in, double *out, int nx, int ny,
                           const double *__restrict__ g, int cut)
{
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(e / ny), j = (int)(e - (size_t)i * ny);
        double nv = 0;
        for (int i2 = i - cut; i2 <= i + cut; ++i2)
            for (int j2 = j - cut; j2 <= j + cut; ++j2)
                if (i2 < nx && i2 >= 0 && j2 >= 0 && j2 < ny)
                    nv += in[(size_t)i2 * ny + j2] * g[abs(i - i2) * (cut + 1) + abs(j - j2)];
        out[e] = nv;
    }
}

__global__ void k_max_partial(const double *__restrict__ a, size_t n, double *partials)
{
    __shared__ double sm[kThreads];
    __shared__ int has[kThreads];
    double m = 0;
    int h = 0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double v = a[k];
        if (!h || v > m) { m = v; h = 1; }
    }
    sm[threadIdx.x] = m;
    has[threadIdx.x] = h;
    __syncthreads();
    for (int off = kThreads / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            double o = sm[threadIdx.x + off];
            int oh = has[threadIdx.x + off];
            if (oh && (!has[threadIdx.x] || o > sm[threadIdx.x])) {
                sm[threadIdx.x] = o;
                has[threadIdx.x] = 1;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = sm[0];
        partials[2 * blockIdx.x + 1] = has[0];
    }
}

__global__ void k_max_finish(const double *partials, int nb, double *out)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double m = 0;
        int h = 0;
        for (int b = 0; b < nb; ++b)
            if (partials[2 * b + 1] != 0 && (!h || partials[2 * b] > m)) {
                m = partials[2 * b];
                h = 1;
            }
        *out = m;
    }
}

// apply_threshold with the reference's loop bounds (i < nx, j < nx) and
// Real_2D::get's (x > nx, y > ny) test: an element at linear index L is
// visited once per pair (i, j = L - i*ny) with 0 <= j < nx, in increasing i.
__global__ void k_threshold(double *a, int nx, int ny, double t, const double *dmax)
{
    const double lim = t * (*dmax);
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        long long L = (long long)e;
        long long ilo = (L - nx + 1 + ny - 1) / ny; // ceil((L-nx+1)/ny) for L-nx+1 >= 0
        if (L - nx + 1 < 0) ilo = 0;
        long long ihi = L / ny;
        if (ihi > nx - 1) ihi = nx - 1;
        if (ilo > ihi) continue;
        double cur = a[e];
        for (long long i = ilo; i <= ihi; ++i) {
            long long j = L - i * ny;
            double v = (j > ny) ? 0.0 : cur;
            cur = (v < lim) ? 0.0 : 1.0;
        }
        a[e] = cur;
    }
}

__global__ void k_divide_by_max(const double *__restrict__ in, double *out, size_t n,
                                const double *dmax)
{
    const double m = *dmax;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        out[k] = in[k] / m;
}

__global__ void k_fresnel_set_t(const double2 *__restrict__ t, const double2 *__restrict__ ill,
                                double2 *esw, int nx, int ny)
{
    const size_t n = (size_t)nx * ny;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n;
         e += (size_t)gridDim.x * blockDim.x) {
        int j = (int)(e % ny);
        if (ny >= nx && j >= nx) continue;
        double2 l = ill[e], tt = t[e];
        esw[e] = make_double2(l.x * tt.x - l.y * tt.y - l.x, l.x * tt.y + l.y * tt.x - l.y);
    }
}

__global__ void k_fresnel_get_t(const double2 *__restrict__ esw, const double2 *__restrict__ ill,
                                double2 *out, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double2 l = ill[k];
        double denom = l.x * l.x + l.y * l.y;
        if (denom != 0) {
            double2 e = esw[k];
            double rn = l.x * (e.x + l.x) + l.y * (e.y + l.y);
            double in = l.x * (e.y + l.y) - l.y * (e.x + l.x);
            out[k] = make_double2(rn / denom, in / denom);
        } else {
            out[k] = make_double2(1.0, 0.0);
        }
    }
}

__global__ void k_autocorr_fill(const double *__restrict__ isqrt, double2 *t, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double comp = (1.0 / sqrt(2.0)) * (isqrt[k] * isqrt[k]);
        t[k] = make_double2(comp, comp);
    }
}

// A pass of radix R (2, 4 or 8) over L signals of length n in ONE shared
// buffer: every thread loads the inputs of its butterflies (at most EPT
// elements) into registers, the block synchronises, then each thread applies
// the twiddles and the butterfly of pass_fixed and stores its outputs.  Same
// arithmetic as pass_fixed, half its shared memory (twice the resident
// blocks).  Requires L * n <= EPT * NT.
template <int R, int EPT, int NT>
__device__ __forceinline__ void pass_one_buffer(double2 *buf, int n, int L, int Ns,
                                                const double2 *__restrict__ W, bool fwd)
{
    constexpr int NB = EPT / R;
    const int m = n / R;
    const int tstep = n / (Ns * R);
    const int total = L * m;
    double2 v[NB][R];
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = threadIdx.x + q * NT;
        if (b < total) {
            const int sig = b / m, j = b - sig * m;
            const double2 *src = buf + (size_t)sig * n;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = src[j + r * m];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int b = threadIdx.x + q * NT;
        if (b < total) {
            const int sig = b / m, j = b - sig * m;
            double2 *dst = buf + (size_t)sig * n;
            const int k = j % Ns;
            double2 *x = v[q];
            if (k > 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    double2 w = __ldg(&W[k * r * tstep]);
                    if (!fwd) w.y = -w.y;
                    x[r] = cmul(x[r], w);
                }
            }
            if (R == 2) {
                double2 a = x[0], c = x[1];
                x[0].x = a.x + c.x; x[0].y = a.y + c.y;
                x[1].x = a.x - c.x; x[1].y = a.y - c.y;
            } else if (R == 4) {
                bf4(x, fwd);
            } else {
                bf8(x, fwd);
            }
            const int base = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[base + r * Ns] = x[r];
        }
    }
    __syncthreads();
}

template <int EPT, int NT>
__device__ void run_passes_one_buffer(double2 *buf, int L, const FftPlan &p,
                                      const double2 *__restrict__ W, bool fwd)
{
    int Ns = 1;
    for (int ip = 0; ip < p.np; ++ip) {
        const int R = p.radix[ip];
        if (R == 8)
            pass_one_buffer<8, EPT, NT>(buf, p.n, L, Ns, W, fwd);
        else if (R == 4)
            pass_one_buffer<4, EPT, NT>(buf, p.n, L, Ns, W, fwd);
        else
            pass_one_buffer<2, EPT, NT>(buf, p.n, L, Ns, W, fwd);
        Ns *= R;
    }
}

template <int EPT, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_fft_rows1(double2 *data, int nx, int ny, int rows,
                                                  FftPlan p, const double2 *__restrict__ W,
                                                  bool fwd)
{
    extern __shared__ double2 sm[];
    const int r0 = blockIdx.x * rows;
    const int nr = min(rows, nx - r0);
    double2 *g = data + (size_t)r0 * ny;
    for (int e = threadIdx.x; e < nr * ny; e += NT) sm[e] = g[e];
    __syncthreads();
    run_passes_one_buffer<EPT, NT>(sm, nr, p, W, fwd);
    for (int e = threadIdx.x; e < nr * ny; e += NT) g[e] = sm[e];
}

template <int EPT, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_fft_cols1(double2 *data, int nx, int ny, int cols,
                                                  FftPlan p, const double2 *__restrict__ W,
                                                  bool fwd)
{
    extern __shared__ double2 sm[];
    const int c0 = blockIdx.x * cols;
    const int nc = min(cols, ny - c0);
    for (int e = threadIdx.x; e < nc * nx; e += NT) {
        int i = e / nc, c = e - i * nc;
        sm[(size_t)c * nx + i] = data[(size_t)i * ny + c0 + c];
    }
    __syncthreads();
    run_passes_one_buffer<EPT, NT>(sm, nc, p, W, fwd);
    for (int e = threadIdx.x; e < nc * nx; e += NT) {
        int i = e / nc, c = e - i * nc;
        data[(size_t)i * ny + c0 + c] = sm[(size_t)c * nx + i];
    }
}

bool pow2_radices(const FftPlan &p)
{
    for (int i = 0; i < p.np; ++i)
        if (p.radix[i] != 2 && p.radix[i] != 4 && p.radix[i] != 8) return false;
    return true;
}

inline int grid_of(size_t n) { return std::min(blocks_for(n), 148 * 16); }

} // namespace

// one-buffer kernels: 8 elements per thread; rows with 256 threads (signals
// of up to 2048 points), columns with 256 threads, or 512 from 2048 points
constexpr int kRowNT = 256, kRowEPT = 8, kRowMinB = 2, kColNT = 256, kColEPT = 8, kColMinB = 2,
              kColWideNT = 512;

void Fft2d::init(int nx_, int ny_)
{
    nx = nx_;
    ny = ny_;
    px = make_plan(nx);
    py = make_plan(ny);
    std::vector<double2> hx = twiddles(nx), hy = twiddles(ny);
    wx.alloc(nx);
    wy.alloc(ny);
    upload_now(wx.p, hx.data(), wx.bytes());
    upload_now(wy.p, hy.data(), wy.bytes());
    const size_t budget = 128 * 1024;
    rows_per_block = std::max(1, 2048 / ny);
    while (rows_per_block > 1 && 2 * (size_t)rows_per_block * ny * sizeof(double2) > budget)
        --rows_per_block;
    cols_per_block = std::max(1, std::min(8, 4096 / nx));
    while (cols_per_block > 1 && 2 * (size_t)cols_per_block * nx * sizeof(double2) > budget)
        --cols_per_block;
    // radix-2/4/8 plans run the one-buffer kernels (measured on B200 at
    // 1024^2 and 2048^2: 10-14% less time per FP64 iteration); columns of
    // 2048 points and more with 512 threads
    row_one = pow2_radices(py) && ny <= kRowEPT * kRowNT;
    if (row_one) rows_per_block = std::max(1, kRowEPT * kRowNT / ny);
    col_wide = nx >= 2048;
    const int col_nt = col_wide ? kColWideNT : kColNT;
    col_one = pow2_radices(px) && nx <= kColEPT * col_nt;
    if (col_one) cols_per_block = std::max(1, std::min(4, kColEPT * col_nt / nx));
    row_smem = (row_one ? 1 : 2) * (size_t)rows_per_block * ny * sizeof(double2);
    col_smem = (col_one ? 1 : 2) * (size_t)cols_per_block * nx * sizeof(double2);
    NADIA_REQUIRE(row_smem <= 227 * 1024 && col_smem <= 227 * 1024, NADIA_ERR_INVALID,
                  "grid too large for the FP64 transform");
    // the attribute belongs to the kernel, not to this plan: every plan sets
    // the same (largest) limit, so a smaller plan made later cannot lower it
    // below what an earlier, larger plan launches with
    NADIA_CUDA(cudaFuncSetAttribute(k_fft_rows, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    227 * 1024));
    NADIA_CUDA(cudaFuncSetAttribute(k_fft_cols, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    227 * 1024));
    NADIA_CUDA(cudaFuncSetAttribute(k_fft_rows1<kRowEPT, kRowNT, kRowMinB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    NADIA_CUDA(cudaFuncSetAttribute(k_fft_cols1<kColEPT, kColNT, kColMinB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    NADIA_CUDA(cudaFuncSetAttribute(k_fft_cols1<kColEPT, kColWideNT, 1>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
}

void Fft2d::exec(double2 *a, bool forward, cudaStream_t s) const
{
    int gr = (nx + rows_per_block - 1) / rows_per_block;
    if (row_one)
        k_fft_rows1<kRowEPT, kRowNT, kRowMinB><<<gr, kRowNT, row_smem, s>>>(a, nx, ny, rows_per_block, py,
                                                                 wy.p, forward);
    else
        k_fft_rows<<<gr, kThreads, row_smem, s>>>(a, nx, ny, rows_per_block, py, wy.p, forward);
    int gc = (ny + cols_per_block - 1) / cols_per_block;
    if (col_one && col_wide)
        k_fft_cols1<kColEPT, kColWideNT, 1><<<gc, kColWideNT, col_smem, s>>>(
            a, nx, ny, cols_per_block, px, wx.p, forward);
    else if (col_one)
        k_fft_cols1<kColEPT, kColNT, kColMinB><<<gc, kColNT, col_smem, s>>>(a, nx, ny, cols_per_block, px,
                                                                 wx.p, forward);
    else
        k_fft_cols<<<gc, kThreads, col_smem, s>>>(a, nx, ny, cols_per_block, px, wx.p, forward);
    NADIA_CUDA(cudaGetLastError());
}

// Odd grids: Complex_2D::invert's swap loop (Complex_2D.c++:318-353) then
// visits some elements twice and never moves the last column (for odd ny),
// so its result depends on the loop order.  The loop is replayed once on the
// host over element indices: out[k] = in[src[k]] multiplied cnt[k] times by
// the scale factor, one multiplication after the other as the loop does.
__global__ void k_invert_gather(const double2 *__restrict__ in, double2 *__restrict__ out,
                                const int *__restrict__ src, const unsigned char *__restrict__ cnt,
                                size_t n, double s)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double2 v = in[src[k]];
        for (int c = cnt[k]; c > 0; --c) v = make_double2(v.x * s, v.y * s);
        out[k] = v;
    }
}

namespace {
// the replayed loop of an odd grid: read-only tables, one per device and
// size, kept for the life of the process (like the twiddle tables)
struct OddInvert {
    int *src = nullptr;
    unsigned char *cnt = nullptr;
};

const OddInvert &odd_invert(int nx, int ny)
{
    static std::mutex mu;
    static std::map<std::tuple<int, int, int>, OddInvert> cache;
    int dev = 0;
    NADIA_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    OddInvert &t = cache[std::make_tuple(dev, nx, ny)];
    if (!t.src) {
        const size_t n = (size_t)nx * ny;
        std::vector<int> src(n);
        std::vector<unsigned char> cnt(n, 0);
        for (size_t k = 0; k < n; ++k) src[k] = (int)k;
        const int mx = nx / 2, my = ny / 2;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < my; ++j) {
                int jn = j + my, in = i + mx;
                if (i >= mx) in = in - 2 * mx;
                const size_t p = (size_t)in * ny + jn, q = (size_t)i * ny + j;
                const int ts = src[p];
                const unsigned char tc = cnt[p];
                src[p] = src[q];
                cnt[p] = (unsigned char)(cnt[q] + 1);
                src[q] = ts;
                cnt[q] = (unsigned char)(tc + 1);
            }
        NADIA_CUDA(cudaMalloc(&t.src, n * sizeof(int)));
        NADIA_CUDA(cudaMalloc(&t.cnt, n));
        upload_now(t.src, src.data(), n * sizeof(int));
        upload_now(t.cnt, cnt.data(), n);
    }
    return t;
}
} // namespace

void invert(double2 *a, int nx, int ny, bool sc, cudaStream_t s, double2 *scratch)
{
    double f = 1;
    if (sc) f = 1.0 / (sqrt((double)(nx * ny)));
    if ((nx | ny) & 1) {
        NADIA_REQUIRE(scratch != nullptr, NADIA_ERR_INVALID, "odd grids need a scratch array");
        const OddInvert &t = odd_invert(nx, ny);
        const size_t n = (size_t)nx * ny;
        k_invert_gather<<<grid_of(n), kThreads, 0, s>>>(a, scratch, t.src, t.cnt, n, f);
        NADIA_CUDA(cudaMemcpyAsync(a, scratch, n * sizeof(double2), cudaMemcpyDeviceToDevice, s));
        return;
    }
    k_invert<<<grid_of((size_t)nx * (ny / 2)), kThreads, 0, s>>>(a, nx, ny, f);
}

void scale_intensity(double2 *c, const double *isqrt, const double *bs, size_t n,
                     double *partials, double *err, cudaStream_t s)
{
    k_scale_intensity<<<kRedBlocks, kThreads, 0, s>>>(c, isqrt, bs, n, partials);
    k_finish_error<<<1, kThreads, 0, s>>>(partials, kRedBlocks, err);
}

void support_constraint(double2 *c, const double *sup, size_t n, cudaStream_t s)
{
    k_support<<<grid_of(n), kThreads, 0, s>>>(c, sup, n);
}

void combine(double2 *x, const double2 *pfs, const double2 *pf, const double2 *ps,
             const double2 *psf, const double w[5], size_t n, cudaStream_t s)
{
    Weights W;
    for (int i = 0; i < 5; ++i) W.w[i] = w[i];
    W.id = 1 + w[4];
    k_combine<<<grid_of(n), kThreads, 0, s>>>(x, pfs, pf, ps, psf, W, n);
}

void invert_factors(double2 *c, const double2 *coef, int nx, int ny, int direction,
                    bool factors_first, cudaStream_t s)
{
    const double f = 1.0 / (sqrt((double)(nx * ny)));
    k_invert_factors<<<grid_of((size_t)nx * (ny / 2)), kThreads, 0, s>>>(
        c, coef, nx, ny, f, direction, factors_first ? 1 : 0);
}

void combine_support(double2 *x, const double2 *pf, const double *support, bool use_ps,
                     bool use_psf, const double w[5], size_t n, cudaStream_t s)
{
    Weights W;
    for (int i = 0; i < 5; ++i) W.w[i] = w[i];
    W.id = 1 + w[4];
    k_combine_support<<<grid_of(n), kThreads, 0, s>>>(x, pf, support, use_ps ? 1 : 0,
                                                     use_psf ? 1 : 0, W, n);
}

void detector_planar(double2 *c, const double *isqrt, const double *bs, int nx, int ny,
                     double *partials, double *err, cudaStream_t s)
{
    const double f = 1.0 / (sqrt((double)(nx * ny))); // invert(scale), Complex_2D.c++:318-353
    k_detector_planar<<<kRedBlocks, kThreads, 0, s>>>(c, isqrt, bs, nx, ny, f, partials);
    k_finish_error<<<1, kThreads, 0, s>>>(partials, kRedBlocks, err);
}

void detector_fresnel(double2 *c, const double2 *coef, const double2 *ill, const double *isqrt,
                      const double *bs, int nx, int ny, double *partials, double *err,
                      cudaStream_t s)
{
    k_detector_fresnel<<<kRedBlocks, kThreads, 0, s>>>(c, coef, ill, isqrt, bs, nx, ny, partials);
    k_finish_error<<<1, kThreads, 0, s>>>(partials, kRedBlocks, err);
}

void multiply_factors(double2 *c, const double2 *coef, int nx, int ny, int direction,
                      cudaStream_t s)
{
    k_multiply_factors<<<grid_of((size_t)nx * ny), kThreads, 0, s>>>(c, coef, nx, ny, direction);
}

void add_scaled(double2 *c, const double2 *b, double sc, size_t n, cudaStream_t s)
{
    k_add_scaled<<<grid_of(n), kThreads, 0, s>>>(c, b, sc, n);
}

void scale(double2 *c, double f, size_t n, cudaStream_t s)
{
    k_scale<<<grid_of(n), kThreads, 0, s>>>(c, f, n);
}

void pad(const double2 *x, int nx, int ny, double2 *p, int px, int py, cudaStream_t s)
{
    size_t n = (size_t)(nx + 2 * px) * (ny + 2 * py);
    k_pad<<<grid_of(n), kThreads, 0, s>>>(x, nx, ny, p, px, py);
}

void unpad(const double2 *p, int nx, int ny, int px, int py, double2 *x, cudaStream_t s)
{
    k_unpad<<<grid_of((size_t)nx * ny), kThreads, 0, s>>>(p, nx, ny, px, py, x);
}

void poly_expand(const double2 *c, const double *spec, int nl, double lambdac, int nx, int ny,
                 int px, int py, double *isc, cudaStream_t s)
{
    k_poly_expand<<<grid_of((size_t)nx * ny), kThreads, 0, s>>>(c, spec, nl, lambdac, nx, ny,
                                                               px, py, isc);
}

void poly_scale(double2 *c, const double *isc, const double *isqrt, const double *bs, int nx,
                int ny, int px, int py, double *partials, double *err, cudaStream_t s)
{
    k_poly_scale<<<kRedBlocks, kThreads, 0, s>>>(c, isc, isqrt, bs, nx, ny, px, py, partials);
    k_finish_error<<<1, kThreads, 0, s>>>(partials, kRedBlocks, err);
}

void magnitude(const double2 *c, double *out, size_t n, cudaStream_t s)
{
    k_magnitude<<<grid_of(n), kThreads, 0, s>>>(c, out, n);
}

void convolve(const double *in, double *out, int nx, int ny, const double *g, int cut,
              cudaStream_t s)
{
    k_convolve<<<grid_of((size_t)nx * ny), kThreads, 0, s>>>(in, out, nx, ny, g, cut);
}

void max_reduce(const double *a, size_t n, double *partials, double *out, cudaStream_t s)
{
    k_max_partial<<<kRedBlocks, kThreads, 0, s>>>(a, n, partials);
    k_max_finish<<<1, 32, 0, s>>>(partials, kRedBlocks, out);
}

void threshold(double *a, int nx, int ny, double t, const double *dmax, cudaStream_t s)
{
    k_threshold<<<grid_of((size_t)nx * ny), kThreads, 0, s>>>(a, nx, ny, t, dmax);
}

void divide_by_max(const double *in, double *out, size_t n, const double *dmax, cudaStream_t s)
{
    k_divide_by_max<<<grid_of(n), kThreads, 0, s>>>(in, out, n, dmax);
}

void fresnel_set_transmission(const double2 *t, const double2 *ill, double2 *esw, int nx, int ny,
                              cudaStream_t s)
{
    k_fresnel_set_t<<<grid_of((size_t)nx * ny), kThreads, 0, s>>>(t, ill, esw, nx, ny);
}

void fresnel_get_transmission(const double2 *esw, const double2 *ill, double2 *out, size_t n,
                              cudaStream_t s)
{
    k_fresnel_get_t<<<grid_of(n), kThreads, 0, s>>>(esw, ill, out, n);
}

// TransmissionConstraint::apply_constraint, TransmissionConstraint.c++:76-172
// region sums of |ln|t|| and |arg t| per block, in a fixed order: each
// thread walks its pixels four at a time (one int4 of the region map, so the
// map streams at full width) and accumulates region pixels in order
__global__ void k_tc_sums(const double2 *__restrict__ t, const int *__restrict__ region, size_t n,
                          int R, double *partials)
{
    double lnA[kMaxRegions], ph[kMaxRegions];
    for (int r = 0; r < R; ++r) lnA[r] = ph[r] = 0;
    const int4 *reg4 = reinterpret_cast<const int4 *>(region);
    const size_t n4 = n / 4; // n = nx*ny with even nx and ny
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n4;
         q += (size_t)gridDim.x * blockDim.x) {
        const int4 rr = __ldg(&reg4[q]);
        const int rv[4] = {rr.x, rr.y, rr.z, rr.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int r = rv[c];
            if (r > 0) {
                const double2 v = t[4 * q + c];
                ph[r - 1] += fabs(atan2(v.y, v.x));
                lnA[r - 1] += fabs(log(mag_of(v)));
            }
        }
    }
    for (int r = 0; r < R; ++r) {
        double a = lnA[r], b = ph[r];
        block_sum2(a, b);
        if (threadIdx.x == 0) {
            partials[2 * ((size_t)blockIdx.x * R + r)] = a;
            partials[2 * ((size_t)blockIdx.x * R + r) + 1] = b;
        }
        __syncthreads();
    }
}

// one block per region: the block partials summed by a fixed tree
__global__ void k_tc_cmean(const double *partials, int nblocks, int R, const double *params,
                           double *cmean)
{
    const int r = blockIdx.x;
    double a = 0, b = 0;
    for (int blk = threadIdx.x; blk < nblocks; blk += blockDim.x) {
        a += partials[2 * ((size_t)blk * R + r)];
        b += partials[2 * ((size_t)blk * R + r) + 1];
    }
    block_sum2(a, b);
    if (threadIdx.x == 0) cmean[r] = params[4 * r + 2] != 0 ? params[4 * r + 3] : a / b;
}

__global__ void k_tc_apply(double2 *t, const int *__restrict__ region, size_t n, int R,
                           const double *__restrict__ params, const double *__restrict__ cmean,
                           int flip, int flip_sign, int unity)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        double2 v = t[k];
        double mag_old = mag_of(v);
        const int r = R > 0 ? region[k] : 0;
        if (r > 0) {
            const double phase_old = atan2(v.y, v.x);
            const double a1 = params[4 * (r - 1)], a2 = params[4 * (r - 1) + 1];
            const double cm = cmean[r - 1];
            const double mag_new = exp((1 - a1) * log(mag_old) + a1 * cm * phase_old);
            const double phase_new = (1 - a2) * phase_old + a2 * log(mag_old) / cm;
            v = set_mag(v, mag_new);
            const double m = mag_of(v); // Complex_2D::set_phase keeps the current magnitude
            v = make_double2(m * cos(phase_new), m * sin(phase_new));
            mag_old = mag_new;
        }
        if (flip && flip_sign * v.y > 0) v.y = -1 * v.y;
        if (unity && mag_old > 1) v = set_mag(v, 1);
        t[k] = v;
    }
}

void autocorr_fill(const double *isqrt, double2 *t, size_t n, cudaStream_t s)
{
    k_autocorr_fill<<<grid_of(n), kThreads, 0, s>>>(isqrt, t, n);
}

void transmission_constraint(double2 *t, const int *region, size_t n, int nregions,
                             const double *params, double *partials, double *cmean,
                             int charge_flip, int flip_sign, int enforce_unity, cudaStream_t s)
{
    if (nregions > 0) {
        k_tc_sums<<<kRedBlocks, kThreads, 0, s>>>(t, region, n, nregions, partials);
        k_tc_cmean<<<nregions, kThreads, 0, s>>>(partials, kRedBlocks, nregions, params, cmean);
    }
    if (nregions > 0 || charge_flip || enforce_unity)
        k_tc_apply<<<grid_of(n), kThreads, 0, s>>>(t, region, n, nregions, params, cmean,
                                                    charge_flip, flip_sign, enforce_unity);
}

} // namespace plain
} // namespace nadia
