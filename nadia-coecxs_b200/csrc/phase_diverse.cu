// phase_diverse.cu -- PhaseDiverseCDI on the GPU (see phase_diverse.h).
// Compiled with --fmad=false: every kernel performs, per pixel, the IEEE
// double operations of the reference's double build in the same order.
#include "phase_diverse.h"

#include <algorithm>
#include <cstring>

namespace nadia {
namespace {

constexpr int kThreads = 256;
constexpr int kArgBlocks = 296;

inline int grid_for(size_t n)
{
    return (int)std::max<size_t>(1, std::min<size_t>((n + kThreads - 1) / kThreads, 148 * 8));
}

void h2d_sync(void *d, const void *h, size_t bytes, cudaStream_t s)
{
    NADIA_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s));
    NADIA_CUDA(cudaStreamSynchronize(s));
}

void d2h_sync(void *h, const void *d, size_t bytes, cudaStream_t s)
{
    NADIA_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
    NADIA_CUDA(cudaStreamSynchronize(s));
}

__global__ void k_fill(double2 *o, size_t n, double re, double im)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        o[k] = make_double2(re, im);
}

// add_to_object's body for one local pixel (PhaseDiverseCDI.c++:556-628)
struct AddArgs {
    const double2 *small;
    const double *w;
    double2 *obj;
    int lnx, lny, nx, ny, x_min, y_min, sc, parallel;
    double xo, yo;
};

__device__ __forceinline__ void blend(const AddArgs &a, double2 *t, double wt, double vr, double vi)
{
    const double2 o = *t;
    double nr = wt * vr + o.x;
    double nim = wt * vi + o.y;
    if (!a.parallel) {
        nr -= wt * o.x;
        nim -= wt * o.y;
    }
    *t = make_double2(nr, nim);
}

__device__ __forceinline__ void add_one(const AddArgs &a, int i_, int j_)
{
    const double wt = a.w[(size_t)i_ * a.lny + j_];
    if (wt == 0) return;
    const int i = (int)(i_ - a.xo - a.x_min) * a.sc;
    const int j = (int)(j_ - a.yo - a.y_min) * a.sc;
    if (!(i >= 0 && j >= 0 && i < a.nx && j < a.ny)) return;
    const double2 f00 = a.small[(size_t)i_ * a.lny + j_];
    if (a.sc == 1) {
        blend(a, a.obj + (size_t)i * a.ny + j, wt, f00.x, f00.y);
        return;
    }
    const double2 f10 = a.small[(size_t)(i_ + 1) * a.lny + j_];
    const double2 f01 = a.small[(size_t)i_ * a.lny + j_ + 1];
    const double2 f11 = a.small[(size_t)(i_ + 1) * a.lny + j_ + 1];
    for (int di = 0; di < a.sc; ++di)
        for (int dj = 0; dj < a.sc; ++dj) {
            const double x = (di + 0.5 * ((a.sc + 1) % 2)) / ((double)a.sc);
            const double y = (dj + 0.5 * ((a.sc + 1) % 2)) / ((double)a.sc);
            const double x1 = 1 - x, y1 = 1 - y;
            const double vr = f00.x * (x1) * (y1) + f10.x * x * (y1) + f01.x * (x1) * y + f11.x * x * y;
            const double vi = f00.y * (x1) * (y1) + f10.y * x * (y1) + f01.y * (x1) * y + f11.y * x * y;
            const int ni = (int)((i_ + 0.5 - a.xo - a.x_min) * a.sc + di);
            const int nj = (int)((j_ + 0.5 - a.yo - a.y_min) * a.sc + dj);
            // the reference's flat index ni*ny + nj: a column past either
            // edge lands in the neighbouring row; outside the whole array
            // the reference writes out of bounds (skipped here)
            const long long f = (long long)ni * a.ny + nj;
            if (f < 0 || f >= (long long)a.nx * a.ny) continue;
            blend(a, a.obj + f, wt, vr, vi);
        }
}

// every interior local pixel at once: valid when no two local pixels reach
// the same object pixel (PhaseDiverse::add_to_object checks)
__global__ void k_add(AddArgs a)
{
    const int w = a.lny - 2;
    const size_t n = (size_t)(a.lnx - 2) * w;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        add_one(a, 1 + (int)(k / w), 1 + (int)(k % w));
}

// the reference's loop order, one thread: positions whose truncation maps
// two local pixels onto one object pixel
__global__ void k_add_in_order(AddArgs a)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int i_ = 1; i_ < a.lnx - 1; ++i_)
        for (int j_ = 1; j_ < a.lny - 1; ++j_) add_one(a, i_, j_);
}

// update_from_object, PhaseDiverseCDI.c++:664-711
__global__ void k_update(const double2 *obj, const double *w, double2 *small, int lnx, int lny,
                         int nx, int ny, int x_min, int y_min, int sc, double xo, double yo)
{
    const size_t n = (size_t)lnx * lny;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        if (w[k] == 0) continue;
        const int i_ = (int)(k / lny), j_ = (int)(k % lny);
        const int i = (int)(i_ - xo - x_min) * sc, j = (int)(j_ - yo - y_min) * sc;
        if (!(i >= 0 && j >= 0 && i < nx && j < ny)) continue;
        if (sc != 1) {
            double re = 0, im = 0;
            for (int di = 0; di < sc; ++di)
                for (int dj = 0; dj < sc; ++dj) {
                    // flat index, as the reference reads (past the array: skipped)
                    const long long f = (long long)(i + di) * ny + j + dj;
                    if (f >= (long long)nx * ny) continue;
                    const double2 o = obj[f];
                    re += o.x;
                    im += o.y;
                }
            const double norm = 1 / ((double)(sc * sc));
            small[k] = make_double2(re * norm, im * norm);
        } else {
            small[k] = obj[(size_t)i * ny + j];
        }
    }
}

// scale_object, PhaseDiverseCDI.c++:290-325
struct FrameRow {
    const double *w;
    double xo, yo;
    int lnx, lny;
};

__global__ void k_scale(double2 *obj, int nx, int ny, int x_min, int y_min, int sc,
                        const FrameRow *fr, int nframes, double factor)
{
    const size_t n = (size_t)nx * ny;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / ny), j = (int)(k % ny);
        bool inside = false;
        for (int f = 0; f < nframes && !inside; ++f) {
            const int i_ = (int)(i / sc + fr[f].xo + x_min);
            const int j_ = (int)(j / sc + fr[f].yo + y_min);
            if (i_ >= 0 && j_ >= 0 && i_ < fr[f].lnx && j_ < fr[f].lny)
                inside = fr[f].w[(size_t)i_ * fr[f].lny + j_] != 0;
        }
        const double2 o = obj[k];
        obj[k] = inside ? make_double2(factor * o.x, factor * o.y) : make_double2(1.0, 0.0);
    }
}

// the object seen through frame n's window (adjust_positions,
// PhaseDiverseCDI.c++:256-272 and 316-327): with magnitudes, `others` and
// `single` of the cross-correlation; without, the window copy of the
// minimum-error search
__global__ void k_window(const double2 *obj, int nx, int ny, int x_min, int y_min, int sc,
                         double bx, double by, int bnx, int bny, double *others, double2 *copy,
                         const double2 *res, int rnx, int rny, int lnx, int lny, double *single)
{
    const size_t n = (size_t)bnx * bny;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / bny), j = (int)(k % bny);
        const int i_ = (int)(i - bx * sc - x_min * sc);
        const int j_ = (int)(j - by * sc - y_min * sc);
        const bool in = i_ >= 0 && j_ >= 0 && i_ < nx && j_ < ny;
        if (copy) {
            if (in) copy[k] = obj[(size_t)i_ * ny + j_];
            continue;
        }
        if (in) {
            const double2 o = obj[(size_t)i_ * ny + j_];
            const double m = sqrt(o.x * o.x + o.y * o.y);
            if (m < 1) others[k] = 1 - m;
        }
        if (i < lnx && j < lny && i < rnx && j < rny) {
            const double2 r = res[(size_t)i * rny + j];
            const double m = sqrt(r.x * r.x + r.y * r.y);
            if (m < 1) single[(size_t)i * lny + j] = 1 - m;
        }
    }
}

// interpolate(Double_2D, Double_2D), utils.c:1305-1352 (big zeroed before)
__global__ void k_interpolate(const double *a, int nx, int ny, double *big, int sc)
{
    const int w = ny - 2;
    const size_t n = (size_t)(nx - 2) * w;
    const int bny = ny * sc;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = 1 + (int)(k / w), j = 1 + (int)(k % w);
        const double f00 = a[(size_t)i * ny + j], f10 = a[(size_t)(i + 1) * ny + j];
        const double f01 = a[(size_t)i * ny + j + 1], f11 = a[(size_t)(i + 1) * ny + j + 1];
        const double ni = (i + 0.5) * sc, nj = (j + 0.5) * sc;
        for (int di = 0; di < sc; ++di)
            for (int dj = 0; dj < sc; ++dj) {
                const double x = (di + 0.5 * ((sc + 1) % 2)) / ((double)sc);
                const double y = (dj + 0.5 * ((sc + 1) % 2)) / ((double)sc);
                const double x1 = 1 - x, y1 = 1 - y;
                const double v = f00 * (x1) * (y1) + f10 * x * (y1) + f01 * (x1) * y + f11 * x * y;
                big[(size_t)(int)(ni + di) * bny + (int)(nj + dj)] = v;
            }
    }
}

// align's canvases (utils.c:1247-1272): the images centred on a grid twice
// their size, as complex (value, 0) ready for the forward transform, their
// 0/1 masks, and the count of mask pixels (weight_sum, a sum of ones)
__global__ void k_place(const double *first, int nx1, int ny1, const double *second, int nx2,
                        int ny2, const double *fw, const double *sw, int cx, int cy,
                        double2 *img1, double2 *img2, double2 *w1, double2 *w2, int count_first,
                        unsigned long long *count)
{
    const size_t n = (size_t)cx * cy;
    unsigned long long local = 0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k / cy), j = (int)(k % cy);
        double a = 0, b = 0, ma = 0, mb = 0;
        if (i >= 0.5 * (cx - nx1) && i < 0.5 * (cx + nx1) && j >= 0.5 * (cy - ny1) &&
            j < 0.5 * (cy + ny1)) {
            const int i_ = (int)(i - 0.5 * (cx - nx1)), j_ = (int)(j - 0.5 * (cy - ny1));
            if (!fw || fw[(size_t)i_ * ny1 + j_] > 0) {
                a = first[(size_t)i_ * ny1 + j_];
                ma = 1.0;
            }
            if (i_ < nx2 && j_ < ny2 && (!sw || sw[(size_t)i_ * ny2 + j_] > 0)) {
                b = second[(size_t)i_ * ny2 + j_];
                mb = 1.0;
            }
            local += (unsigned long long)(count_first ? ma : mb);
        }
        img1[k] = make_double2(a, 0);
        img2[k] = make_double2(b, 0);
        w1[k] = make_double2(ma, 0);
        w2[k] = make_double2(mb, 0);
    }
    if (local) atomicAdd(count, local);
}

// conj(F1) * F2 in Complex_2D::multiply's order (Complex_2D.c++:203-228) on
// the half spectrum kept by a real-to-complex transform, extended to the full
// grid by Hermitian symmetry for the complex-to-real transform
__device__ __forceinline__ double2 cross(double2 f1, double2 f2)
{
    const double ar = f1.x, ai = -1 * f1.y;
    return make_double2(f2.x * ar - f2.y * ai, f2.x * ai + f2.y * ar);
}

__global__ void k_cross(const double2 *f1, const double2 *f2, double2 *p, int cx, int cy)
{
    const int h = cy / 2 + 1;
    const size_t n = (size_t)cx * cy;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(k / cy), y = (int)(k % cy);
        if (y < h) {
            p[k] = cross(f1[k], f2[k]);
        } else {
            const size_t m = (size_t)((cx - x) % cx) * cy + (cy - y);
            const double2 q = cross(f1[m], f2[m]);
            p[k] = make_double2(q.x, -q.y);
        }
    }
}

// align's search (utils.c:1283-1300): the largest correlation / overlap
// ratio among pixels with enough overlap whose shift is in range, the first
// in row order among equals -- the result of the reference's sequential scan
__device__ __forceinline__ bool better(double r, double i, double r2, double i2)
{
    return r > r2 || (r == r2 && i2 >= 0 && i >= 0 && i < i2) || (i >= 0 && i2 < 0);
}

__global__ void k_argmax(const double2 *corr, const double2 *ov, int cx, int cy, double factor,
                         double frac, int min_x, int max_x, int min_y, int max_y, double *part)
{
    __shared__ double sr[kThreads], si[kThreads];
    double br = 0, bi = -1;
    const size_t n = (size_t)cx * cy;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x) {
        const double o = ov[k].x;
        if (!(o / factor > frac)) continue;
        const double r = corr[k].x / o;
        if (!(r > 0)) continue;
        const int i = (int)(k / cy), j = (int)(k % cy);
        int ti = -i, tj = -j;
        if (i >= cx / 2.0) ti = -i + cx;
        if (j >= cy / 2.0) tj = -j + cy;
        if (!(ti >= min_x && ti < max_x && tj >= min_y && tj < max_y)) continue;
        if (better(r, (double)k, br, bi)) {
            br = r;
            bi = (double)k;
        }
    }
    sr[threadIdx.x] = br;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s && better(sr[threadIdx.x + s], si[threadIdx.x + s], sr[threadIdx.x],
                                      si[threadIdx.x])) {
            sr[threadIdx.x] = sr[threadIdx.x + s];
            si[threadIdx.x] = si[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = sr[0];
        part[2 * blockIdx.x + 1] = si[0];
    }
}

__global__ void k_argmax_final(double *part, int nb)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double br = 0, bi = -1;
    for (int b = 0; b < nb; ++b)
        if (better(part[2 * b], part[2 * b + 1], br, bi)) {
            br = part[2 * b];
            bi = part[2 * b + 1];
        }
    part[0] = br;
    part[1] = bi;
}

// Can the interior local pixels of one axis be blended all at once?  Along
// the axis, every local index i_ in [1, n-1) whose base (int)(i_ - off) * sc
// lies in [0, extent) writes the indices (int)((i_ + 0.5 - off) * sc + d),
// d < sc (sc == 1: the base itself).  They must not meet those of another
// local index (truncation toward zero maps (-1, 0) and [0, 1) both to 0),
// and along the inner axis they must stay in [0, extent): outside it the
// reference's flat index wraps into the neighbouring row.  Along the outer
// axis an index outside [0, extent) is outside the whole array and skipped.
bool axis_parallel_safe(int n, double pos, int pmin, int sc, int extent, bool inner)
{
    int last = -1; // the largest index written so far; writes grow with i_
    for (int i_ = 1; i_ < n - 1; ++i_) {
        const int base = (int)(i_ - pos - pmin) * sc; // the kernel's expressions
        if (!(base >= 0 && base < extent)) continue;
        int lo, hi;
        if (sc == 1) {
            lo = hi = base;
        } else {
            lo = (int)((i_ + 0.5 - pos - pmin) * sc + 0);
            hi = (int)((i_ + 0.5 - pos - pmin) * sc + (sc - 1));
        }
        if (lo <= last) return false;
        if (inner && (lo < 0 || hi >= extent)) return false;
        last = hi;
    }
    return true;
}

} // namespace

PhaseDiverse::PhaseDiverse(double beta_, double gamma_, bool parallel_, int granularity)
    : beta(beta_), gamma(gamma_), parallel(parallel_), scale(granularity)
{
    NADIA_REQUIRE(granularity >= 1 && granularity <= 16, NADIA_ERR_INVALID,
                  "granularity must be between 1 and 16");
    NADIA_CUDA(cudaGetDevice(&device));
    NADIA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    own_st.s = st;
    NADIA_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    AllocScope scope(st);
    d_count.alloc(1);
    d_best.alloc(2 * kArgBlocks);
}

PhaseDiverse::~PhaseDiverse()
{
    if (st) cudaStreamSynchronize(st);
    for (Solver *f : frames) --f->pd_refs;
    if (ev) cudaEventDestroy(ev);
}

void PhaseDiverse::join(cudaStream_t from, cudaStream_t to)
{
    if (from == to) return;
    NADIA_CUDA(cudaEventRecord(ev, from));
    NADIA_CUDA(cudaStreamWaitEvent(to, ev, 0));
}

// the object's stream waits for everything queued on the frames' streams, so
// a synchronisation of st covers all of this object's work
void PhaseDiverse::rejoin_frames()
{
    for (size_t n = 0; n < frames.size(); ++n) to_object((int)n);
}

void PhaseDiverse::sync()
{
    rejoin_frames();
    NADIA_CUDA(cudaStreamSynchronize(st));
}

void PhaseDiverse::realloc_object(int nx_, int ny_)
{
    AllocScope scope(st);
    object_buf.alloc((size_t)nx_ * ny_);
    NADIA_CUDA(cudaMemsetAsync(object_buf.p, 0, object_buf.bytes(), st));
    obj = object_buf.p;
    nx = nx_;
    ny = ny_;
}

// add_new_position, PhaseDiverseCDI.c++:104-160
void PhaseDiverse::add_position(Solver *f, double x, double y, double a)
{
    AllocScope scope(st);
    NADIA_REQUIRE(f, NADIA_ERR_INVALID, "null frame");
    NADIA_REQUIRE(f->prec == NADIA_FP64 || f->kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                  "PolyCDI phase-diverse frames run in the FP64 form");
    NADIA_REQUIRE(f->device == device, NADIA_ERR_INVALID,
                  "the frame lives on another device than the phase-diverse object");
    weights_set = false;
    const int lnx = f->nx, lny = f->ny;
    frames.push_back(f);
    ++f->pd_refs;
    xpos.push_back(x);
    ypos.push_back(y);
    alpha.push_back(a);
    rnx.push_back(lnx);
    rny.push_back(lny);
    result.emplace_back((size_t)lnx * lny);
    NADIA_CUDA(cudaMemsetAsync(result.back().p, 0, result.back().bytes(), st));
    weight.emplace_back((size_t)lnx * lny);
    NADIA_CUDA(cudaMemsetAsync(weight.back().p, 0, weight.back().bytes(), st));
    base.emplace_back();
    if (!obj) {
        x_min = (int)(-x);
        y_min = (int)(-y);
        realloc_object(lnx * scale, lny * scale);
    }
    int extra_x = 0, extra_y = 0;
    const int gx0 = (int)(0 - x - x_min) * scale, gy0 = (int)(0 - y - y_min) * scale;
    const int gx1 = (int)(lnx - x - x_min) * scale, gy1 = (int)(lny - y - y_min) * scale;
    if (gx0 < 0) {
        x_min = (int)(-x);
        extra_x += -gx0;
    }
    if (gy0 < 0) {
        y_min = (int)(-y);
        extra_y += -gy0;
    }
    if (gx1 > nx) extra_x += gx1 - nx;
    if (gy1 > ny) extra_y += gy1 - ny;
    if (extra_x || extra_y) realloc_object(nx + extra_x, ny + extra_y);
    NADIA_CUDA(cudaStreamSynchronize(st));
}

void PhaseDiverse::remove_positions()
{
    sync();
    for (Solver *f : frames) --f->pd_refs;
    frames.clear();
}

// set_up_weights, PhaseDiverseCDI.c++:450-530: each weight's
// alpha * pow(|illumination| / max, gamma) (0 outside the support) on the
// host in the reference's order, recomputed only when its inputs change;
// series mode multiplies it by beta on the device, parallel mode
// normalises over the frames on the host
__global__ void k_times(const double *a, double f, double *out, size_t n)
{
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
         k += (size_t)gridDim.x * blockDim.x)
        out[k] = a[k] * f;
}

void PhaseDiverse::set_up_weights()
{
    if (weights_set) return;
    weights_set = true;
    AllocScope scope(st);
    const int frames_n = (int)frames.size();
    for (int n = 0; n < frames_n; ++n) {
        Solver *f = frames[n];
        const int lnx = rnx[n], lny = rny[n];
        // after remove_positions the reference pairs new frames with the
        // earlier positions' arrays by index; only equal sizes are defined
        NADIA_REQUIRE(f->nx == lnx && f->ny == lny, NADIA_ERR_UNSUPPORTED,
                      "a frame added after remove_positions differs in size from the "
                      "position it takes over");
        Base &b = base[n];
        if (b.frame == f && b.version == f->weights_version && b.gamma == gamma &&
            b.alpha == alpha[n])
            continue;
        std::vector<double> support(f->n), mag;
        f->get_support(support.data());
        double max = 0;
        if (f->kind == NADIA_FRESNEL) {
            std::vector<double> ill(2 * f->n);
            f->get_illumination_at_sample(ill.data());
            mag.resize((size_t)lnx * lny);
            for (size_t k = 0; k < mag.size(); ++k)
                mag[k] = std::sqrt(ill[2 * k] * ill[2 * k] + ill[2 * k + 1] * ill[2 * k + 1]);
            max = mag[0];
            for (double v : mag)
                if (v > max) max = v;
        }
        b.h.resize((size_t)lnx * lny);
        for (int i = 0; i < lnx; ++i)
            for (int j = 0; j < lny; ++j) {
                double value = f->kind == NADIA_FRESNEL ? mag[(size_t)i * lny + j] / max : 1;
                value = alpha[n] * std::pow(value, gamma);
                if (support[(size_t)i * f->ny + j] <= 0.0) value = 0;
                b.h[(size_t)i * lny + j] = value;
            }
        if (b.d.n != b.h.size()) b.d.alloc(b.h.size());
        h2d_sync(b.d.p, b.h.data(), b.h.size() * sizeof(double), st);
        b.frame = f;
        b.version = f->weights_version;
        b.gamma = gamma;
        b.alpha = alpha[n];
    }
    if (!parallel) {
        for (int n = 0; n < frames_n; ++n) {
            const size_t m = (size_t)rnx[n] * rny[n];
            k_times<<<grid_for(m), kThreads, 0, st>>>(base[n].d.p, beta, weight[n].p, m);
        }
        NADIA_CUDA(cudaGetLastError());
        return;
    }
    std::vector<std::vector<double>> w(frames_n);
    for (int n = 0; n < frames_n; ++n) w[n] = base[n].h;
    std::vector<double> norm((size_t)nx * ny, 0.0);
    for (int n = 0; n < frames_n; ++n)
        for (int i_ = 0; i_ < rnx[n]; ++i_)
            for (int j_ = 0; j_ < rny[n]; ++j_) {
                const int i = (int)(i_ - xpos[n] - x_min), j = (int)(j_ - ypos[n] - y_min);
                if (i >= 0 && j >= 0 && i < nx && j < ny) {
                    const double v = w[n][(size_t)i_ * rny[n] + j_];
                    double &t = norm[(size_t)i * ny + j];
                    t = n == 0 ? v : v + t;
                }
            }
    for (int n = 0; n < frames_n; ++n)
        for (int i_ = 0; i_ < rnx[n]; ++i_)
            for (int j_ = 0; j_ < rny[n]; ++j_) {
                const int i = (int)(i_ - xpos[n] - x_min), j = (int)(j_ - ypos[n] - y_min);
                if (i >= 0 && j >= 0 && i < nx && j < ny) {
                    double &v = w[n][(size_t)i_ * rny[n] + j_];
                    const double nn = norm[(size_t)i * ny + j];
                    v = nn <= 0 ? 0 : beta * v / nn;
                }
            }
    for (int n = 0; n < frames_n; ++n)
        h2d_sync(weight[n].p, w[n].data(), w[n].size() * sizeof(double), st);
}

// get_result / set_result (PhaseDiverseCDI.c++:330-345) on the frame's stream
void PhaseDiverse::get_result(int n, double2 *dst)
{
    to_frame(n);
    frames[n]->transmission_to_device(dst);
    to_object(n);
}

void PhaseDiverse::set_result(int n, const double2 *src)
{
    to_frame(n);
    frames[n]->transmission_from_device(src);
}

// add_to_object, PhaseDiverseCDI.c++:537-640
void PhaseDiverse::add_to_object(int n)
{
    get_result(n, result[n].p);
    set_up_weights();
    AddArgs a{result[n].p, weight[n].p, obj,  rnx[n], rny[n], nx,        ny,
              x_min,       y_min,       scale, parallel ? 1 : 0, xpos[n], ypos[n]};
    if (a.lnx < 3 || a.lny < 3) return;
    const bool in_order = !axis_parallel_safe(a.lnx, xpos[n], x_min, scale, nx, false) ||
                          !axis_parallel_safe(a.lny, ypos[n], y_min, scale, ny, true);
    if (in_order)
        k_add_in_order<<<1, 32, 0, st>>>(a);
    else
        k_add<<<grid_for((size_t)(a.lnx - 2) * (a.lny - 2)), kThreads, 0, st>>>(a);
    NADIA_CUDA(cudaGetLastError());
}

// update_from_object, PhaseDiverseCDI.c++:664-711
void PhaseDiverse::update_from_object(int n)
{
    set_up_weights();
    k_update<<<grid_for((size_t)rnx[n] * rny[n]), kThreads, 0, st>>>(
        obj, weight[n].p, result[n].p, rnx[n], rny[n], nx, ny, x_min, y_min, scale, xpos[n],
        ypos[n]);
    NADIA_CUDA(cudaGetLastError());
    set_result(n, result[n].p);
}

// scale_object, PhaseDiverseCDI.c++:290-325
void PhaseDiverse::scale_object(double factor)
{
    AllocScope scope(st);
    set_up_weights();
    std::vector<FrameRow> rows(frames.size());
    for (size_t f = 0; f < frames.size(); ++f)
        rows[f] = FrameRow{weight[f].p, xpos[f], ypos[f], rnx[f], rny[f]};
    if (d_frames.n < rows.size() * sizeof(FrameRow))
        d_frames.alloc(std::max<size_t>(rows.size(), 8) * sizeof(FrameRow));
    if (!rows.empty()) h2d_sync(d_frames.p, rows.data(), rows.size() * sizeof(FrameRow), st);
    k_scale<<<grid_for((size_t)nx * ny), kThreads, 0, st>>>(
        obj, nx, ny, x_min, y_min, scale, (const FrameRow *)d_frames.p, (int)rows.size(), factor);
    NADIA_CUDA(cudaGetLastError());
}

// initialise_estimate, PhaseDiverseCDI.c++:163-177
void PhaseDiverse::initialise_estimate()
{
    AllocScope scope(st);
    if (!obj) return;
    k_fill<<<grid_for((size_t)nx * ny), kThreads, 0, st>>>(obj, (size_t)nx * ny, 1.0, 0.0);
    NADIA_CUDA(cudaGetLastError());
    for (size_t n = 0; n < frames.size(); ++n) add_to_object((int)n);
    sync();
}

// iterate, PhaseDiverseCDI.c++:180-230.  In parallel mode each frame's
// iterations run on its own stream, concurrently with the other frames'.
void PhaseDiverse::iterate()
{
    AllocScope scope(st);
    for (size_t n = 0; n < frames.size(); ++n) {
        update_from_object((int)n);
        frames[n]->iterate(iterations_per_cycle);
        if (!parallel) add_to_object((int)n);
    }
    if (parallel) {
        scale_object(1 - beta);
        for (size_t n = 0; n < frames.size(); ++n) add_to_object((int)n);
    }
    sync();
}

void PhaseDiverse::set_feedback_parameter(double b)
{
    beta = b;
    weights_set = false;
}

void PhaseDiverse::set_amplification_factor(double g)
{
    gamma = g;
    weights_set = false;
}

bool PhaseDiverse::set_probe_scaling(int n, double a)
{
    const bool ok = n >= 0 && n < (int)alpha.size();
    if (ok) alpha[n] = a;
    weights_set = false;
    return ok;
}

void PhaseDiverse::get_transmission(double *h)
{
    NADIA_REQUIRE(obj, NADIA_ERR_STATE, "no position has been added");
    sync();
    d2h_sync(h, obj, (size_t)nx * ny * sizeof(double2), st);
}

// set_transmission, PhaseDiverseCDI.c++:81-101
void PhaseDiverse::set_transmission(int nx_, int ny_, const double *h)
{
    NADIA_REQUIRE(nx_ > 0 && ny_ > 0, NADIA_ERR_INVALID, "empty transmission function");
    sync();
    if (!obj) realloc_object(nx_, ny_);
    NADIA_REQUIRE(nx_ == nx && ny_ == ny, NADIA_ERR_INVALID,
                  "the transmission function does not have the dimensions of the current one");
    h2d_sync(obj, h, (size_t)nx * ny * sizeof(double2), st);
}

// align, utils.c:1151-1300, on device images
void PhaseDiverse::align(const double *first, int nx1, int ny1, const double *second, int nx2,
                         int ny2, int &offset_x, int &offset_y, int min_x, int max_x, int min_y,
                         int max_y, const double *first_w, const double *second_w,
                         double overlap_fraction)
{
    AllocScope scope(st);
    const int cx = nx1 > nx2 ? nx1 * 2 : nx2 * 2;
    const int cy = ny1 > ny2 ? ny1 * 2 : ny2 * 2;
    if (min_x == max_x || min_y == max_y) {
        min_x = (int)(1 - cx / 2.0);
        max_x = (int)(cx / 2.0);
        min_y = (int)(1 - cy / 2.0);
        max_y = (int)(cy / 2.0);
    }
    const size_t N = (size_t)cx * cy;
    DevBuf<double2> a(N), b(N), wa(N), wb(N), p(N);
    plain::Fft2d fft;
    fft.init(cx, cy);
    NADIA_CUDA(cudaMemsetAsync(d_count.p, 0, sizeof(unsigned long long), st));
    k_place<<<grid_for(N), kThreads, 0, st>>>(first, nx1, ny1, second, nx2, ny2, first_w,
                                              second_w, cx, cy, a.p, b.p, wa.p, wb.p,
                                              nx1 * ny1 < nx2 * ny2 ? 1 : 0, d_count.p);
    NADIA_CUDA(cudaGetLastError());
    fft.exec(a.p, true, st);
    fft.exec(b.p, true, st);
    k_cross<<<grid_for(N), kThreads, 0, st>>>(a.p, b.p, p.p, cx, cy); // correlation
    fft.exec(p.p, false, st);
    fft.exec(wa.p, true, st);
    fft.exec(wb.p, true, st);
    k_cross<<<grid_for(N), kThreads, 0, st>>>(wa.p, wb.p, a.p, cx, cy); // overlap
    fft.exec(a.p, false, st);
    unsigned long long count = 0;
    d2h_sync(&count, d_count.p, sizeof(count), st);
    const double weight_sum = (double)count;
    const double overlap_factor = weight_sum * cx * cy;
    k_argmax<<<kArgBlocks, kThreads, 0, st>>>(p.p, a.p, cx, cy, overlap_factor, overlap_fraction,
                                               min_x, max_x, min_y, max_y, d_best.p);
    k_argmax_final<<<1, 32, 0, st>>>(d_best.p, kArgBlocks);
    NADIA_CUDA(cudaGetLastError());
    double best[2];
    d2h_sync(best, d_best.p, sizeof(best), st);
    if (best[1] >= 0) {
        const long long k = (long long)best[1];
        const int i = (int)(k / cy), j = (int)(k % cy);
        offset_x = i >= cx / 2.0 ? -i + cx : -i;
        offset_y = j >= cy / 2.0 ? -j + cy : -j;
    }
}

// check_position, PhaseDiverseCDI.c++:395-447
bool PhaseDiverse::check_position(int n, double step, int min_x, int max_x, int min_y,
                                  int max_y, int tries)
{
    AllocScope scope(st);
    const double x = xpos[n], y = ypos[n];
    if (step < 1.0 / scale) return true;
    if (tries > 10 || x < (x + min_x) || x > (x + max_x) || y < (y + min_y) || y > (y + max_y))
        return false;
    Solver *single = frames[n];
    double best_x = x, best_y = y, best_error = 100;
    const size_t on = (size_t)nx * ny, sn = (size_t)rnx[n] * rny[n];
    DevBuf<double2> object_copy(on), single_copy(sn);
    NADIA_CUDA(cudaMemcpyAsync(object_copy.p, obj, on * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    NADIA_CUDA(cudaMemcpyAsync(single_copy.p, result[n].p, sn * sizeof(double2),
                               cudaMemcpyDeviceToDevice, st));
    beta = 0.5;
    weights_set = false;
    for (int i = -1; i < 2; ++i)
        for (int j = -1; j < 2; ++j) {
            const double tx = x + i * step, ty = y + j * step;
            xpos[n] = tx;
            ypos[n] = ty;
            add_to_object(n);
            update_from_object(n);
            single->iterate(1);
            const double e = single->get_error();
            if (e < best_error) {
                best_error = e;
                best_x = tx;
                best_y = ty;
            }
            to_object(n);
            NADIA_CUDA(cudaMemcpyAsync(obj, object_copy.p, on * sizeof(double2),
                                       cudaMemcpyDeviceToDevice, st));
            set_result(n, single_copy.p);
            NADIA_CUDA(cudaMemcpyAsync(result[n].p, single_copy.p, sn * sizeof(double2),
                                       cudaMemcpyDeviceToDevice, st));
        }
    to_object(n);
    NADIA_CUDA(cudaStreamSynchronize(st)); // the copies are released behind their last use
    xpos[n] = best_x;
    ypos[n] = best_y;
    if (best_x == x && best_y == y) step = step / 2.0;
    if (!check_position(n, step, min_x, max_x, min_y, max_y, ++tries)) {
        xpos[n] = x;
        ypos[n] = y;
        return false;
    }
    beta = 1.0;
    weights_set = false;
    return true;
}

// adjust_positions, PhaseDiverseCDI.c++:232-392
void PhaseDiverse::adjust_positions(int type, bool forward, int min_x, int max_x, int min_y,
                                    int max_y, double step_size)
{
    AllocScope scope(st);
    NADIA_REQUIRE(type == CROSS_CORRELATION || type == MINIMUM_ERROR, NADIA_ERR_INVALID,
                  "the alignment type is neither CROSS_CORRELATION nor MINIMUM_ERROR");
    NADIA_REQUIRE(obj && !frames.empty(), NADIA_ERR_STATE, "no position has been added");
    const bool parallel_c = parallel;
    double2 *saved = obj;
    const int nx_c = nx, ny_c = ny, x_min_c = x_min, y_min_c = y_min;
    const double beta_c = beta;
    const int sc = scale;
    parallel = false;
    int n = 1, limit = (int)frames.size();
    if (!forward) {
        n = (int)frames.size() - 2;
        limit = -1;
    }
    DevBuf<double2> temp_object((size_t)nx * ny);
    k_fill<<<grid_for((size_t)nx * ny), kThreads, 0, st>>>(temp_object.p, (size_t)nx * ny, 1.0, 0.0);
    NADIA_CUDA(cudaGetLastError());
    obj = temp_object.p;
    beta = 1.0;
    weights_set = false;
    const int first = forward ? 0 : (int)frames.size() - 1;
    to_frame(first);
    frames[first]->iterate(1);
    get_result(first, result[first].p);
    add_to_object(first);
    while (n != limit) {
        const double bx = xpos[n], by = ypos[n];
        const int lnx = rnx[0], lny = rny[0];
        const int bnx = lnx * sc, bny = lny * sc;
        to_frame(n);
        frames[n]->iterate(1);
        get_result(n, result[n].p);
        if (type == CROSS_CORRELATION) {
            DevBuf<double> single((size_t)lnx * lny), others((size_t)bnx * bny);
            DevBuf<double> weight_int((size_t)bnx * bny), single_int;
            NADIA_CUDA(cudaMemsetAsync(single.p, 0, single.bytes(), st));
            NADIA_CUDA(cudaMemsetAsync(others.p, 0, others.bytes(), st));
            NADIA_CUDA(cudaMemsetAsync(weight_int.p, 0, weight_int.bytes(), st));
            k_window<<<grid_for((size_t)bnx * bny), kThreads, 0, st>>>(
                obj, nx, ny, x_min, y_min, sc, bx, by, bnx, bny, others.p, nullptr, result[n].p,
                rnx[n], rny[n], lnx, lny, single.p);
            NADIA_CUDA(cudaGetLastError());
            Solver *f = frames[n];
            to_object(n); // the frame's support
            const double *single_img = single.p;
            DevBuf<double> fsup;
            const double *fsupport = f->support.p;
            if (f->prec != NADIA_FP64) { // the FP32 form keeps its support in its own layout
                std::vector<double> h(f->n);
                f->get_support(h.data());
                fsup.alloc(f->n);
                h2d_sync(fsup.p, h.data(), f->n * sizeof(double), st);
                fsupport = fsup.p;
            }
            if (sc == 1) {
                NADIA_CUDA(cudaMemcpyAsync(weight_int.p, fsupport,
                                           std::min(weight_int.bytes(), f->n * sizeof(double)),
                                           cudaMemcpyDeviceToDevice, st));
            } else {
                single_int.alloc((size_t)bnx * bny);
                NADIA_CUDA(cudaMemsetAsync(single_int.p, 0, single_int.bytes(), st));
                if (lnx > 2 && lny > 2)
                    k_interpolate<<<grid_for((size_t)(lnx - 2) * (lny - 2)), kThreads, 0, st>>>(
                        single.p, lnx, lny, single_int.p, sc);
                if (f->nx > 2 && f->ny > 2 && f->nx * sc == bnx && f->ny * sc == bny)
                    k_interpolate<<<grid_for((size_t)(f->nx - 2) * (f->ny - 2)), kThreads, 0, st>>>(
                        fsupport, f->nx, f->ny, weight_int.p, sc);
                NADIA_CUDA(cudaGetLastError());
                single_img = single_int.p;
            }
            int new_x = 0, new_y = 0;
            align(single_img, bnx, bny, others.p, bnx, bny, new_x, new_y, min_x, max_x, min_y,
                  max_y, weight_int.p, others.p, 0.2);
            xpos[n] = bx + new_x / ((double)sc);
            ypos[n] = by + new_y / ((double)sc);
            NADIA_CUDA(cudaStreamSynchronize(st));
        } else {
            DevBuf<double2> temp((size_t)bnx * bny);
            NADIA_CUDA(cudaMemsetAsync(temp.p, 0, temp.bytes(), st));
            k_window<<<grid_for((size_t)bnx * bny), kThreads, 0, st>>>(
                obj, nx, ny, x_min, y_min, sc, bx, by, bnx, bny, nullptr, temp.p, nullptr, 0, 0,
                0, 0, nullptr);
            NADIA_CUDA(cudaGetLastError());
            obj = temp.p;
            nx = bnx;
            ny = bny;
            x_min = (int)(-xpos[n]);
            y_min = (int)(-ypos[n]);
            check_position(n, step_size, min_x, max_x, min_y, max_y, 0);
            NADIA_CUDA(cudaStreamSynchronize(st));
            obj = temp_object.p;
            nx = nx_c;
            ny = ny_c;
            x_min = x_min_c;
            y_min = y_min_c;
        }
        weights_set = false;
        add_to_object(n);
        n += forward ? 1 : -1;
    }
    sync();
    obj = saved;
    nx = nx_c;
    ny = ny_c;
    x_min = x_min_c;
    y_min = y_min_c;
    parallel = parallel_c;
    beta = beta_c;
    weights_set = false;
}

} // namespace nadia
