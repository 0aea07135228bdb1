// solver.cu -- host logic of one reconstruction and the plain FP64 iteration.
// Each method cites the reference code whose behaviour it reproduces.
#include "solver.h"

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>

#include "batch.h"
#include "fused32.h"

namespace nadia {

namespace {
std::atomic<unsigned long long> g_uid{1};
std::mutex g_pool_mu;
bool g_pool_set[64] = {};
} // namespace

void retain_pool_memory()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (g_pool_set[dev]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~(uint64_t)0;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    g_pool_set[dev] = true;
}

namespace {
void h2d(void *d, const void *h, size_t bytes, cudaStream_t s)
{
    NADIA_CUDA(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s));
    NADIA_CUDA(cudaStreamSynchronize(s));
}
void d2h(void *h, const void *d, size_t bytes, cudaStream_t s)
{
    NADIA_CUDA(cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s));
    NADIA_CUDA(cudaStreamSynchronize(s));
}
// The C library's srand(seed)/rand() sequence (the reference seeds and draws
// with them in initialise_estimate) from a private generator state: glibc's
// rand() is random() on a 128-byte TYPE_3 state, which initstate_r/random_r
// reproduce exactly, so reconstructions can initialise concurrently.
class GlibcRand {
public:
    explicit GlibcRand(int seed)
    {
        std::memset(&rd_, 0, sizeof rd_);
        std::memset(state_, 0, sizeof state_);
        initstate_r((unsigned)seed, state_, sizeof state_, &rd_);
    }
    int operator()()
    {
        int32_t r = 0;
        random_r(&rd_, &r);
        return r;
    }

private:
    random_data rd_;
    char state_[128];
};

// Real_2D::get_max, Double_2D.h:252-265
double host_max(const double *a, size_t n)
{
    if (n == 0) return 0;
    double m = a[0];
    for (size_t k = 0; k < n; ++k)
        if (a[k] > m) m = a[k];
    return m;
}
} // namespace

Solver::Solver(int kind_, int nx_, int ny_, int prec_, int n_best_)
    : kind(kind_), nx(nx_), ny(ny_), prec(prec_), n_best(n_best_)
{
    NADIA_REQUIRE(kind >= NADIA_PLANAR && kind <= NADIA_FRESNEL_WF, NADIA_ERR_INVALID,
                  "unknown kind");
    NADIA_REQUIRE(prec == NADIA_FP64 || prec == NADIA_FP32, NADIA_ERR_INVALID,
                  "unknown precision");
    NADIA_REQUIRE(nx >= 2 && ny >= 2, NADIA_ERR_INVALID, "grid sizes must be at least 2");
    // Complex_2D::invert assumes even sizes (Complex_2D.c++:327-331); PlanarCDI
    // in the FP64 form reproduces what it does on odd ones, the other kinds
    // index quarter tables or padded grids past their ends there
    NADIA_REQUIRE((nx % 2 == 0 && ny % 2 == 0) || (kind == NADIA_PLANAR && prec == NADIA_FP64),
                  NADIA_ERR_INVALID,
                  "odd grid sizes run in PlanarCDI's FP64 form only; other kinds and the FP32 "
                  "form need even sizes");
    NADIA_REQUIRE(n_best >= 0 && n_best <= 64, NADIA_ERR_INVALID, "n_best must be in [0, 64]");
    FftPlan tmpx = make_plan(nx), tmpy = make_plan(ny);
    (void)tmpx; (void)tmpy;
    n = (size_t)nx * ny;
    uid = g_uid++;
    NADIA_CUDA(cudaGetDevice(&device));
    NADIA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    own_st.s = st;
    AllocScope scope(st); // this reconstruction's buffers are ordered on its stream
    h_isqrt.assign(n, 0.0);
    h_support.assign(n, 0.0);
    d_err.alloc(1);
    d_ring.alloc(kRing);
    partials.alloc(2 * plain::kRedBlocks + 64);
    NADIA_CUDA(cudaMemsetAsync(d_err.p, 0, sizeof(double), st));
    NADIA_CUDA(cudaMemsetAsync(d_ring.p, 0, d_ring.bytes(), st));
    best_err.assign(n_best, 1.0);   // BaseCDI.c++:48
    best_slot.resize(n_best);
    for (int i = 0; i < n_best; ++i) best_slot[i] = i;
    dmax.alloc(2);
    if (prec == NADIA_FP64) {
        x.alloc(n);
        support.alloc(n);
        isqrt.alloc(n);
        recon.alloc(n);
        tmp.alloc(n);
        NADIA_CUDA(cudaMemsetAsync(x.p, 0, x.bytes(), st));
        NADIA_CUDA(cudaMemsetAsync(support.p, 0, support.bytes(), st));
        NADIA_CUDA(cudaMemsetAsync(isqrt.p, 0, isqrt.bytes(), st));
        fft.init(nx, ny);
        for (int i = 0; i < n_best; ++i) {
            best64.emplace_back(n);
            NADIA_CUDA(cudaMemsetAsync(best64.back().p, 0, best64.back().bytes(), st));
        }
    } else {
        f32.reset(new Fused32(*this));
        for (int i = 0; i < n_best; ++i) {
            best32.emplace_back(n);
            NADIA_CUDA(cudaMemsetAsync(best32.back().p, 0, best32.back().bytes(), st));
        }
    }
    algorithm = NADIA_CUSTOM;   // BaseCDI.c++:63-64
    set_algorithm(NADIA_ER);
    NADIA_CUDA(cudaStreamSynchronize(st));
}

Solver::~Solver()
{
    forget_batches_with(uid);
    if (st) {
        cudaStreamSynchronize(st);
        f32.reset();
    }
    // the buffers are released behind the stream's work as the members go;
    // own_st, declared before them, destroys the stream last
}

void Solver::sync()
{
    AllocScope scope(st);
    NADIA_CUDA(cudaStreamSynchronize(st));
    if (f32) f32->check_device_flag();
}

// ------------------------------------------------------------------ inputs

std::vector<double> Solver::gauss_table(double gauss_width, int cut) const
{
    // BaseCDI.c++:441-447
    std::vector<double> g((size_t)(cut + 1) * (cut + 1));
    for (int i = 0; i <= cut; i++)
        for (int j = 0; j <= cut; j++) {
            double denom = 2.0 * gauss_width * gauss_width;
            g[(size_t)i * (cut + 1) + j] = exp(-1 * (i * i + j * j) / denom);
        }
    return g;
}

void Solver::plain_convolve(double *arr, double gauss_width, int cut)
{
    AllocScope scope(st);
    // the table stays on the device while the width and cut-off repeat, so
    // a periodic shrinkwrap neither allocates nor waits for the stream
    if (!(gauss && gauss_width == gauss_width_ && cut == gauss_cut_)) {
        std::vector<double> g = gauss_table(gauss_width, cut);
        gauss.alloc(g.size());
        h2d(gauss.p, g.data(), g.size() * sizeof(double), st);
        gauss_width_ = gauss_width;
        gauss_cut_ = cut;
    }
    plain::convolve(arr, tmp.p, nx, ny, gauss.p, cut, st);
    NADIA_CUDA(cudaMemcpyAsync(arr, tmp.p, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
}

void Solver::upload_support()
{
    AllocScope scope(st);
    if (prec == NADIA_FP64)
        h2d(support.p, h_support.data(), n * sizeof(double), st);
    else
        f32->upload_support(h_support.data());
}

// BaseCDI::set_support, BaseCDI.c++:95-108
void Solver::set_support(const double *obj, bool soften)
{
    AllocScope scope(st);
    ++weights_version;
    double max = host_max(obj, n);
    for (size_t k = 0; k < n; ++k) h_support[k] = obj[k] / max;
    h_support_valid = true;
    upload_support();
    if (soften) {
        if (prec == NADIA_FP64) {
            plain_convolve(support.p, 3, 5);
        } else {
            f32->soften_support();
        }
        h_support_valid = false;
    }
}

// BaseCDI::set_intensity, BaseCDI.c++:118-124
void Solver::set_intensity(const double *I)
{
    AllocScope scope(st);
    for (size_t k = 0; k < n; ++k) h_isqrt[k] = sqrt(I[k]);
    if (prec == NADIA_FP64)
        h2d(isqrt.p, h_isqrt.data(), n * sizeof(double), st);
    else
        f32->upload_intensity();
}

// BaseCDI::set_beam_stop, BaseCDI.c++:112-116
void Solver::set_beam_stop(const double *mask)
{
    AllocScope scope(st);
    has_beam_stop = true;
    h_beam_stop.assign(mask, mask + n);
    if (prec == NADIA_FP64) {
        if (!beam_stop) beam_stop.alloc(n);
        h2d(beam_stop.p, mask, n * sizeof(double), st);
    } else {
        f32->upload_beam_stop(mask);
    }
}

// PolyCDI::set_spectrum(Double_2D), PolyCDI.c++:66-89
void Solver::set_spectrum(const double *wl_weight, int nl)
{
    AllocScope scope(st);
    NADIA_REQUIRE(kind == NADIA_POLY, NADIA_ERR_INVALID, "set_spectrum needs a PolyCDI handle");
    NADIA_REQUIRE(nl >= 1, NADIA_ERR_INVALID, "empty spectrum");
    NADIA_CUDA(cudaStreamSynchronize(st)); // buffers of an earlier spectrum may be replaced
    std::vector<double> sp(wl_weight, wl_weight + 2 * (size_t)nl);
    double maxweight = 0, totweight = 0, lc = 0;
    for (int i = 0; i < nl; i++) {
        if (sp[2 * i + 1] > maxweight) {
            lc = sp[2 * i];
            maxweight = sp[2 * i + 1];
        }
        totweight += sp[2 * i + 1];
    }
    NADIA_REQUIRE(maxweight > 0, NADIA_ERR_INVALID, "spectrum has no positive weight");
    for (int i = 0; i < nl; i++) sp[2 * i + 1] = sp[2 * i + 1] / totweight;
    int npx = (int)((sp[0] / lc - 1.0) * nx / 2);
    int npy = (int)((sp[0] / lc - 1.0) * ny / 2);
    NADIA_REQUIRE(npx >= 0 && npy >= 0, NADIA_ERR_INVALID,
                  "negative padding: list the longest wavelength first (PolyCDI derives the "
                  "padding from row 0)");
    FftPlan tx = make_plan(nx + 2 * npx), ty = make_plan(ny + 2 * npy);
    (void)tx; (void)ty;
    spectrum = sp;
    nlambda = nl;
    lambdac = lc;
    px = npx;
    py = npy;
    has_spectrum = true;
    if (prec == NADIA_FP64) {
        d_spec.alloc(2 * (size_t)nl);
        h2d(d_spec.p, spectrum.data(), d_spec.bytes(), st);
        padded.alloc((size_t)(nx + 2 * px) * (ny + 2 * py));
        isc.alloc(n);
        fft_pad.init(nx + 2 * px, ny + 2 * py);
    } else {
        f32->set_spectrum();
    }
}

void Solver::require_poly_ready() const
{
    NADIA_REQUIRE(kind != NADIA_POLY || has_spectrum, NADIA_ERR_STATE,
                  "PolyCDI needs set_spectrum before it can project");
}

// FresnelCDI::FresnelCDI, FresnelCDI.c++:20-44
void Solver::fresnel_init(const double *wf, double wl, double zfd_, double zfs_, double pixel_,
                          double norm_)
{
    AllocScope scope(st);
    norm = norm_;
    h_illum.assign(2 * n, 0.0);
    for (size_t k = 0; k < 2 * n; ++k) h_illum[k] = wf[k] * norm;
    if (prec == NADIA_FP64) {
        illum.alloc(n);
        illum_sample.alloc(n);
        coef.alloc((size_t)(nx / 2) * (ny / 2));
        h2d(illum.p, h_illum.data(), illum.bytes(), st);
    } else {
        f32->upload_illumination();
    }
    fresnel_set_experimental_parameters(wl, zfd_, zfs_, pixel_);
}

// FresnelCDI::set_experimental_parameters, FresnelCDI.c++:57-95
void Solver::fresnel_set_experimental_parameters(double wl, double zfd_, double zfs_,
                                                 double pixel_)
{
    AllocScope scope(st);
    ++weights_version;
    wavelength = wl;
    pixel = pixel_;
    zfd = zfd_;
    zfs = zfs_;
    const int qy = ny / 2;
    double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    double zsd = zfd - zfs;
    double factor = pixel * pixel * M_PI / (wavelength) * ((1 / zfd) - (1 / zsd));
    std::vector<double2> hc((size_t)(nx / 2) * qy);
    for (int i = 0; i < nx / 2; i++)
        for (int j = 0; j < qy; j++) {
            double phi = factor * ((x_mid - i) * (x_mid - i) + (y_mid - j) * (y_mid - j));
            hc[(size_t)i * qy + j] = make_double2(cos(phi), sin(phi));
        }
    if (prec == NADIA_FP64) {
        h2d(coef.p, hc.data(), coef.bytes(), st);
        NADIA_CUDA(cudaMemcpyAsync(illum_sample.p, illum.p, n * sizeof(double2),
                                   cudaMemcpyDeviceToDevice, st));
        plain_propagate_from(illum_sample.p, false);
        NADIA_CUDA(cudaStreamSynchronize(st));
    } else {
        f32->set_fresnel_geometry(factor);
    }
}

// BaseCDI::apply_support (BaseCDI.c++:130-134) and FresnelCDI::apply_support
// (FresnelCDI.c++:203-215): the support, then the transmission constraint --
// on the estimate itself, or for FresnelCDI on its transmission function
// (get_transmission_function applies the constraint, set_transmission_function
// writes the estimate back)
void Solver::plain_apply_support(double2 *c)
{
    AllocScope scope(st);
    plain::support_constraint(c, support.p, n, st);
    if (!tc.active) return;
    if (kind == NADIA_FRESNEL) {
        plain::fresnel_get_transmission(c, illum_sample.p, tc.tbuf.p, n, st);
        apply_transmission_constraint(tc.tbuf.p);
        plain::fresnel_set_transmission(tc.tbuf.p, illum_sample.p, c, nx, ny, st);
    } else {
        apply_transmission_constraint(c);
    }
}

// TransmissionConstraint::apply_constraint (TransmissionConstraint.c++:76-172),
// ending with the caller's custom function, run on the host copy
void Solver::apply_transmission_constraint(double2 *t)
{
    plain::transmission_constraint(t, tc.region.p, n, tc.nregions, tc.params.p, tc.partials.p,
                                   tc.cmean.p, tc.flip, tc.flip_sign, tc.unity, st);
    if (tc.custom) {
        std::vector<double> h(2 * n);
        d2h(h.data(), t, n * sizeof(double2), st);
        tc.custom(h.data(), nx, ny, tc.user);
        h2d(t, h.data(), n * sizeof(double2), st);
    }
}

// BaseCDI::set_complex_constraint (BaseCDI.h:471-473) with a
// TransmissionConstraint built as TransmissionConstraint.c++:20-73 builds it:
// regions in order, the earlier region keeping a shared pixel; fixed_c NaN
// leaves a region's c_mean free (ComplexConstraint::set_fixed_c otherwise)
void Solver::set_transmission_constraint(int unity, int flip, int flip_sign, int nregions,
                                         const double *regions, const double *alpha,
                                         const double *fixed_c)
{
    AllocScope scope(st);
    NADIA_REQUIRE(nregions >= 0 && nregions <= plain::kMaxRegions, NADIA_ERR_INVALID,
                  "between 0 and 16 complex-constraint regions");
    NADIA_REQUIRE(nregions == 0 || n % 4 == 0, NADIA_ERR_UNSUPPORTED,
                  "complex-constraint regions need a pixel count divisible by 4");
    if (prec == NADIA_FP32) {
        // the per-pixel part runs inside the fused row pass; regions split
        // the row pass around their sums (fused32_tc.cuh)
        NADIA_REQUIRE(kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                      "PolyCDI constraints run in the FP64 form: convert the reconstruction "
                      "first");
        NADIA_REQUIRE(nregions == 0 || (regions && alpha), NADIA_ERR_INVALID,
                      "complex-constraint regions need their masks and alphas");
        std::vector<int> map(nregions > 0 ? n : 0, 0);
        std::vector<double> prm(4 * (size_t)nregions, 0.0);
        for (int r = 0; r < nregions; ++r) {
            for (size_t k = 0; k < n; ++k)
                if (regions[(size_t)r * n + k] > 0 && map[k] == 0) map[k] = r + 1;
            prm[4 * r] = alpha[2 * r];
            prm[4 * r + 1] = alpha[2 * r + 1];
            const bool fixed = fixed_c && fixed_c[r] == fixed_c[r];
            prm[4 * r + 2] = fixed ? 1.0 : 0.0;
            prm[4 * r + 3] = fixed ? fixed_c[r] : 0.0;
        }
        f32->set_constraint(true, unity != 0, flip != 0, flip_sign, nregions, map.data(),
                            prm.data());
        tc.active = true;
        tc.unity = unity ? 1 : 0;
        tc.flip = flip ? 1 : 0;
        tc.flip_sign = flip_sign > 0 ? 1 : -1;
        tc.nregions = nregions;
        tc.custom = nullptr;
        tc.user = nullptr;
        return;
    }
    NADIA_REQUIRE(nregions == 0 || (regions && alpha), NADIA_ERR_INVALID,
                  "complex-constraint regions need their masks and alphas");
    NADIA_CUDA(cudaStreamSynchronize(st)); // buffers of an earlier constraint may be replaced
    tc.active = true;
    tc.unity = unity ? 1 : 0;
    tc.flip = flip ? 1 : 0;
    tc.flip_sign = flip_sign > 0 ? 1 : -1;
    tc.nregions = nregions;
    std::vector<int> map(n, 0);
    std::vector<double> prm(4 * (size_t)std::max(nregions, 1), 0.0);
    for (int r = 0; r < nregions; ++r) {
        for (size_t k = 0; k < n; ++k)
            if (regions[(size_t)r * n + k] > 0 && map[k] == 0) map[k] = r + 1;
        prm[4 * r] = alpha[2 * r];
        prm[4 * r + 1] = alpha[2 * r + 1];
        const bool fixed = fixed_c && fixed_c[r] == fixed_c[r];
        prm[4 * r + 2] = fixed ? 1.0 : 0.0;
        prm[4 * r + 3] = fixed ? fixed_c[r] : 0.0;
    }
    tc.region.alloc(n);
    tc.params.alloc(prm.size());
    tc.partials.alloc(2 * (size_t)plain::kRedBlocks * std::max(nregions, 1));
    tc.cmean.alloc(std::max(nregions, 1));
    if (kind == NADIA_FRESNEL && !tc.tbuf) tc.tbuf.alloc(n);
    h2d(tc.region.p, map.data(), n * sizeof(int), st);
    h2d(tc.params.p, prm.data(), prm.size() * sizeof(double), st);
}

void Solver::set_transmission_custom(void (*fn)(double *, int, int, void *), void *user)
{
    NADIA_REQUIRE(tc.active, NADIA_ERR_STATE, "set a transmission constraint first");
    NADIA_REQUIRE(!fn || prec == NADIA_FP64, NADIA_ERR_UNSUPPORTED,
                  "a custom constraint function runs in the FP64 form: convert the "
                  "reconstruction first");
    tc.custom = fn;
    tc.user = user;
}

void Solver::clear_transmission_constraint()
{
    NADIA_CUDA(cudaStreamSynchronize(st));
    if (prec == NADIA_FP32 && tc.active) f32->set_constraint(false, false, false, 1);
    tc.active = false;
    tc.custom = nullptr;
    tc.user = nullptr;
    tc.nregions = 0;
}

// FresnelCDI_WF::FresnelCDI_WF, FresnelCDI_WF.c++:31-79: the quarter table
// of the zone-plate-to-detector factor, (sin phi, -cos phi) / sqrt(nx*ny),
// computed on the host in the reference's operation order (pow(x, 2) included)
void Solver::fresnel_wf_init(double wl, double zone_focal, double focal_detector, double pixel_)
{
    AllocScope scope(st);
    NADIA_REQUIRE(kind == NADIA_FRESNEL_WF, NADIA_ERR_INVALID, "needs a FresnelCDI_WF handle");
    NADIA_REQUIRE(wl > 0 && zone_focal != 0 && focal_detector != 0 && pixel_ > 0,
                  NADIA_ERR_INVALID, "FresnelCDI_WF needs a wavelength, non-zero distances and "
                                     "a pixel size");
    wavelength = wl;
    z12 = zone_focal;
    z23 = focal_detector;
    pixel = pixel_;
    if (prec == NADIA_FP32) {
        f32->set_wf_geometry();
        return;
    }
    const int qy = ny / 2;
    const double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    const double scaling_x = wl * z23 / (pixel * nx);
    const double scaling_y = wl * z23 / (pixel * ny);
    const double nrm = 1 / (sqrt(nx * ny));
    std::vector<double2> hc((size_t)(nx / 2) * qy);
    for (int i = 0; i < nx / 2; i++)
        for (int j = 0; j < qy; j++) {
            double rho_2 = pow(scaling_x * (x_mid - i), 2) + pow(scaling_y * (y_mid - j), 2);
            double phi = rho_2 / z12 + rho_2 / z23;
            phi *= M_PI / wl;
            hc[(size_t)i * qy + j] = make_double2(sin(phi) * nrm, -cos(phi) * nrm);
        }
    coef.alloc(hc.size());
    h2d(coef.p, hc.data(), coef.bytes(), st);
}

// FresnelCDI_WF::set_support(z_diameter, size), FresnelCDI_WF.c++:184-203:
// the projected zone-plate disk (centre (nx-1)/2 in integer arithmetic, on
// both axes) set to 1 over the current support, then convolve(support, 3, 5)
void Solver::fresnel_wf_set_support(double z_diameter, double size)
{
    ++weights_version;
    AllocScope scope(st);
    NADIA_REQUIRE(kind == NADIA_FRESNEL_WF, NADIA_ERR_INVALID, "needs a FresnelCDI_WF handle");
    if (!h_support_valid) get_support(h_support.data());
    const double center_pixel = (nx - 1) / 2;
    const double delta_z = (z12 / z23) * pixel;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            double i_ = i - center_pixel;
            double j_ = j - center_pixel;
            double r = delta_z * sqrt(i_ * i_ + j_ * j_);
            if (r < size * z_diameter / 2.0) h_support[(size_t)i * ny + j] = 1;
        }
    upload_support();
    if (prec == NADIA_FP64)
        plain_convolve(support.p, 3, 5);
    else
        f32->soften_support();
    h_support_valid = false;
}

// FresnelCDI::set_norm, FresnelCDI.c++:139-148
void Solver::fresnel_set_norm(double nn)
{
    AllocScope scope(st);
    NADIA_REQUIRE(kind == NADIA_FRESNEL, NADIA_ERR_INVALID, "set_norm needs a FresnelCDI handle");
    ++weights_version;
    double old = norm;
    norm = nn;
    double f = nn / old;
    for (size_t k = 0; k < 2 * n; ++k) h_illum[k] *= f;
    if (prec == NADIA_FP64) {
        plain::scale(illum.p, f, n, st);
        plain::scale(illum_sample.p, f, n, st);
    } else {
        f32->scale_illumination(f);
    }
}

// FresnelCDI::auto_set_norm, FresnelCDI.c++:129-137
void Solver::fresnel_auto_set_norm()
{
    AllocScope scope(st);
    NADIA_REQUIRE(kind == NADIA_FRESNEL, NADIA_ERR_INVALID,
                  "auto_set_norm needs a FresnelCDI handle");
    double wf_norm = 0, int_norm = 0;
    for (size_t k = 0; k < n; ++k)
        wf_norm += sqrt(h_illum[2 * k] * h_illum[2 * k] + h_illum[2 * k + 1] * h_illum[2 * k + 1]);
    for (size_t k = 0; k < n; ++k) int_norm += h_isqrt[k];
    fresnel_set_norm(int_norm / wf_norm);
}

// --------------------------------------------------------------- algorithm

// BaseCDI::set_algorithm, BaseCDI.c++:192-237
void Solver::set_algorithm(int alg)
{
    AllocScope scope(st);
    if (algorithm == alg) return;
    double b = beta;
    double m[10] = {0};
    bool known = true;
    switch (alg) {
    case NADIA_ER: break;
    case NADIA_BIO: m[1] = b; break;
    case NADIA_BOO: m[1] = b; m[8] = 1; break;
    case NADIA_HIO: m[1] = b; m[2] = 1; break;
    case NADIA_DM: m[0] = b; m[2] = 1; m[4] = 1; break;
    case NADIA_SF: m[1] = 1; m[3] = 1; break;
    case NADIA_ASR: m[1] = 1; m[2] = 1; break;
    case NADIA_HPR: m[1] = b; m[2] = 1; break;
    case NADIA_RAAR: m[1] = 1; m[2] = b; m[8] = (1 - b); break;
    default: known = false; // "Algorithm unknown": weights unchanged
    }
    if (known) set_custom(m);
    algorithm = alg;
}

// BaseCDI::set_custom_algorithm, BaseCDI.c++:240-255
void Solver::set_custom(const double m[10])
{
    AllocScope scope(st);
    w[PSF] = m[0] + m[1] + m[2] + m[3];
    w[PFS] = -m[0] + m[4] + m[5] + m[6];
    w[PS] = -m[2] - m[5] - m[7] + m[9];
    w[PF] = -m[1] - m[4] + m[7] + m[8];
    w[PI] = -m[3] - m[6] - m[8] - m[9];
    algorithm = NADIA_CUSTOM;
}

// BaseCDI::set_relaxation_parameter, BaseCDI.h:264-267
void Solver::set_relaxation_parameter(double b)
{
    AllocScope scope(st);
    beta = b;
    set_algorithm(algorithm);
}

// ---------------------------------------------------------------- estimate

// PlanarCDI.c++:39-62 / PolyCDI.c++:102-126 / FresnelCDI.c++:152-201
void Solver::initialise_estimate(int seed)
{
    AllocScope scope(st);
    std::vector<double> h(2 * n, 0.0);
    GlibcRand rnd(seed);
    if (kind == NADIA_FRESNEL) {
        for (size_t k = 0; k < n; ++k) {
            double real = 1 - 0.2 * rnd() / ((double)RAND_MAX);
            h[2 * k] = real;
            h[2 * k + 1] = 0;
        }
        if (prec == NADIA_FP64) {
            DevBuf<double2> t(n);
            h2d(t.p, h.data(), t.bytes(), st);
            plain::fresnel_set_transmission(t.p, illum_sample.p, x.p, nx, ny, st);
            plain_apply_support(x.p); // FresnelCDI.c++:199 (apply_support)
            sync();
        } else {
            f32->fresnel_initialise(h.data());
        }
        return;
    }
    if (!h_support_valid) {
        get_support(h_support.data());
    }
    if (kind == NADIA_FRESNEL_WF) {
        // FresnelCDI_WF::initialise_estimate, FresnelCDI_WF.c++:134-152: sqrt(I)
        // inside the support, 0 outside (the seed is not used)
        for (size_t k = 0; k < n; ++k) {
            h[2 * k] = h_support[k] ? h_isqrt[k] : 0;
            h[2 * k + 1] = 0;
        }
        set_esw(h.data());
        return;
    }
    int max_value = (int)host_max(h_isqrt.data(), n);
    for (size_t k = 0; k < n; ++k) {
        if (!h_support[k]) {
            h[2 * k] = 0;
            h[2 * k + 1] = 0;
        } else {
            // `max_value*rand()` is an int product that wraps modulo 2^32
            int p1 = (int)((unsigned)max_value * (unsigned)rnd());
            double r = h_support[k] * (p1 / (double)RAND_MAX);
            int p2 = (int)((unsigned)max_value * (unsigned)rnd());
            double im = h_support[k] * (p2 / (double)RAND_MAX);
            h[2 * k] = r;
            h[2 * k + 1] = im;
        }
    }
    set_esw(h.data());
}

void Solver::set_esw(const double *h)
{
    AllocScope scope(st);
    if (prec == NADIA_FP64)
        h2d(x.p, h, n * sizeof(double2), st);
    else
        f32->set_x(h);
}

void Solver::get_esw(double *h)
{
    AllocScope scope(st);
    if (prec == NADIA_FP64)
        d2h(h, x.p, n * sizeof(double2), st);
    else
        f32->get_x(h);
}

void Solver::set_esw_f32(const float *h)
{
    AllocScope scope(st);
    if (prec == NADIA_FP32) {
        f32->set_x_f32(h);
        return;
    }
    std::vector<double> d(2 * n);
    for (size_t k = 0; k < 2 * n; ++k) d[k] = h[k];
    set_esw(d.data());
}

void Solver::get_esw_f32(float *h)
{
    AllocScope scope(st);
    if (prec == NADIA_FP32) {
        f32->get_x_f32(h);
        return;
    }
    std::vector<double> d(2 * n);
    get_esw(d.data());
    for (size_t k = 0; k < 2 * n; ++k) h[k] = (float)d[k];
}

void Solver::set_transmission(const double *h)
{
    AllocScope scope(st);
    if (kind != NADIA_FRESNEL) {
        set_esw(h);
        return;
    }
    if (prec == NADIA_FP64) {
        DevBuf<double2> t(n);
        h2d(t.p, h, t.bytes(), st);
        plain::fresnel_set_transmission(t.p, illum_sample.p, x.p, nx, ny, st);
        sync();
    } else {
        f32->fresnel_set_transmission(h);
    }
}

void Solver::get_transmission(double *h)
{
    AllocScope scope(st);
    if (kind != NADIA_FRESNEL) {
        get_esw(h);
        return;
    }
    if (prec == NADIA_FP64) {
        DevBuf<double2> t(n);
        plain::fresnel_get_transmission(x.p, illum_sample.p, t.p, n, st);
        if (tc.active) apply_transmission_constraint(t.p); // FresnelCDI.c++:352-353
        d2h(h, t.p, t.bytes(), st);
    } else {
        f32->fresnel_get_transmission(h);
    }
}

void Solver::transmission_to_device(double2 *dst)
{
    AllocScope scope(st);
    if (prec == NADIA_FP32) {
        NADIA_REQUIRE(kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                      "PolyCDI phase-diverse frames run in the FP64 form");
        f32->transmission_to_device(dst);
        return;
    }
    if (kind == NADIA_FRESNEL) {
        plain::fresnel_get_transmission(x.p, illum_sample.p, dst, n, st);
        if (tc.active) apply_transmission_constraint(dst); // FresnelCDI.c++:352-353
    } else {
        NADIA_CUDA(cudaMemcpyAsync(dst, x.p, n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
    }
}

void Solver::transmission_from_device(const double2 *src)
{
    AllocScope scope(st);
    if (prec == NADIA_FP32) {
        NADIA_REQUIRE(kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                      "PolyCDI phase-diverse frames run in the FP64 form");
        f32->transmission_from_device(src);
        return;
    }
    if (kind == NADIA_FRESNEL)
        plain::fresnel_set_transmission(src, illum_sample.p, x.p, nx, ny, st);
    else
        NADIA_CUDA(cudaMemcpyAsync(x.p, src, n * sizeof(double2), cudaMemcpyDeviceToDevice, st));
}

void Solver::convert_to_fp64()
{
    AllocScope scope(st);
    if (prec == NADIA_FP64) return;
    ++weights_version;
    // read the FP32 state back
    std::vector<double> xh(2 * n), sup(n);
    f32->get_x(xh.data());
    get_support(sup.data());
    std::vector<std::vector<double>> best(n_best);
    for (int i = 0; i < n_best; ++i) {
        std::vector<float> f(2 * n);
        d2h(f.data(), best32[i].p, n * sizeof(float2), st);
        best[i].assign(f.begin(), f.end());
    }
    forget_batches_with(uid); // batch plans hold FP32 handles only
    NADIA_CUDA(cudaStreamSynchronize(st));
    const bool had_tc = tc.active;
    const int tcu = tc.unity, tcf = tc.flip, tcs = tc.flip_sign;
    tc.active = false;
    f32.reset();
    best32.clear();
    prec = NADIA_FP64;
    // the FP64 buffers, as the constructor makes them
    x.alloc(n);
    support.alloc(n);
    isqrt.alloc(n);
    recon.alloc(n);
    tmp.alloc(n);
    fft.init(nx, ny);
    gauss_width_ = -1;
    gauss_cut_ = -1;
    h2d(x.p, xh.data(), n * sizeof(double2), st);
    h_support = sup;
    h_support_valid = true;
    h2d(support.p, h_support.data(), n * sizeof(double), st);
    h2d(isqrt.p, h_isqrt.data(), n * sizeof(double), st);
    if (has_beam_stop) {
        beam_stop.alloc(n);
        h2d(beam_stop.p, h_beam_stop.data(), n * sizeof(double), st);
    }
    for (int i = 0; i < n_best; ++i) {
        best64.emplace_back(n);
        h2d(best64.back().p, best[i].data(), n * sizeof(double2), st);
    }
    if (kind == NADIA_FRESNEL) {
        illum.alloc(n);
        illum_sample.alloc(n);
        coef.alloc((size_t)(nx / 2) * (ny / 2));
        h2d(illum.p, h_illum.data(), illum.bytes(), st);
        fresnel_set_experimental_parameters(wavelength, zfd, zfs, pixel);
    }
    if (kind == NADIA_POLY && has_spectrum) {
        d_spec.alloc(2 * (size_t)nlambda);
        h2d(d_spec.p, spectrum.data(), d_spec.bytes(), st);
        padded.alloc((size_t)(nx + 2 * px) * (ny + 2 * py));
        isc.alloc(n);
        fft_pad.init(nx + 2 * px, ny + 2 * py);
    }
    if (had_tc) set_transmission_constraint(tcu, tcf, tcs, 0, nullptr, nullptr, nullptr);
    NADIA_CUDA(cudaStreamSynchronize(st));
}

void Solver::get_illumination_at_sample(double *h)
{
    AllocScope scope(st);
    NADIA_REQUIRE(kind == NADIA_FRESNEL, NADIA_ERR_INVALID, "needs a FresnelCDI handle");
    if (prec == NADIA_FP64)
        d2h(h, illum_sample.p, n * sizeof(double2), st);
    else
        f32->get_illumination_at_sample(h);
}

// ------------------------------------------------------------ plain FP64 path

// the gather target of the quadrant swap on odd grids (allocated once, on
// this reconstruction's stream; null for even grids)
double2 *Solver::odd_scratch()
{
    if (!((nx | ny) & 1)) return nullptr;
    if (!odd_tmp) {
        AllocScope scope(st);
        odd_tmp.alloc(n);
    }
    return odd_tmp.p;
}

void Solver::plain_propagate_to(double2 *c, bool pg)
{
    AllocScope scope(st);
    if (kind == NADIA_FRESNEL_WF) {
        // FresnelCDI_WF::propagate_to_detector, FresnelCDI_WF.c++:176-182
        fft.exec(c, true, st);
        plain::invert_factors(c, coef.p, nx, ny, -1, true, st); // factors, then the swap
        fft.exec(c, true, st);
    } else if (kind == NADIA_FRESNEL) {
        // FresnelCDI::propagate_to_detector, FresnelCDI.c++:245-250
        plain::invert(c, nx, ny, true, st);
        fft.exec(c, true, st);
        plain::multiply_factors(c, coef.p, nx, ny, -1, st);
    } else if (pg) {
        // PolyCDI::propagate_to_detector, PolyCDI.c++:389-394 (padded grid)
        fft_pad.exec(c, true, st);
        plain::invert(c, nx + 2 * px, ny + 2 * py, true, st);
    } else {
        // PlanarCDI::propagate_to_detector, PlanarCDI.c++:65-68
        fft.exec(c, true, st);
        plain::invert(c, nx, ny, true, st, odd_scratch());
    }
}

void Solver::plain_propagate_from(double2 *c, bool pg)
{
    AllocScope scope(st);
    if (kind == NADIA_FRESNEL_WF) {
        // FresnelCDI_WF::propagate_from_detector, FresnelCDI_WF.c++:165-173
        fft.exec(c, false, st);
        plain::invert_factors(c, coef.p, nx, ny, +1, false, st); // the swap, then factors
        fft.exec(c, false, st);
    } else if (kind == NADIA_FRESNEL) {
        // FresnelCDI::propagate_from_detector, FresnelCDI.c++:238-243
        plain::multiply_factors(c, coef.p, nx, ny, +1, st);
        fft.exec(c, false, st);
        plain::invert(c, nx, ny, true, st);
    } else if (pg) {
        plain::invert(c, nx + 2 * px, ny + 2 * py, true, st);
        fft_pad.exec(c, false, st);
    } else {
        // PlanarCDI::propagate_from_detector, PlanarCDI.c++:70-73
        plain::invert(c, nx, ny, true, st, odd_scratch());
        fft.exec(c, false, st);
    }
}

void Solver::plain_scale(double2 *c)
{
    AllocScope scope(st);
    if (kind == NADIA_FRESNEL) {
        // FresnelCDI::scale_intensity, FresnelCDI.c++:217-236
        plain::add_scaled(c, illum.p, 1.0, n, st);
        plain::scale_intensity(c, isqrt.p, bs_ptr(), n, partials.p, d_err.p, st);
        plain::add_scaled(c, illum.p, -1.0, n, st);
    } else if (kind == NADIA_POLY) {
        // PolyCDI::scale_intensity, PolyCDI.c++:255-292 (padded field)
        plain::poly_expand(c, d_spec.p, nlambda, lambdac, nx, ny, px, py, isc.p, st);
        plain::poly_scale(c, isc.p, isqrt.p, bs_ptr(), nx, ny, px, py, partials.p, d_err.p, st);
    } else {
        plain::scale_intensity(c, isqrt.p, bs_ptr(), n, partials.p, d_err.p, st);
    }
}

// BaseCDI::project_intensity, BaseCDI.c++:156-160; PolyCDI wraps each
// projection in get_padded / get_unpadded (PolyCDI.c++:143-152, 175-181)
void Solver::plain_project(double2 *c)
{
    AllocScope scope(st);
    if (kind == NADIA_POLY) {
        plain::pad(c, nx, ny, padded.p, px, py, st);
        plain_propagate_to(padded.p, true);
        plain_scale(padded.p);
        plain_propagate_from(padded.p, true);
        plain::unpad(padded.p, nx, ny, px, py, c, st);
    } else if (kind == NADIA_PLANAR && nx % 2 == 0 && ny % 2 == 0) {
        // propagate_to, scale_intensity, propagate_from with the element-wise
        // steps between the transforms in one kernel (the swap pairs of an
        // even grid)
        fft.exec(c, true, st);
        plain::detector_planar(c, isqrt.p, bs_ptr(), nx, ny, partials.p, d_err.p, st);
        fft.exec(c, false, st);
    } else if (kind == NADIA_FRESNEL) {
        plain::invert(c, nx, ny, true, st);
        fft.exec(c, true, st);
        plain::detector_fresnel(c, coef.p, illum.p, isqrt.p, bs_ptr(), nx, ny, partials.p,
                                d_err.p, st);
        fft.exec(c, false, st);
        plain::invert(c, nx, ny, true, st);
    } else {
        plain_propagate_to(c, false);
        plain_scale(c);
        plain_propagate_from(c, false);
    }
}

// reallocate_temp_complex_memory, BaseCDI.c++:257-275
void Solver::ensure_temps()
{
    AllocScope scope(st);
    if (w[PFS] != 0 && !tPFS) tPFS.alloc(n);
    if (w[PF] != 0 && !tPF) tPF.alloc(n);
    if (w[PS] != 0 && !tPS) tPS.alloc(n);
    if (w[PSF] != 0 && !tPSF) tPSF.alloc(n);
}

// BaseCDI::iterate, BaseCDI.c++:297-387; PolyCDI::iterate, PolyCDI.c++:130-250
void Solver::plain_iterate_once()
{
    AllocScope scope(st);
    const size_t nb = n * sizeof(double2);
    if (kind == NADIA_FRESNEL_WF) {
        // FresnelCDI_WF::iterate, FresnelCDI_WF.c++:155-162: a fixed algorithm
        plain_propagate_from(x.p, false);
        plain_apply_support(x.p);
        plain_propagate_to(x.p, false);
        plain_scale(x.p);
        return;
    }
    if (algorithm == NADIA_ER) {
        plain_project(x.p);
        plain_apply_support(x.p);
        return;
    }
    if (!tc.active && w[PFS] == 0 && (w[PSF] == 0 || w[PF] != 0)) {
        // the support projections formed inside the combine (same arithmetic)
        const bool pf = w[PF] != 0;
        if (pf) {
            if (!tPF) tPF.alloc(n);
            NADIA_CUDA(cudaMemcpyAsync(tPF.p, x.p, nb, cudaMemcpyDeviceToDevice, st));
            plain_project(tPF.p);
        }
        plain::combine_support(x.p, pf ? tPF.p : nullptr, support.p, w[PS] != 0, w[PSF] != 0,
                               w, n, st);
        return;
    }
    ensure_temps();
    if (w[PFS] != 0) {
        NADIA_CUDA(cudaMemcpyAsync(tPFS.p, x.p, nb, cudaMemcpyDeviceToDevice, st));
        plain_apply_support(tPFS.p);
        plain_project(tPFS.p);
    }
    if (w[PF] != 0) {
        NADIA_CUDA(cudaMemcpyAsync(tPF.p, x.p, nb, cudaMemcpyDeviceToDevice, st));
        plain_project(tPF.p);
    }
    if (w[PS] != 0) {
        NADIA_CUDA(cudaMemcpyAsync(tPS.p, x.p, nb, cudaMemcpyDeviceToDevice, st));
        plain_apply_support(tPS.p);
    }
    if (w[PSF] != 0) {
        if (w[PF] != 0) {
            NADIA_CUDA(cudaMemcpyAsync(tPSF.p, tPF.p, nb, cudaMemcpyDeviceToDevice, st));
            plain_apply_support(tPSF.p);
        } else {
            NADIA_CUDA(cudaMemcpyAsync(tPSF.p, x.p, nb, cudaMemcpyDeviceToDevice, st));
            plain_project(tPSF.p);
            plain_apply_support(tPSF.p);
        }
    }
    plain::combine(x.p, w[PFS] != 0 ? tPFS.p : nullptr, w[PF] != 0 ? tPF.p : nullptr,
                   w[PS] != 0 ? tPS.p : nullptr, w[PSF] != 0 ? tPSF.p : nullptr, w, n, st);
}

void Solver::record_error()
{
    NADIA_CUDA(cudaMemcpyAsync(d_ring.p + (iters % kRing), d_err.p, sizeof(double),
                               cudaMemcpyDeviceToDevice, st));
    ++iters;
}

// BaseCDI::update_n_best, BaseCDI.c++:390-413
void Solver::update_n_best()
{
    AllocScope scope(st);
    if (n_best <= 0) return;
    double cur = get_error();
    int place = 0;
    for (; place < n_best && cur > best_err[place]; place++)
        ;
    if (place < n_best) {
        int slot = best_slot[n_best - 1];
        if (prec == NADIA_FP64)
            NADIA_CUDA(cudaMemcpyAsync(best64[slot].p, x.p, n * sizeof(double2),
                                       cudaMemcpyDeviceToDevice, st));
        else
            f32->copy_x_to(best32[slot].p);
        for (int i = n_best - 1; i > place; i--) {
            best_err[i] = best_err[i - 1];
            best_slot[i] = best_slot[i - 1];
        }
        best_err[place] = cur;
        best_slot[place] = slot;
    }
}

void Solver::iterate(int count)
{
    AllocScope scope(st);
    NADIA_REQUIRE(count >= 0, NADIA_ERR_INVALID, "negative iteration count");
    require_poly_ready();
    if (prec == NADIA_FP32 && n_best == 0) {
        f32->iterate(count);
        return;
    }
    for (int it = 0; it < count; ++it) {
        if (prec == NADIA_FP64)
            plain_iterate_once();
        else
            f32->iterate(1);
        if (prec == NADIA_FP64) record_error();
        if (kind != NADIA_FRESNEL_WF) update_n_best(); // FresnelCDI_WF::iterate keeps none

    }
    NADIA_CUDA(cudaGetLastError());
}

double Solver::get_error()
{
    AllocScope scope(st);
    double e = 0;
    d2h(&e, d_err.p, sizeof(double), st);
    if (f32) f32->check_device_flag();
    return e;
}

void Solver::get_error_history(double *out, int count)
{
    AllocScope scope(st);
    NADIA_REQUIRE(count >= 0 && count <= kRing && count <= iters, NADIA_ERR_RANGE,
                  "fewer iterations recorded than requested");
    std::vector<double> ring(kRing);
    d2h(ring.data(), d_ring.p, d_ring.bytes(), st);
    for (int i = 0; i < count; ++i) out[i] = ring[(size_t)((iters - count + i) % kRing)];
}

// BaseCDI::apply_shrinkwrap, BaseCDI.c++:416-429
void Solver::apply_shrinkwrap(double gauss_width, double thresh)
{
    AllocScope scope(st);
    ++weights_version;
    if (prec == NADIA_FP32) {
        f32->shrinkwrap(gauss_width, thresh);
        h_support_valid = false;
        return;
    }
    plain::magnitude(x.p, recon.p, n, st);
    plain_convolve(recon.p, gauss_width, 4);
    plain::max_reduce(recon.p, n, partials.p, dmax.p, st);
    plain::threshold(recon.p, nx, ny, thresh, dmax.p, st);
    plain::max_reduce(recon.p, n, partials.p, dmax.p + 1, st);
    plain::divide_by_max(recon.p, support.p, n, dmax.p + 1, st);
    h_support_valid = false;
    NADIA_CUDA(cudaGetLastError());
}

void Solver::get_support(double *h)
{
    AllocScope scope(st);
    if (h_support_valid) {
        if (h != h_support.data()) std::memcpy(h, h_support.data(), n * sizeof(double));
        return;
    }
    if (prec == NADIA_FP64)
        d2h(h, support.p, n * sizeof(double), st);
    else
        f32->get_support(h);
    if (h != h_support.data()) std::memcpy(h_support.data(), h, n * sizeof(double));
    h_support_valid = true;
}

// BaseCDI::get_best_result, BaseCDI.c++:82-91
void Solver::get_best(int index, double *err, double *h)
{
    AllocScope scope(st);
    NADIA_REQUIRE(index >= 0 && index < n_best, NADIA_ERR_RANGE,
                  "index out of bounds in get_best_result");
    *err = best_err[index];
    int slot = best_slot[index];
    if (prec == NADIA_FP64) {
        d2h(h, best64[slot].p, n * sizeof(double2), st);
    } else {
        std::vector<float> f(2 * n);
        d2h(f.data(), best32[slot].p, n * sizeof(float2), st);
        for (size_t k = 0; k < 2 * n; ++k) h[k] = f[k];
    }
}

void Solver::reset_best()
{
    AllocScope scope(st);
    for (int i = 0; i < n_best; ++i) best_err[i] = 1;
}

// single operators on a caller's field (IDL_interface.c:947-985)
void Solver::single_op(int op, double *field)
{
    AllocScope scope(st);
    NADIA_REQUIRE(kind != NADIA_POLY, NADIA_ERR_UNSUPPORTED,
                  "single operators act on the unpadded grid (PLANAR, FRESNEL)");
    if (prec == NADIA_FP32) {
        f32->single_op(op, field);
        return;
    }
    DevBuf<double2> c(n);
    h2d(c.p, field, c.bytes(), st);
    switch (op) {
    case 0: plain_propagate_to(c.p, false); break;
    case 1: plain_propagate_from(c.p, false); break;
    case 2: plain_scale(c.p); break;
    case 3: plain_apply_support(c.p); break;
    case 4: plain_project(c.p); break;
    default: throw Error(NADIA_ERR_INVALID, "unknown operator");
    }
    d2h(field, c.p, c.bytes(), st);
}

// PlanarCDI::get_intensity_autocorrelation, PlanarCDI.c++:13-36
void Solver::autocorrelation(double *out)
{
    AllocScope scope(st);
    NADIA_REQUIRE(kind == NADIA_PLANAR, NADIA_ERR_INVALID, "needs a PlanarCDI handle");
    if (prec == NADIA_FP32) {
        f32->autocorrelation(out);
        return;
    }
    DevBuf<double2> t(n);
    DevBuf<double> m(n);
    plain::autocorr_fill(isqrt.p, t.p, n, st);
    fft.exec(t.p, false, st);
    plain::invert(t.p, nx, ny, true, st, odd_scratch());
    plain::magnitude(t.p, m.p, n, st);
    d2h(out, m.p, m.bytes(), st);
}

} // namespace nadia
