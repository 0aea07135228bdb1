// solver.h -- one reconstruction (the state of one PlanarCDI / FresnelCDI /
// PolyCDI object) resident on a CUDA device.  The algorithm bookkeeping
// (weights, relaxation quirk, n-best ranking, error history) lives here on
// the host; the arithmetic runs in the plain FP64 kernels (plain64.cu) or
// the fused FP32 engine (fused32.cu).
#pragma once

#include <memory>
#include <vector>

#include "common.h"
#include "plain64.h"

namespace nadia {

class Fused32;

enum { PSF = 0, PFS = 1, PS = 2, PF = 3, PI = 4 }; // BaseCDI.h:76

struct Solver {
    int kind = NADIA_PLANAR, nx = 0, ny = 0, prec = NADIA_FP64, n_best = 0;
    size_t n = 0;
    int device = 0;
    unsigned long long uid = 0; // unique per handle (batch plans key on it)
    int pd_refs = 0;            // phase-diverse reconstructions holding this one as a frame
    // bumped whenever the support or the Fresnel illumination changes (the
    // inputs of a phase-diverse object's weights)
    unsigned long long weights_version = 0;
    OwnedStream own_st;         // outlives every buffer below
    cudaStream_t st = nullptr;

    // algorithm state (BaseCDI.h:87-150)
    double beta = 0.9;
    int algorithm = NADIA_CUSTOM;
    double w[5] = {0, 0, 0, 0, 0};

    // host copies used by initialise_estimate and auto_set_norm
    std::vector<double> h_isqrt;
    std::vector<double> h_support;
    bool h_support_valid = true;
    bool has_beam_stop = false;
    std::vector<double> h_beam_stop; // the mask as given (kept for convert_to_fp64)

    // error history: one slot per iteration on the device
    static constexpr int kRing = 65536;
    long long iters = 0;
    DevBuf<double> d_err;     // [0] current error
    DevBuf<double> d_ring;    // kRing errors
    DevBuf<double> partials;  // reduction scratch

    // n-best (BaseCDI.c++:43-50, 390-413): slot buffers, rank order, errors
    std::vector<DevBuf<double2>> best64;
    std::vector<DevBuf<float2>> best32;
    std::vector<int> best_slot;
    std::vector<double> best_err;

    // FP64 device state
    DevBuf<double2> x, tPFS, tPF, tPS, tPSF;
    DevBuf<double2> odd_tmp;  // odd grids: the quadrant swap's gather target
    double2 *odd_scratch();
    DevBuf<double> support, isqrt, beam_stop;
    plain::Fft2d fft;
    DevBuf<double> recon, tmp, gauss, dmax;
    double gauss_width_ = -1; // the blur table now in `gauss`
    int gauss_cut_ = -1;

    // FresnelCDI
    std::vector<double> h_illum; // detector white field x norm (interleaved)
    double norm = 1, wavelength = 0, zfd = 0, zfs = 0, pixel = 0;
    double z12 = 0, z23 = 0; // FresnelCDI_WF: zone plate to focus, focus to detector
    DevBuf<double2> illum, illum_sample, coef;

    // PolyCDI
    std::vector<double> spectrum; // (wavelength, normalised weight) rows
    int nlambda = 0, px = 0, py = 0;
    double lambdac = 0;
    bool has_spectrum = false;
    DevBuf<double> d_spec, isc;
    DevBuf<double2> padded;
    plain::Fft2d fft_pad;

    // TransmissionConstraint set by BaseCDI::set_complex_constraint (FP64 form)
    struct TransConstraint {
        bool active = false;
        int unity = 0, flip = 0, flip_sign = 1, nregions = 0;
        DevBuf<int> region;       // n: 0 or the 1-based region of each pixel
        DevBuf<double> params;    // per region: alpha1, alpha2, c fixed?, fixed c
        DevBuf<double> partials;  // region sums per reduction block
        DevBuf<double> cmean;     // per region
        DevBuf<double2> tbuf;     // FresnelCDI: the transmission function being constrained
        void (*custom)(double *, int, int, void *) = nullptr;
        void *user = nullptr;
    } tc;

    std::unique_ptr<Fused32> f32;

    Solver(int kind, int nx, int ny, int prec, int n_best);
    ~Solver();

    // inputs
    void set_support(const double *obj, bool soften);
    void set_intensity(const double *I);
    void set_beam_stop(const double *mask);
    void set_spectrum(const double *wl_weight, int nl);
    void fresnel_init(const double *white_field, double wl, double zfd, double zfs, double pixel,
                      double norm);
    void fresnel_set_experimental_parameters(double wl, double zfd, double zfs, double pixel);
    void fresnel_set_norm(double nn);
    void fresnel_auto_set_norm();
    void fresnel_wf_init(double wl, double zone_focal, double focal_detector, double pixel);
    void fresnel_wf_set_support(double z_diameter, double size);
    void set_transmission_constraint(int unity, int flip, int flip_sign, int nregions,
                                     const double *regions, const double *alpha,
                                     const double *fixed_c);
    void set_transmission_custom(void (*fn)(double *, int, int, void *), void *user);
    void clear_transmission_constraint();

    // algorithm
    void set_algorithm(int alg);
    void set_custom(const double m[10]);
    void set_relaxation_parameter(double b);

    // estimate
    void initialise_estimate(int seed);
    void set_esw(const double *h);
    void get_esw(double *h);
    void set_esw_f32(const float *h);
    void get_esw_f32(float *h);
    void set_transmission(const double *h);
    void get_transmission(double *h);
    void get_illumination_at_sample(double *h);

    // run
    void iterate(int count);
    double get_error();
    void get_error_history(double *out, int count);
    void apply_shrinkwrap(double gauss_width, double threshold);
    void get_support(double *h);
    void get_best(int index, double *err, double *h);
    void reset_best();
    void single_op(int op, double *field);
    void autocorrelation(double *out);
    void sync();

    // FP64 plain path internals
    void plain_iterate_once();
    void plain_project(double2 *c);
    void plain_propagate_to(double2 *c, bool padded_grid);
    void plain_propagate_from(double2 *c, bool padded_grid);
    void plain_scale(double2 *c);
    void plain_convolve(double *arr, double gauss_width, int cut);
    void plain_apply_support(double2 *c);
    void apply_transmission_constraint(double2 *t);

    // The result a PhaseDiverseCDI exchanges with this reconstruction
    // (PhaseDiverseCDI.c++:330-345), device to device and ordered on st:
    // FresnelCDI's transmission function (get_transmission_function with its
    // constraint, set_transmission_function), else the exit-surface wave.
    // FP64 form only.
    void transmission_to_device(double2 *dst);
    void transmission_from_device(const double2 *src);

    // Moves an FP32 reconstruction to the FP64 form in place: the estimate,
    // support, intensity, beam stop, illumination and geometry, spectrum,
    // algorithm, error history and n-best results carry over (FP32 values
    // widened); later iterations run the plain FP64 path.  No-op on FP64.
    void convert_to_fp64();
    void ensure_temps();
    void update_n_best();
    void record_error();
    void require_poly_ready() const;
    const double *bs_ptr() const { return has_beam_stop ? beam_stop.p : nullptr; }
    std::vector<double> gauss_table(double gauss_width, int cut) const;
    void upload_support();
};

// read_spec semantics (NADIA/src/io_spec.c:61-133): rows of (1/energy, weight).
std::vector<double> read_spec_file(const char *path);

} // namespace nadia
