// plain64.h -- the plain FP64 path: one kernel per loop of the reference
// (NADIA/src/Complex_2D.c++, BaseCDI.c++, PlanarCDI.c++, FresnelCDI.c++,
// PolyCDI.c++), each performing the same sequence of IEEE-754 double
// operations per element as the reference's double build, so results agree
// bit for bit except for the order of the error-metric sums.  plain64.cu is
// compiled with --fmad=false so no multiply-add is contracted.
#pragma once

#include "common.h"

namespace nadia {
namespace plain {

// Number of blocks used by the two-stage reductions (fixed, so the summation
// order is the same on every call).
constexpr int kRedBlocks = 592;

// In-place unnormalised 2-D DFT of an nx-by-ny row-major double2 array with
// the canonical Stockham schedule: every row (length ny), then every column.
struct Fft2d {
    int nx = 0, ny = 0;
    FftPlan px{}, py{};
    DevBuf<double2> wx, wy;
    int rows_per_block = 1, cols_per_block = 1;
    size_t row_smem = 0, col_smem = 0;
    bool row_one = false, col_one = false; // radix-2/4/8 plans: the one-buffer kernels
    bool col_wide = false;                 // columns of 2048 points and more: 512 threads
    void init(int nx, int ny);
    void exec(double2 *a, bool forward, cudaStream_t s) const;
};

// Complex_2D::invert(scale), Complex_2D.c++:318-353 (even sizes).
// scratch: nx*ny values, needed for odd sizes (the swap loop's replay is a
// gather into it), unused otherwise
void invert(double2 *a, int nx, int ny, bool scale, cudaStream_t s, double2 *scratch = nullptr);

// BaseCDI::scale_intensity, BaseCDI.c++:163-189.  beam_stop may be null.
// Writes diff/mag to *err (device).
void scale_intensity(double2 *c, const double *isqrt, const double *beam_stop, size_t n,
                     double *partials, double *err, cudaStream_t s);

// BaseCDI::support_constraint, BaseCDI.c++:136-154.
void support_constraint(double2 *c, const double *support, size_t n, cudaStream_t s);

// The combine loop of BaseCDI::iterate, BaseCDI.c++:346-383.  Null term
// pointers are skipped, as the reference skips zero weights.
void combine(double2 *x, const double2 *pfs, const double2 *pf, const double2 *ps,
             const double2 *psf, const double w[5], size_t n, cudaStream_t s);

// The combine with Ps and PsPf formed on the fly from the support (valid
// without a transmission constraint and without the PfPs term); pf may be
// null (no Pf term, and then no PsPf term).
void combine_support(double2 *x, const double2 *pf, const double *support, bool use_ps,
                     bool use_psf, const double w[5], size_t n, cudaStream_t s);

// The detector side of project_intensity between its two transforms, one
// kernel each: PlanarCDI invert -> scale_intensity -> invert (PlanarCDI.c++:
// 65-73); FresnelCDI multiply_factors -> add(W) -> scale_intensity ->
// add(-W) -> multiply_factors (FresnelCDI.c++:217-250).  Error to *err.
void detector_planar(double2 *c, const double *isqrt, const double *bs, int nx, int ny,
                     double *partials, double *err, cudaStream_t s);
void detector_fresnel(double2 *c, const double2 *coef, const double2 *ill, const double *isqrt,
                      const double *bs, int nx, int ny, double *partials, double *err,
                      cudaStream_t s);

// invert(scale) and multiply_factors in one pass, the factors applied before
// the swap (factors_first) or after it -- FresnelCDI_WF's propagations.
void invert_factors(double2 *c, const double2 *coef, int nx, int ny, int direction,
                    bool factors_first, cudaStream_t s);

// FresnelCDI::multiply_factors, FresnelCDI.c++:98-126 (quarter table coef).
void multiply_factors(double2 *c, const double2 *coef, int nx, int ny, int direction,
                      cudaStream_t s);

// Complex_2D::add(c2, scale), Complex_2D.c++:184-199.
void add_scaled(double2 *c, const double2 *b, double scale, size_t n, cudaStream_t s);

// Complex_2D::scale, Complex_2D.c++:170-180.
void scale(double2 *c, double f, size_t n, cudaStream_t s);

// get_padded / get_unpadded, Complex_2D.c++:403-460 (zero padding).
void pad(const double2 *x, int nx, int ny, double2 *p, int px, int py, cudaStream_t s);
void unpad(const double2 *p, int nx, int ny, int px, int py, double2 *x, cudaStream_t s);

// PolyCDI::expand_wl, PolyCDI.c++:296-334, evaluated on the central window
// (the only part the reference reads back).  spec: nlambda (wavelength,
// normalised weight) pairs on the device.
void poly_expand(const double2 *c, const double *spec, int nlambda, double lambdac, int nx,
                 int ny, int px, int py, double *isqrt_calc, cudaStream_t s);

// PolyCDI::scale_intensity, PolyCDI.c++:255-292 (c is the padded field).
void poly_scale(double2 *c, const double *isqrt_calc, const double *isqrt,
                const double *beam_stop, int nx, int ny, int px, int py, double *partials,
                double *err, cudaStream_t s);

// get_2d(MAG), Complex_2D.c++:159-165.
void magnitude(const double2 *c, double *out, size_t n, cudaStream_t s);

// BaseCDI::convolve, BaseCDI.c++:432-474.  gauss: (cut+1)^2 table (device).
void convolve(const double *in, double *out, int nx, int ny, const double *gauss, int cut,
              cudaStream_t s);

// Real_2D::get_max, Double_2D.h:252-265 -> *out (device).
void max_reduce(const double *a, size_t n, double *partials, double *out, cudaStream_t s);

// BaseCDI::apply_threshold, BaseCDI.c++:477-492, with its `j < nx` inner
// bound; *dmax is the maximum taken before thresholding.
void threshold(double *a, int nx, int ny, double t, const double *dmax, cudaStream_t s);

// out[k] = in[k] / *dmax (BaseCDI::set_support, BaseCDI.c++:95-102).
void divide_by_max(const double *in, double *out, size_t n, const double *dmax,
                   cudaStream_t s);

// FresnelCDI::set_transmission_function, FresnelCDI.c++:253-283 (with its
// `j < nx` inner bound).
void fresnel_set_transmission(const double2 *t, const double2 *ill, double2 *esw, int nx,
                              int ny, cudaStream_t s);

// FresnelCDI::get_transmission_function, FresnelCDI.c++:298-355.
void fresnel_get_transmission(const double2 *esw, const double2 *ill, double2 *out, size_t n,
                              cudaStream_t s);

// PlanarCDI::get_intensity_autocorrelation, first loop (PlanarCDI.c++:18-25).
void autocorr_fill(const double *isqrt, double2 *t, size_t n, cudaStream_t s);

// TransmissionConstraint::apply_constraint (TransmissionConstraint.c++:76-172)
// on the device.  region[k] is 0 or the 1-based region of pixel k; params
// holds (alpha1, alpha2, c fixed?, fixed c) per region.  Region sums are
// reduced in a fixed order (kRedBlocks blocks, then one thread per region).
constexpr int kMaxRegions = 16;
void transmission_constraint(double2 *t, const int *region, size_t n, int nregions,
                             const double *params, double *partials, double *cmean,
                             int charge_flip, int flip_sign, int enforce_unity, cudaStream_t s);

} // namespace plain
} // namespace nadia
