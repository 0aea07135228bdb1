/*
 * nadia_oracle.c -- TEST INFRASTRUCTURE (oracle). Not part of the product.
 *
 * A plain-C, double-precision restatement of NADIA's phase-retrieval loop
 * (PlanarCDI, FresnelCDI, PolyCDI over BaseCDI), written to follow the
 * reference's sequence of floating-point operations so that it agrees with
 * the reference (compiled in oracle/_ref against the FFTW shim) and with the
 * CUDA FP64 path bit for bit.  Every function cites the reference lines it
 * restates.  Only the tests, the smoke check and the CPU-baseline leg of the
 * benchmark may load this library.
 *
 * Conventions: complex arrays are interleaved (re,im) doubles, real arrays
 * doubles, element (x,y) at index x*ny+y (NADIA/include/Complex_2D.h:179-194).
 * Build with -ffp-contract=off -fno-fast-math.
 *
 * Parity pinning: the FFT is the canonical schedule of canon_fft.h (FFTW is
 * absent; its unnormalised DFT definition is what both sides compute).  The
 * loop itself is pinned against the reference sources compiled with the shim
 * (oracle/build_oracle.py) and against fixtures in tests/golden/.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <ctype.h>
#include "canon_fft.h"

CANON_FFT_DEFINE(d, double)

enum { PSF, PFS, PS, PF, PI_ }; /* NADIA/include/BaseCDI.h:32 (term order) */
enum { ER, BIO, BOO, HIO, DM, SF, ASR, HPR, RAAR, CUSTOM }; /* BaseCDI.h:37 */
enum { KIND_PLANAR = 0, KIND_FRESNEL = 1, KIND_POLY = 2, KIND_FRESNEL_WF = 3 };

/* TransmissionConstraint (NADIA/include/TransmissionConstraint.h:200-375,
 * NADIA/src/TransmissionConstraint.c++) with its ComplexConstraint regions */
typedef struct orc_tc {
    int active;
    int enforce_unity, charge_flip, flip_sign;
    int nregions;
    double *region_map;    /* nx*ny: 0, or the 1-based region that claimed the pixel */
    double *alpha1, *alpha2, *c_mean;
    int *fixed_c;
    void (*custom)(double *t, int nx, int ny, void *user);
    void *user;
} orc_tc;

typedef struct orc_solver {
    int kind, nx, ny;
    double beta;
    double *complex_;      /* the estimate (exit-surface wave), nx*ny*2 */
    double *support;       /* nx*ny */
    double *isqrt;         /* sqrt of the intensity, nx*ny */
    double *beam_stop;     /* NULL = not in use */
    int algorithm;
    double w[5];           /* algorithm_structure[PSF..PI] */
    double current_error;
    int n_best;
    double **best;         /* n_best arrays of nx*ny*2 */
    double *best_err;
    double *tPFS, *tPF, *tPS, *tPSF;
    canon_ctxd *fft;       /* nx-by-ny transform */
    /* FresnelCDI */
    double *illum;         /* detector-plane white field x norm */
    double *illum_sample;  /* illumination propagated to the sample plane */
    double *coef;          /* (nx/2)*(ny/2)*2 quarter table */
    double norm, wavelength, pixel, zfd, zfs;
    /* FresnelCDI_WF: zone-plate-to-focus and focus-to-detector distances */
    double z12, z23;
    /* PolyCDI */
    double *spectrum;      /* nlambda*2: (wavelength, weight) */
    int nlambda, px, py;
    double lambdac;
    double *isqrt_calc;    /* nx*ny */
    canon_ctxd *fft_pad;   /* padded transform */
    int pnx, pny;
    orc_tc tc;
} orc_solver;

static double *zd(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

/* ---------------- Complex_2D helpers (NADIA/src/Complex_2D.c++) ---------------- */

/* get_mag, Complex_2D.h:265-268 */
static inline double mag_of(const double *c) { return sqrt(c[0] * c[0] + c[1] * c[1]); }

/* set_mag, Complex_2D.h:205-215 */
static inline void set_mag(double *c, double value)
{
    double mag = mag_of(c);
    if (mag == 0) {
        c[0] = value;
        c[1] = 0;
    } else {
        c[0] *= value / mag;
        c[1] *= value / mag;
    }
}

/* invert(bool scale), Complex_2D.c++:318-353 (quadrant swap, optional 1/sqrt(nx*ny)) */
static void invert(double *a, int nx, int ny, int scale)
{
    int mx = nx / 2, my = ny / 2;
    double s = 1;
    if (scale) s = 1.0 / (sqrt((double)(nx * ny)));
    for (int i = 0; i < nx; ++i) {
        for (int j = 0; j < my; ++j) {
            int jn = j + my, in = i + mx;
            if (i >= mx) in = in - 2 * mx;
            double *p = a + 2 * ((size_t)in * ny + jn), *q = a + 2 * ((size_t)i * ny + j);
            double tr = p[0], ti = p[1];
            p[0] = q[0] * s;
            p[1] = q[1] * s;
            q[0] = tr * s;
            q[1] = ti * s;
        }
    }
}

/* get_padded, Complex_2D.c++:403-444; the padding is zero (see fftw_shim.c) */
static double *get_padded(const double *a, int nx, int ny, int xa, int ya)
{
    int mx = nx + 2 * xa, my = ny + 2 * ya;
    double *p = zd((size_t)mx * my * 2);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            p[2 * ((size_t)(i + xa) * my + j + ya)] = a[2 * ((size_t)i * ny + j)];
            p[2 * ((size_t)(i + xa) * my + j + ya) + 1] = a[2 * ((size_t)i * ny + j) + 1];
        }
    return p;
}

/* get_unpadded, Complex_2D.c++:447-460 (writes into an nx*ny array) */
static void get_unpadded(const double *p, int mx, int my, int xa, int ya, double *out)
{
    int nx = mx - 2 * xa, ny = my - 2 * ya;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            out[2 * ((size_t)i * ny + j)] = p[2 * ((size_t)(i + xa) * my + j + ya)];
            out[2 * ((size_t)i * ny + j) + 1] = p[2 * ((size_t)(i + xa) * my + j + ya) + 1];
        }
}

/* Real_2D::get_max, Double_2D.h:252-265 */
static double get_max(const double *a, size_t n)
{
    if (n == 0) return 0;
    double m = a[0];
    for (size_t k = 0; k < n; ++k)
        if (a[k] > m) m = a[k];
    return m;
}

/* Real_2D::get_sum, Double_2D.h:210-216 */
static double get_sum(const double *a, size_t n)
{
    double t = 0;
    for (size_t k = 0; k < n; ++k) t += a[k];
    return t;
}

/* ---------------- BaseCDI (NADIA/src/BaseCDI.c++) ---------------- */

/* convolve, BaseCDI.c++:432-474: truncated, unnormalised Gaussian, edge skip */
static void convolve(double *arr, int nx, int ny, double gauss_width, int cut)
{
    double *g = zd((size_t)(cut + 1) * (cut + 1));
    for (int i = 0; i <= cut; ++i)
        for (int j = 0; j <= cut; ++j) {
            double denom = 2.0 * gauss_width * gauss_width;
            g[i * (cut + 1) + j] = exp(-1 * (i * i + j * j) / denom);
        }
    double *tmp = zd((size_t)nx * ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            double nv = 0;
            for (int i2 = i - cut; i2 <= i + cut; ++i2)
                for (int j2 = j - cut; j2 <= j + cut; ++j2)
                    if (i2 < nx && i2 >= 0 && j2 >= 0 && j2 < ny)
                        nv += arr[(size_t)i2 * ny + j2] *
                              g[(int)fabs((double)(i - i2)) * (cut + 1) + (int)fabs((double)(j - j2))];
            tmp[(size_t)i * ny + j] = nv;
        }
    memcpy(arr, tmp, sizeof(double) * (size_t)nx * ny);
    free(tmp);
    free(g);
}

/* Real_2D::get with its (x>nx, y>ny) bound test, Double_2D.h:134-143; an
 * index past the end of the buffer reads as 0 here (undefined in the reference) */
static double real_get(const double *a, int nx, int ny, int x, int y)
{
    if (x < 0 || x > nx) return 0;
    if (y < 0 || y > ny) return 0;
    long long k = (long long)x * ny + y;
    if (k >= (long long)nx * ny) return 0;
    return a[k];
}

/* apply_threshold, BaseCDI.c++:477-492, including its `j < nx` inner bound;
 * writes past the end of the buffer are skipped (undefined in the reference) */
static void apply_threshold(double *a, int nx, int ny, double threshold)
{
    double max = get_max(a, (size_t)nx * ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < nx; ++j) {
            long long k = (long long)i * ny + j;
            double v = real_get(a, nx, ny, i, j) < (threshold * max) ? 0.0 : 1.0;
            if (k < (long long)nx * ny) a[k] = v;
        }
}

/* set_support, BaseCDI.c++:95-108 */
static void set_support_arr(orc_solver *s, const double *obj, int soften)
{
    size_t n = (size_t)s->nx * s->ny;
    double max = get_max(obj, n);
    for (size_t k = 0; k < n; ++k) s->support[k] = obj[k] / max;
    if (soften) convolve(s->support, s->nx, s->ny, 3, 5);
}

/* support_constraint, BaseCDI.c++:136-154 */
static void support_constraint(orc_solver *s, double *c)
{
    size_t n = (size_t)s->nx * s->ny;
    for (size_t k = 0; k < n; ++k) {
        double sv = s->support[k];
        if (sv == 0) {
            c[2 * k] = 0;
            c[2 * k + 1] = 0;
        } else if (sv < 1) {
            c[2 * k] = c[2 * k] * sv;
            c[2 * k + 1] = c[2 * k + 1] * sv;
        }
    }
}

/* BaseCDI::scale_intensity, BaseCDI.c++:163-189 */
static void base_scale_intensity(orc_solver *s, double *c)
{
    double norm2_mag = 0, norm2_diff = 0;
    size_t n = (size_t)s->nx * s->ny;
    for (size_t k = 0; k < n; ++k) {
        if (s->beam_stop == NULL || s->beam_stop[k] > 0) {
            double cis = s->isqrt[k];
            double cm = mag_of(c + 2 * k);
            set_mag(c + 2 * k, cis);
            norm2_mag += cis * cis;
            norm2_diff += (cm - cis) * (cm - cis);
        }
    }
    s->current_error = (norm2_diff / norm2_mag);
}

/* FresnelCDI::multiply_factors, FresnelCDI.c++:98-126 (direction -1 / +1) */
static void multiply_factors(orc_solver *s, double *c, int direction)
{
    int nx = s->nx, ny = s->ny, qy = ny / 2;
    double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            double *p = c + 2 * ((size_t)i * ny + j);
            double old_real = p[0], old_imag = p[1];
            int i_ = (int)(x_mid - fabs(x_mid - i));
            int j_ = (int)(y_mid - fabs(y_mid - j));
            double cr = s->coef[2 * ((size_t)i_ * qy + j_)];
            double ci = direction * s->coef[2 * ((size_t)i_ * qy + j_) + 1];
            p[0] = old_real * cr - old_imag * ci;
            p[1] = old_imag * cr + old_real * ci;
        }
}

static void propagate_to_detector(orc_solver *s, double *c)
{
    if (s->kind == KIND_FRESNEL_WF) {
        /* FresnelCDI_WF::propagate_to_detector, FresnelCDI_WF.c++:176-182 */
        canon_fft2d_execd(s->fft, (canon_cd *)c, 1);
        multiply_factors(s, c, -1);
        invert(c, s->nx, s->ny, 1);
        canon_fft2d_execd(s->fft, (canon_cd *)c, 1);
    } else if (s->kind == KIND_FRESNEL) {
        /* FresnelCDI::propagate_to_detector, FresnelCDI.c++:245-250 */
        invert(c, s->nx, s->ny, 1);
        canon_fft2d_execd(s->fft, (canon_cd *)c, 1);
        multiply_factors(s, c, -1);
    } else if (s->kind == KIND_POLY) {
        /* PolyCDI::propagate_to_detector on the padded grid, PolyCDI.c++:389-394 */
        canon_fft2d_execd(s->fft_pad, (canon_cd *)c, 1);
        invert(c, s->pnx, s->pny, 1);
    } else {
        /* PlanarCDI::propagate_to_detector, PlanarCDI.c++:65-68 */
        canon_fft2d_execd(s->fft, (canon_cd *)c, 1);
        invert(c, s->nx, s->ny, 1);
    }
}

static void propagate_from_detector(orc_solver *s, double *c)
{
    if (s->kind == KIND_FRESNEL_WF) {
        /* FresnelCDI_WF::propagate_from_detector, FresnelCDI_WF.c++:165-173 */
        canon_fft2d_execd(s->fft, (canon_cd *)c, 0);
        invert(c, s->nx, s->ny, 1);
        multiply_factors(s, c, +1);
        canon_fft2d_execd(s->fft, (canon_cd *)c, 0);
    } else if (s->kind == KIND_FRESNEL) {
        /* FresnelCDI::propagate_from_detector, FresnelCDI.c++:238-243 */
        multiply_factors(s, c, +1);
        canon_fft2d_execd(s->fft, (canon_cd *)c, 0);
        invert(c, s->nx, s->ny, 1);
    } else if (s->kind == KIND_POLY) {
        /* PolyCDI.c++:397-402 */
        invert(c, s->pnx, s->pny, 1);
        canon_fft2d_execd(s->fft_pad, (canon_cd *)c, 0);
    } else {
        /* PlanarCDI.c++:70-73 */
        invert(c, s->nx, s->ny, 1);
        canon_fft2d_execd(s->fft, (canon_cd *)c, 0);
    }
}

/* PolyCDI::expand_wl, PolyCDI.c++:296-334 (c is the padded field) */
static void poly_expand_wl(orc_solver *s, const double *c)
{
    int nx = s->nx, ny = s->ny, mx = s->pnx, my = s->pny;
    double *ip = zd((size_t)mx * my);
    for (int sn = 0; sn < s->nlambda; ++sn) {
        double lambda = s->spectrum[2 * sn], weightl = s->spectrum[2 * sn + 1];
        double lf = lambda / s->lambdac;
        for (int i = 0; i < mx; ++i)
            for (int j = 0; j < my; ++j) {
                double xval = lf * (i - nx / 2.0) + nx / 2.0;
                double yval = lf * (j - ny / 2.0) + ny / 2.0;
                if (((xval >= 0) && (xval < mx)) && ((yval >= 0) && (yval < my))) {
                    int xi = (int)xval, yi = (int)yval;
                    double m = mag_of(c + 2 * ((size_t)xi * my + yi));
                    ip[(size_t)i * my + j] = ip[(size_t)i * my + j] + weightl * pow(m, 2);
                }
            }
    }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            s->isqrt_calc[(size_t)i * ny + j] = sqrt(ip[(size_t)(i + s->px) * my + j + s->py]);
    free(ip);
}

/* PolyCDI::scale_intensity, PolyCDI.c++:255-292 (c is the padded field) */
static void poly_scale_intensity(orc_solver *s, double *c)
{
    double norm2_mag = 0, norm2_diff = 0;
    int nx = s->nx, ny = s->ny, my = s->pny;
    poly_expand_wl(s, c);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            size_t k = (size_t)i * ny + j;
            if (s->beam_stop == NULL || s->beam_stop[k] > 0) {
                double calc = s->isqrt_calc[k], meas = s->isqrt[k], scaled;
                double *p = c + 2 * ((size_t)(i + s->px) * my + j + s->py);
                if (calc == 0.0)
                    scaled = 0.0;
                else
                    scaled = mag_of(p) * meas / calc;
                set_mag(p, scaled);
                norm2_mag += meas * meas;
                norm2_diff += (meas - calc) * (meas - calc);
            }
        }
    s->current_error = norm2_diff / norm2_mag;
}

static void scale_intensity(orc_solver *s, double *c)
{
    size_t n = (size_t)s->nx * s->ny;
    if (s->kind == KIND_FRESNEL) {
        /* FresnelCDI::scale_intensity, FresnelCDI.c++:217-236 (Complex_2D::add,
         * Complex_2D.c++:184-199, with scale 1 and -1) */
        for (size_t k = 0; k < 2 * n; ++k) c[k] += 1.0 * s->illum[k];
        base_scale_intensity(s, c);
        for (size_t k = 0; k < 2 * n; ++k) c[k] += -1.0 * s->illum[k];
    } else if (s->kind == KIND_POLY) {
        poly_scale_intensity(s, c);
    } else {
        base_scale_intensity(s, c);
    }
}

/* BaseCDI::project_intensity, BaseCDI.c++:156-160 */
static void project_intensity(orc_solver *s, double *c)
{
    propagate_to_detector(s, c);
    scale_intensity(s, c);
    propagate_from_detector(s, c);
}

/* Poly: pad -> project -> unpad around one projection, PolyCDI.c++:143-152,175-181 */
static void poly_project(orc_solver *s, double *c)
{
    double *p = get_padded(c, s->nx, s->ny, s->px, s->py);
    project_intensity(s, p);
    get_unpadded(p, s->pnx, s->pny, s->px, s->py, c);
    free(p);
}

static void project(orc_solver *s, double *c)
{
    if (s->kind == KIND_POLY)
        poly_project(s, c);
    else
        project_intensity(s, c);
}

/* apply_support: BaseCDI.c++:130-134 and FresnelCDI.c++:203-215 (no complex
 * constraint attached) */
/* TransmissionConstraint::apply_constraint, TransmissionConstraint.c++:76-172:
 * per-region c_mean = sum|ln|T|| / sum|arg T| (unless fixed), then per pixel
 * the region update (ComplexConstraint::get_new_mag / get_new_phase,
 * TransmissionConstraint.h:100-118) applied with set_mag then set_phase,
 * charge flipping, unit magnitude, and the caller's custom function */
static void apply_constraint(orc_solver *s, double *t)
{
    orc_tc *tc = &s->tc;
    int nx = s->nx, ny = s->ny;
    int regions = tc->nregions;
    if (regions > 0) {
        double *mean_lnA = zd((size_t)regions), *mean_phase = zd((size_t)regions);
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) {
                double rm = tc->region_map[(size_t)i * ny + j];
                if (rm > 0) {
                    int r = (int)rm - 1;
                    double *p = t + 2 * ((size_t)i * ny + j);
                    mean_phase[r] += fabs(atan2(p[1], p[0]));
                    mean_lnA[r] += fabs(log(mag_of(p)));
                }
            }
        for (int r = 0; r < regions; r++)
            if (!tc->fixed_c[r]) tc->c_mean[r] = mean_lnA[r] / mean_phase[r];
        free(mean_lnA);
        free(mean_phase);
    }
    if (regions > 0 || tc->charge_flip || tc->enforce_unity) {
        for (int i = 0; i < nx; i++)
            for (int j = 0; j < ny; j++) {
                double *p = t + 2 * ((size_t)i * ny + j);
                double phase_old = atan2(p[1], p[0]);
                double mag_old = mag_of(p);
                double rm = regions > 0 ? tc->region_map[(size_t)i * ny + j] : 0;
                if (regions > 0 && rm > 0) {
                    int r = (int)rm - 1;
                    double a1 = tc->alpha1[r], a2 = tc->alpha2[r], cm = tc->c_mean[r];
                    double mag_new = exp((1 - a1) * log(mag_old) + a1 * cm * phase_old);
                    double phase_new = (1 - a2) * phase_old + a2 * log(mag_old) / cm;
                    set_mag(p, mag_new);
                    double m = mag_of(p);             /* Complex_2D::set_phase */
                    p[0] = m * cos(phase_new);
                    p[1] = m * sin(phase_new);
                    mag_old = mag_new;
                }
                if (tc->charge_flip && tc->flip_sign * p[1] > 0) p[1] = -1 * p[1];
                if (tc->enforce_unity && mag_old > 1) set_mag(p, 1);
            }
    }
    if (tc->custom) tc->custom(t, nx, ny, tc->user);
}

static void fresnel_set_transmission(orc_solver *s, const double *t, double *esw);
static void fresnel_get_transmission(orc_solver *s, const double *esw, double *res);

/* BaseCDI::apply_support, BaseCDI.c++:130-134; FresnelCDI::apply_support,
 * FresnelCDI.c++:203-215 (the constraint acts on the transmission function) */
static void apply_support(orc_solver *s, double *c)
{
    support_constraint(s, c);
    if (!s->tc.active) return;
    if (s->kind == KIND_FRESNEL) {
        double *t = zd(2 * (size_t)s->nx * s->ny);
        fresnel_get_transmission(s, c, t);
        fresnel_set_transmission(s, t, c);
        free(t);
    } else {
        apply_constraint(s, c);
    }
}

/* BaseCDI::set_complex_constraint (BaseCDI.h:471-473) with a
 * TransmissionConstraint built as TransmissionConstraint.c++:20-73 does:
 * regions added in order, a pixel claimed by an earlier region stays with it;
 * fixed_c[r] is NaN for a free c_mean (ComplexConstraint::set_fixed_c). */
void orc_set_transmission_constraint(orc_solver *s, int enforce_unity, int charge_flip,
                                     int flip_sign, int nregions, const double *regions,
                                     const double *alpha, const double *fixed_c)
{
    orc_tc *tc = &s->tc;
    size_t n = (size_t)s->nx * s->ny;
    free(tc->region_map); free(tc->alpha1); free(tc->alpha2); free(tc->c_mean); free(tc->fixed_c);
    memset(tc, 0, sizeof(*tc));
    tc->active = 1;
    tc->enforce_unity = enforce_unity;
    tc->charge_flip = charge_flip;
    tc->flip_sign = flip_sign > 0 ? 1 : -1;
    tc->nregions = nregions;
    if (nregions > 0) {
        tc->region_map = zd(n);
        tc->alpha1 = zd((size_t)nregions);
        tc->alpha2 = zd((size_t)nregions);
        tc->c_mean = zd((size_t)nregions);
        tc->fixed_c = (int *)calloc((size_t)nregions, sizeof(int));
        for (int r = 0; r < nregions; ++r) {
            for (size_t k = 0; k < n; ++k)
                if (regions[r * n + k] > 0 && !(tc->region_map[k] > 0)) tc->region_map[k] = r + 1;
            tc->alpha1[r] = alpha[2 * r];
            tc->alpha2[r] = alpha[2 * r + 1];
            if (fixed_c && fixed_c[r] == fixed_c[r]) {
                tc->fixed_c[r] = 1;
                tc->c_mean[r] = fixed_c[r];
            }
        }
    }
}

void orc_set_transmission_custom(orc_solver *s, void (*f)(double *, int, int, void *), void *user)
{
    s->tc.custom = f;
    s->tc.user = user;
}

void orc_clear_transmission_constraint(orc_solver *s)
{
    orc_tc *tc = &s->tc;
    free(tc->region_map); free(tc->alpha1); free(tc->alpha2); free(tc->c_mean); free(tc->fixed_c);
    memset(tc, 0, sizeof(*tc));
}

/* set_custom_algorithm, BaseCDI.c++:240-255 */
static void set_custom(orc_solver *s, const double *m)
{
    s->w[PSF] = m[0] + m[1] + m[2] + m[3];
    s->w[PFS] = -m[0] + m[4] + m[5] + m[6];
    s->w[PS] = -m[2] - m[5] - m[7] + m[9];
    s->w[PF] = -m[1] - m[4] + m[7] + m[8];
    s->w[PI_] = -m[3] - m[6] - m[8] - m[9];
    s->algorithm = CUSTOM;
}

/* set_algorithm, BaseCDI.c++:192-237 */
void orc_set_algorithm(orc_solver *s, int alg)
{
    if (s->algorithm == alg) return;
    double b = s->beta;
    double m[10] = {0};
    int known = 1;
    switch (alg) {
    case ER: break;
    case BIO: m[1] = b; break;
    case BOO: m[1] = b; m[8] = 1; break;
    case HIO: m[1] = b; m[2] = 1; break;
    case DM: m[0] = b; m[2] = 1; m[4] = 1; break;
    case SF: m[1] = 1; m[3] = 1; break;
    case ASR: m[1] = 1; m[2] = 1; break;
    case HPR: m[1] = b; m[2] = 1; break;
    case RAAR: m[1] = 1; m[2] = b; m[8] = (1 - b); break;
    default: known = 0;
    }
    if (known) set_custom(s, m);
    s->algorithm = alg;
}

void orc_set_custom_algorithm(orc_solver *s, const double *m) { set_custom(s, m); }

/* set_relaxation_parameter, BaseCDI.h:264-267: a no-op for the weights until
 * the algorithm changes */
void orc_set_relaxation_parameter(orc_solver *s, double beta)
{
    s->beta = beta;
    orc_set_algorithm(s, s->algorithm);
}

/* update_n_best, BaseCDI.c++:390-413 */
static void update_n_best(orc_solver *s)
{
    int place = 0;
    for (; place < s->n_best && s->current_error > s->best_err[place]; place++)
        ;
    if (s->n_best > 0 && place < s->n_best) {
        double *tp = s->best[s->n_best - 1];
        memcpy(tp, s->complex_, sizeof(double) * 2 * (size_t)s->nx * s->ny);
        for (int i = s->n_best - 1; i > place; i--) {
            s->best_err[i] = s->best_err[i - 1];
            s->best[i] = s->best[i - 1];
        }
        s->best_err[place] = s->current_error;
        s->best[place] = tp;
    }
}

/* BaseCDI::iterate, BaseCDI.c++:297-387, and PolyCDI::iterate,
 * PolyCDI.c++:130-250 (same structure, each projection padded) */
void orc_iterate(orc_solver *s)
{
    size_t n = (size_t)s->nx * s->ny, nb = sizeof(double) * 2 * n;
    double *x = s->complex_;
    if (s->kind == KIND_FRESNEL_WF) {
        /* FresnelCDI_WF::iterate, FresnelCDI_WF.c++:155-162: a fixed algorithm
         * on the detector-plane field, no n-best bookkeeping */
        propagate_from_detector(s, x);
        apply_support(s, x);
        propagate_to_detector(s, x);
        scale_intensity(s, x);
        return;
    }
    if (s->algorithm == ER) {
        project(s, x);
        apply_support(s, x);
        update_n_best(s);
        return;
    }
    if (s->w[PFS] != 0) {
        memcpy(s->tPFS, x, nb);
        apply_support(s, s->tPFS);
        project(s, s->tPFS);
    }
    if (s->w[PF] != 0) {
        memcpy(s->tPF, x, nb);
        project(s, s->tPF);
    }
    if (s->w[PS] != 0) {
        memcpy(s->tPS, x, nb);
        apply_support(s, s->tPS);
    }
    if (s->w[PSF] != 0) {
        if (s->w[PF] != 0) {
            memcpy(s->tPSF, s->tPF, nb);
            apply_support(s, s->tPSF);
        } else {
            memcpy(s->tPSF, x, nb);
            project(s, s->tPSF);
            apply_support(s, s->tPSF);
        }
    }
    for (size_t k = 0; k < n; ++k) {
        double vr = (1 + s->w[PI_]) * x[2 * k];
        double vi = (1 + s->w[PI_]) * x[2 * k + 1];
        if (s->w[PFS] != 0) { vr += s->w[PFS] * s->tPFS[2 * k]; vi += s->w[PFS] * s->tPFS[2 * k + 1]; }
        if (s->w[PF] != 0) { vr += s->w[PF] * s->tPF[2 * k]; vi += s->w[PF] * s->tPF[2 * k + 1]; }
        if (s->w[PS] != 0) { vr += s->w[PS] * s->tPS[2 * k]; vi += s->w[PS] * s->tPS[2 * k + 1]; }
        if (s->w[PSF] != 0) { vr += s->w[PSF] * s->tPSF[2 * k]; vi += s->w[PSF] * s->tPSF[2 * k + 1]; }
        x[2 * k] = vr;
        x[2 * k + 1] = vi;
    }
    update_n_best(s);
}

/* apply_shrinkwrap, BaseCDI.c++:416-429 */
void orc_apply_shrinkwrap(orc_solver *s, double gauss_width, double threshold)
{
    size_t n = (size_t)s->nx * s->ny;
    double *recon = zd(n);
    for (size_t k = 0; k < n; ++k) recon[k] = mag_of(s->complex_ + 2 * k);
    convolve(recon, s->nx, s->ny, gauss_width, 4);
    apply_threshold(recon, s->nx, s->ny, threshold);
    set_support_arr(s, recon, 0);
    free(recon);
}

/* ---------------- construction ---------------- */

static orc_solver *base_create(int kind, int nx, int ny, int n_best)
{
    orc_solver *s = (orc_solver *)calloc(1, sizeof(orc_solver));
    size_t n = (size_t)nx * ny;
    s->kind = kind; s->nx = nx; s->ny = ny;
    s->beta = 0.9;                                /* BaseCDI.c++:38 */
    s->complex_ = zd(2 * n);
    s->support = zd(n);
    s->isqrt = zd(n);
    s->n_best = n_best;
    if (n_best > 0) {                             /* BaseCDI.c++:43-50 */
        s->best = (double **)calloc((size_t)n_best, sizeof(double *));
        s->best_err = zd((size_t)n_best);
        for (int i = 0; i < n_best; ++i) { s->best[i] = zd(2 * n); s->best_err[i] = 1; }
    }
    s->tPFS = zd(2 * n); s->tPF = zd(2 * n); s->tPS = zd(2 * n); s->tPSF = zd(2 * n);
    s->fft = canon_ctx_created(nx, ny);
    s->algorithm = CUSTOM;                        /* BaseCDI.c++:63-64 */
    orc_set_algorithm(s, ER);
    return s;
}

orc_solver *orc_planar_create(int nx, int ny, int n_best)
{
    return base_create(KIND_PLANAR, nx, ny, n_best);
}

/* FresnelCDI_WF::FresnelCDI_WF, FresnelCDI_WF.c++:31-79: the quarter table of
 * the zone-plate-to-detector propagation factor, (sin phi, -cos phi)/sqrt(N) */
orc_solver *orc_fresnel_wf_create(int nx, int ny, double wavelength, double zone_focal_length,
                                  double focal_detector_length, double pixel_size, int n_best)
{
    orc_solver *s = base_create(KIND_FRESNEL_WF, nx, ny, n_best);
    s->wavelength = wavelength;
    s->z12 = zone_focal_length;
    s->z23 = focal_detector_length;
    s->pixel = pixel_size;
    int qy = ny / 2;
    s->coef = zd((size_t)2 * (nx / 2) * qy);
    double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    double z12 = s->z12, z23 = s->z23;
    double scaling_x = wavelength * z23 / (pixel_size * nx);
    double scaling_y = wavelength * z23 / (pixel_size * ny);
    double norm = 1 / (sqrt(nx * ny));
    for (int i = 0; i < nx / 2; i++)
        for (int j = 0; j < qy; j++) {
            double rho_2 = pow(scaling_x * (x_mid - i), 2) + pow(scaling_y * (y_mid - j), 2);
            double phi = rho_2 / z12 + rho_2 / z23;
            phi *= M_PI / wavelength;
            s->coef[2 * ((size_t)i * qy + j)] = sin(phi) * norm;
            s->coef[2 * ((size_t)i * qy + j) + 1] = -cos(phi) * norm;
        }
    return s;
}

/* FresnelCDI_WF::set_support(z_diameter, size), FresnelCDI_WF.c++:184-203: a
 * disk of the zone plate's projected size (the centre is (nx-1)/2 in integer
 * arithmetic, on both axes), then convolve(support, 3, 5); pixels outside the
 * disk keep their earlier support values */
void orc_fresnel_wf_set_support(orc_solver *s, double z_diameter, double size)
{
    int nx = s->nx, ny = s->ny;
    double center_pixel = (nx - 1) / 2;
    double delta_z = (s->z12 / s->z23) * s->pixel;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
            double i_ = i - center_pixel;
            double j_ = j - center_pixel;
            double r = delta_z * sqrt(i_ * i_ + j_ * j_);
            if (r < size * z_diameter / 2.0) s->support[(size_t)i * ny + j] = 1;
        }
    convolve(s->support, nx, ny, 3, 5);
}

/* FresnelCDI::set_experimental_parameters, FresnelCDI.c++:57-95 */
void orc_fresnel_set_experimental_parameters(orc_solver *s, double wavelength, double zfd,
                                             double zfs, double pixel)
{
    int nx = s->nx, ny = s->ny, qy = ny / 2;
    s->wavelength = wavelength; s->pixel = pixel; s->zfd = zfd; s->zfs = zfs;
    double x_mid = (nx - 1) / 2.0, y_mid = (ny - 1) / 2.0;
    double zsd = zfd - zfs;
    double factor = pixel * pixel * M_PI / (wavelength) * ((1 / zfd) - (1 / zsd));
    for (int i = 0; i < nx / 2.0; i++)
        for (int j = 0; j < ny / 2.0; j++) {
            if (i >= nx / 2 || j >= qy) continue; /* outside the (nx/2)x(ny/2) table */
            double phi = factor * ((x_mid - i) * (x_mid - i) + (y_mid - j) * (y_mid - j));
            s->coef[2 * ((size_t)i * qy + j)] = cos(phi);
            s->coef[2 * ((size_t)i * qy + j) + 1] = sin(phi);
        }
    memcpy(s->illum_sample, s->illum, sizeof(double) * 2 * (size_t)nx * ny);
    propagate_from_detector(s, s->illum_sample);
}

/* FresnelCDI::FresnelCDI, FresnelCDI.c++:20-44 */
orc_solver *orc_fresnel_create(int nx, int ny, const double *white_field, double wavelength,
                               double zfd, double zfs, double pixel, double normalisation,
                               int n_best)
{
    orc_solver *s = base_create(KIND_FRESNEL, nx, ny, n_best);
    size_t n = (size_t)nx * ny;
    s->norm = normalisation;
    s->illum = zd(2 * n);
    s->illum_sample = zd(2 * n);
    s->coef = zd(2 * (size_t)(nx / 2) * (ny / 2) + 2);
    for (size_t k = 0; k < 2 * n; ++k) s->illum[k] = white_field[k] * normalisation;
    orc_fresnel_set_experimental_parameters(s, wavelength, zfd, zfs, pixel);
    return s;
}

/* FresnelCDI::set_norm, FresnelCDI.c++:139-148 */
void orc_fresnel_set_norm(orc_solver *s, double new_norm)
{
    double old = s->norm;
    size_t n = (size_t)s->nx * s->ny;
    s->norm = new_norm;
    double f = new_norm / old;
    for (size_t k = 0; k < 2 * n; ++k) s->illum[k] *= f;
    for (size_t k = 0; k < 2 * n; ++k) s->illum_sample[k] *= f;
}

/* FresnelCDI::auto_set_norm, FresnelCDI.c++:129-137 */
void orc_fresnel_auto_set_norm(orc_solver *s)
{
    size_t n = (size_t)s->nx * s->ny;
    double *t = zd(n);
    for (size_t k = 0; k < n; ++k) t[k] = mag_of(s->illum + 2 * k);
    double wf_norm = get_sum(t, n);
    double int_norm = get_sum(s->isqrt, n);
    free(t);
    orc_fresnel_set_norm(s, int_norm / wf_norm);
}

/* FresnelCDI::set_transmission_function, FresnelCDI.c++:253-283, including
 * the `j < nx` inner bound; writes past the end of the buffer are skipped */
static void fresnel_set_transmission(orc_solver *s, const double *t, double *esw)
{
    int nx = s->nx, ny = s->ny;
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < nx; j++) {
            long long k = (long long)i * ny + j;
            if (k >= (long long)nx * ny) continue;
            double ill_r = s->illum_sample[2 * k], tr = t[2 * k];
            double ill_i = s->illum_sample[2 * k + 1], ti = t[2 * k + 1];
            esw[2 * k] = ill_r * tr - ill_i * ti - ill_r;
            esw[2 * k + 1] = ill_r * ti + ill_i * tr - ill_i;
        }
}

/* FresnelCDI::get_transmission_function, FresnelCDI.c++:298-355 */
static void fresnel_get_transmission(orc_solver *s, const double *esw, double *res)
{
    size_t n = (size_t)s->nx * s->ny;
    for (size_t k = 0; k < n; ++k) {
        double ill_r = s->illum_sample[2 * k], ill_i = s->illum_sample[2 * k + 1];
        double denom = ill_r * ill_r + ill_i * ill_i;
        if (denom != 0) {
            double er = esw[2 * k], ei = esw[2 * k + 1];
            double rn = ill_r * (er + ill_r) + ill_i * (ei + ill_i);
            double in = ill_r * (ei + ill_i) - ill_i * (er + ill_r);
            res[2 * k] = rn / denom;
            res[2 * k + 1] = in / denom;
        } else {
            res[2 * k] = 1.0;
            res[2 * k + 1] = 0.0;
        }
    }
    if (s->tc.active) apply_constraint(s, res); /* FresnelCDI.c++:352-353 */
}

/* PolyCDI::PolyCDI, PolyCDI.c++:25-35 (its own `beta` member never reaches
 * the algorithm table, PolyCDI.h:53 vs BaseCDI.h:113) */
orc_solver *orc_poly_create(int nx, int ny, double beta, int n_best)
{
    (void)beta;
    orc_solver *s = base_create(KIND_POLY, nx, ny, n_best);
    s->isqrt_calc = zd((size_t)nx * ny);
    return s;
}

/* PolyCDI::set_spectrum(Double_2D), PolyCDI.c++:66-89; rows (wavelength, weight) */
void orc_poly_set_spectrum(orc_solver *s, const double *wl_weight, int nlambda)
{
    free(s->spectrum);
    s->spectrum = zd(2 * (size_t)nlambda);
    memcpy(s->spectrum, wl_weight, sizeof(double) * 2 * (size_t)nlambda);
    s->nlambda = nlambda;
    double maxweight = 0, totweight = 0;
    for (int i = 0; i < nlambda; i++) {
        if (s->spectrum[2 * i + 1] > maxweight) {
            s->lambdac = s->spectrum[2 * i];
            maxweight = s->spectrum[2 * i + 1];
        }
        totweight += s->spectrum[2 * i + 1];
    }
    for (int i = 0; i < nlambda; i++) s->spectrum[2 * i + 1] = s->spectrum[2 * i + 1] / totweight;
    s->px = (int)((s->spectrum[0] / s->lambdac - 1.0) * s->nx / 2);
    s->py = (int)((s->spectrum[0] / s->lambdac - 1.0) * s->ny / 2);
    s->pnx = s->nx + 2 * s->px;
    s->pny = s->ny + 2 * s->py;
    canon_ctx_destroyd(s->fft_pad);
    s->fft_pad = canon_ctx_created(s->pnx, s->pny);
}

/* read_spec, NADIA/src/io_spec.c:61-133: tab-separated lines; leading lines
 * whose first token does not start with a digit are dropped; column 0 is an
 * energy stored as its reciprocal; values pass through float.  Fills
 * `out` (capacity rows) and returns the number of rows, or -1. */
int orc_read_spec(const char *path, double *out, int capacity)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[4096];
    char **tok = NULL;
    int ntok = 0, cap = 0;
    while (fgets(line, sizeof line, f)) {
        size_t L = strlen(line);
        if (L && line[L - 1] == '\n') line[--L] = 0;
        char *p = line;
        for (;;) {
            char *tab = strchr(p, '\t');
            size_t len = tab ? (size_t)(tab - p) : strlen(p);
            if (!tab && len == 0) break;
            if (ntok == cap) { cap = cap ? 2 * cap : 64; tok = (char **)realloc(tok, sizeof(char *) * cap); }
            tok[ntok] = (char *)malloc(len + 1);
            memcpy(tok[ntok], p, len);
            tok[ntok][len] = 0;
            ntok++;
            if (!tab) break;
            p = tab + 1;
        }
        if (ntok > 0 && !isdigit((unsigned char)tok[0][0])) {
            for (int k = 0; k < ntok; ++k) free(tok[k]);
            ntok = 0;
        }
    }
    fclose(f);
    int rows = ntok / 2;
    float value = 0;
    for (int i = 0, k = 0; i < rows && i < capacity; ++i)
        for (int j = 0; j < 2; ++j, ++k) {
            float v;
            value = (sscanf(tok[k], "%f", &v) == 1) ? v : 0.0f;
            if (j == 0) value = 1.0 / value;
            out[2 * i + j] = value;
        }
    for (int k = 0; k < ntok; ++k) free(tok[k]);
    free(tok);
    return rows;
}

/* ---------------- the remaining public surface ---------------- */

void orc_destroy(orc_solver *s)
{
    if (!s) return;
    free(s->complex_); free(s->support); free(s->isqrt); free(s->beam_stop);
    for (int i = 0; i < s->n_best; ++i) free(s->best[i]);
    free(s->best); free(s->best_err);
    free(s->tPFS); free(s->tPF); free(s->tPS); free(s->tPSF);
    canon_ctx_destroyd(s->fft); canon_ctx_destroyd(s->fft_pad);
    free(s->illum); free(s->illum_sample); free(s->coef);
    free(s->spectrum); free(s->isqrt_calc);
    orc_clear_transmission_constraint(s);
    free(s);
}

void orc_set_support(orc_solver *s, const double *obj, int soften) { set_support_arr(s, obj, soften); }

/* set_intensity, BaseCDI.c++:118-124 */
void orc_set_intensity(orc_solver *s, const double *I)
{
    size_t n = (size_t)s->nx * s->ny;
    for (size_t k = 0; k < n; ++k) s->isqrt[k] = sqrt(I[k]);
}

/* set_beam_stop, BaseCDI.c++:112-116 */
void orc_set_beam_stop(orc_solver *s, const double *mask)
{
    size_t n = (size_t)s->nx * s->ny;
    if (!s->beam_stop) s->beam_stop = zd(n);
    memcpy(s->beam_stop, mask, sizeof(double) * n);
}

/* PlanarCDI::initialise_estimate, PlanarCDI.c++:39-62 (also PolyCDI.c++:102-126),
 * and FresnelCDI::initialise_estimate, FresnelCDI.c++:152-201 */
void orc_initialise_estimate(orc_solver *s, int seed)
{
    size_t n = (size_t)s->nx * s->ny;
    srand(seed);
    if (s->kind == KIND_FRESNEL_WF) {
        /* FresnelCDI_WF::initialise_estimate, FresnelCDI_WF.c++:134-152:
         * sqrt(I) inside the support, 0 outside (the seed is unused) */
        for (size_t k = 0; k < n; ++k) {
            s->complex_[2 * k] = s->support[k] ? s->isqrt[k] : 0;
            s->complex_[2 * k + 1] = 0;
        }
        return;
    }
    if (s->kind == KIND_FRESNEL) {
        double *t = zd(2 * n);
        for (size_t k = 0; k < n; ++k) {
            double real = 1 - 0.2 * rand() / ((double)RAND_MAX);
            t[2 * k] = real;
            t[2 * k + 1] = 0;
        }
        fresnel_set_transmission(s, t, s->complex_);
        apply_support(s, s->complex_);
        free(t);
        return;
    }
    /* `int max_value = intensity_sqrt.get_max()` truncates; `max_value*rand()`
     * is an int multiplication that wraps modulo 2^32 */
    int max_value = (int)get_max(s->isqrt, n);
    for (size_t k = 0; k < n; ++k) {
        if (!s->support[k]) {
            s->complex_[2 * k] = 0;
            s->complex_[2 * k + 1] = 0;
        } else {
            int p1 = (int)((unsigned)max_value * (unsigned)rand());
            double r = s->support[k] * (p1 / (double)RAND_MAX);
            int p2 = (int)((unsigned)max_value * (unsigned)rand());
            double im = s->support[k] * (p2 / (double)RAND_MAX);
            s->complex_[2 * k] = r;
            s->complex_[2 * k + 1] = im;
        }
    }
}

void orc_set_esw(orc_solver *s, const double *esw)
{
    memcpy(s->complex_, esw, sizeof(double) * 2 * (size_t)s->nx * s->ny);
}
void orc_get_esw(orc_solver *s, double *esw)
{
    memcpy(esw, s->complex_, sizeof(double) * 2 * (size_t)s->nx * s->ny);
}
double orc_get_error(orc_solver *s) { return s->current_error; }
void orc_get_support(orc_solver *s, double *out)
{
    memcpy(out, s->support, sizeof(double) * (size_t)s->nx * s->ny);
}

/* get_transmission: FresnelCDI::get_transmission_function for Fresnel; the
 * exit-surface wave itself for Planar and Poly (PolyCDI.h:210 declares
 * get_transmission without defining it) */
void orc_get_transmission(orc_solver *s, double *out)
{
    if (s->kind == KIND_FRESNEL)
        fresnel_get_transmission(s, s->complex_, out);
    else
        orc_get_esw(s, out);
}
void orc_set_transmission(orc_solver *s, const double *t)
{
    if (s->kind == KIND_FRESNEL)
        fresnel_set_transmission(s, t, s->complex_);
    else
        orc_set_esw(s, t);
}
void orc_get_illumination_at_sample(orc_solver *s, double *out)
{
    if (s->illum_sample) memcpy(out, s->illum_sample, sizeof(double) * 2 * (size_t)s->nx * s->ny);
}

/* get_best_result, BaseCDI.c++:82-91; returns 0 when the index is out of range */
int orc_get_best_result(orc_solver *s, int index, double *err, double *esw)
{
    if (index >= 0 && index < s->n_best) {
        *err = s->best_err[index];
        memcpy(esw, s->best[index], sizeof(double) * 2 * (size_t)s->nx * s->ny);
        return 1;
    }
    return 0;
}
void orc_reset_best(orc_solver *s)
{
    for (int i = 0; i < s->n_best; ++i) s->best_err[i] = 1;
}

/* the single operators, as the IDL interface exposes them
 * (NADIA/interfaces/idl/IDL_interface.c:947-985); Poly operates on the
 * padded grid in the reference, so these act on an nx*ny field for Planar
 * and Fresnel only */
void orc_propagate_to_detector(orc_solver *s, double *c) { propagate_to_detector(s, c); }
void orc_propagate_from_detector(orc_solver *s, double *c) { propagate_from_detector(s, c); }
void orc_scale_intensity(orc_solver *s, double *c) { scale_intensity(s, c); }
void orc_apply_support(orc_solver *s, double *c) { apply_support(s, c); }
void orc_project_intensity(orc_solver *s, double *c) { project(s, c); }

/* PlanarCDI::get_intensity_autocorrelation, PlanarCDI.c++:13-36 */
void orc_get_intensity_autocorrelation(orc_solver *s, double *out)
{
    size_t n = (size_t)s->nx * s->ny;
    double *t = zd(2 * n);
    for (size_t k = 0; k < n; ++k) {
        double component = (1.0 / sqrt(2.0)) * (s->isqrt[k] * s->isqrt[k]);
        t[2 * k] = component;
        t[2 * k + 1] = component;
    }
    canon_fft2d_execd(s->fft, (canon_cd *)t, 0);
    invert(t, s->nx, s->ny, 1);
    for (size_t k = 0; k < n; ++k) out[k] = mag_of(t + 2 * k);
    free(t);
}

/* the canonical 2-D transform on its own, for the FFT known-answer tests */
int orc_fft2d(double *a, int nx, int ny, int forward)
{
    canon_ctxd *c = canon_ctx_created(nx, ny);
    if (!c) return -1;
    canon_fft2d_execd(c, (canon_cd *)a, forward);
    canon_ctx_destroyd(c);
    return 0;
}

int orc_padding(orc_solver *s, int *px, int *py)
{
    *px = s->px;
    *py = s->py;
    return 0;
}

/* ===================== PhaseDiverseCDI (NADIA/src/PhaseDiverseCDI.c++) =====================
 *
 * Frames are orc_solver reconstructions (Fresnel: the transmission function is
 * exchanged, PhaseDiverseCDI.c++:330-345; others: the exit-surface wave) placed
 * at (x, y) on a global object.  remove_positions forgets the frames only; the
 * positions, scalings, weights and per-frame results stay indexed as before
 * (PhaseDiverseCDI.c++:60-66).  Arrays the reference leaves uninitialised
 * (new Complex_2D) are zero here, as under the FFTW shim's fftw_malloc. */

typedef struct orc_pd {
    double beta, gamma;
    int parallel, scale;
    int nframes;            /* singleCDI.size() */
    int npos, cap;          /* x_position.size() and capacity */
    orc_solver **frame;
    double *xpos, *ypos, *alpha;
    double **result;        /* single_result: lnx*lny*2 each */
    double **weight;        /* weights: lnx*lny each */
    int *rnx, *rny;         /* sizes of result/weight n */
    double *object;         /* nx*ny*2, NULL before the first position */
    int nx, ny, x_min, y_min;
    int iterations_per_cycle;
    int weights_set;
} orc_pd;

orc_pd *orc_pd_create(double beta, double gamma, int parallel, int granularity)
{
    orc_pd *p = (orc_pd *)calloc(1, sizeof(orc_pd));
    p->beta = beta;
    p->gamma = gamma;
    p->parallel = parallel != 0;
    p->scale = granularity;
    p->iterations_per_cycle = 1;
    return p;
}

void orc_pd_destroy(orc_pd *p)
{
    if (!p) return;
    for (int n = 0; n < p->npos; ++n) {
        free(p->result[n]);
        free(p->weight[n]);
    }
    free(p->frame); free(p->xpos); free(p->ypos); free(p->alpha);
    free(p->result); free(p->weight); free(p->rnx); free(p->rny);
    free(p->object);
    free(p);
}

/* the get_global/local_x/y_pos helpers, PhaseDiverseCDI.h:380-397 (int results) */
static inline int pd_gx(const orc_pd *p, int x, double off) { return (int)(x - off - p->x_min); }
static inline int pd_gy(const orc_pd *p, int y, double off) { return (int)(y - off - p->y_min); }
static inline int pd_lx(const orc_pd *p, int x, double off) { return (int)(x + off + p->x_min); }
static inline int pd_ly(const orc_pd *p, int y, double off) { return (int)(y + off + p->y_min); }

/* reallocate_object_memory, PhaseDiverseCDI.c++:68-75 */
static void pd_realloc_object(orc_pd *p, int nx, int ny)
{
    free(p->object);
    p->object = zd(2 * (size_t)nx * ny);
    p->nx = nx;
    p->ny = ny;
}

/* add_new_position, PhaseDiverseCDI.c++:104-160 */
void orc_pd_add_position(orc_pd *p, orc_solver *frame, double x, double y, double alpha)
{
    p->weights_set = 0;
    const int lnx = frame->nx, lny = frame->ny;
    if (p->nframes >= p->cap || p->npos >= p->cap) {
        int cap = p->cap ? 2 * p->cap : 8;
        p->frame = (orc_solver **)realloc(p->frame, cap * sizeof(void *));
        p->xpos = (double *)realloc(p->xpos, cap * sizeof(double));
        p->ypos = (double *)realloc(p->ypos, cap * sizeof(double));
        p->alpha = (double *)realloc(p->alpha, cap * sizeof(double));
        p->result = (double **)realloc(p->result, cap * sizeof(double *));
        p->weight = (double **)realloc(p->weight, cap * sizeof(double *));
        p->rnx = (int *)realloc(p->rnx, cap * sizeof(int));
        p->rny = (int *)realloc(p->rny, cap * sizeof(int));
        p->cap = cap;
    }
    p->frame[p->nframes++] = frame;
    const int k = p->npos++;
    p->xpos[k] = x;
    p->ypos[k] = y;
    p->alpha[k] = alpha;
    p->result[k] = zd(2 * (size_t)lnx * lny);
    p->weight[k] = zd((size_t)lnx * lny);
    p->rnx[k] = lnx;
    p->rny[k] = lny;
    if (!p->object) {
        p->x_min = (int)(-x);
        p->y_min = (int)(-y);
        pd_realloc_object(p, lnx * p->scale, lny * p->scale);
    }
    int extra_x = 0, extra_y = 0;
    const int gx0 = pd_gx(p, 0, x) * p->scale, gy0 = pd_gy(p, 0, y) * p->scale;
    const int gx1 = pd_gx(p, lnx, x) * p->scale, gy1 = pd_gy(p, lny, y) * p->scale;
    if (gx0 < 0) {
        p->x_min = (int)(-x);
        extra_x += -gx0;
    }
    if (gy0 < 0) {
        p->y_min = (int)(-y);
        extra_y += -gy0;
    }
    if (gx1 > p->nx) extra_x += gx1 - p->nx;
    if (gy1 > p->ny) extra_y += gy1 - p->ny;
    if (extra_x || extra_y) pd_realloc_object(p, p->nx + extra_x, p->ny + extra_y);
}

void orc_pd_remove_positions(orc_pd *p) { p->nframes = 0; }

/* set_up_weights, PhaseDiverseCDI.c++:450-530 */
static void pd_set_up_weights(orc_pd *p)
{
    if (p->weights_set) return;
    p->weights_set = 1;
    const int frames = p->nframes;
    for (int n = 0; n < frames; ++n) {
        const int lnx = p->rnx[n], lny = p->rny[n];
        orc_solver *f = p->frame[n];
        double *illum_mag = NULL, max = 0;
        if (f->kind == KIND_FRESNEL) {
            /* the frame's size is the result's size for the frames added since
             * the last remove_positions; the reference reads illum by the
             * result's size too */
            illum_mag = zd((size_t)lnx * lny);
            for (size_t k = 0; k < (size_t)lnx * lny; ++k) illum_mag[k] = mag_of(f->illum_sample + 2 * k);
            max = illum_mag[0];
            for (size_t k = 0; k < (size_t)lnx * lny; ++k)
                if (illum_mag[k] > max) max = illum_mag[k];
        }
        for (int i = 0; i < lnx; ++i)
            for (int j = 0; j < lny; ++j) {
                double value = f->kind == KIND_FRESNEL ? illum_mag[(size_t)i * lny + j] / max : 1;
                value = p->alpha[n] * pow(value, p->gamma);
                if (f->support[(size_t)i * f->ny + j] <= 0.0) value = 0;
                if (!p->parallel) value *= p->beta;
                p->weight[n][(size_t)i * lny + j] = value;
            }
        free(illum_mag);
    }
    if (!p->parallel) return;
    double *norm = zd((size_t)p->nx * p->ny);
    for (int n = 0; n < frames; ++n)
        for (int i_ = 0; i_ < p->rnx[n]; ++i_)
            for (int j_ = 0; j_ < p->rny[n]; ++j_) {
                const int i = pd_gx(p, i_, p->xpos[n]), j = pd_gy(p, j_, p->ypos[n]);
                if (i >= 0 && j >= 0 && i < p->nx && j < p->ny) {
                    const double w = p->weight[n][(size_t)i_ * p->rny[n] + j_];
                    double *t = &norm[(size_t)i * p->ny + j];
                    *t = n == 0 ? w : w + *t;
                }
            }
    for (int n = 0; n < frames; ++n)
        for (int i_ = 0; i_ < p->rnx[n]; ++i_)
            for (int j_ = 0; j_ < p->rny[n]; ++j_) {
                const int i = pd_gx(p, i_, p->xpos[n]), j = pd_gy(p, j_, p->ypos[n]);
                if (i >= 0 && j >= 0 && i < p->nx && j < p->ny) {
                    double *w = &p->weight[n][(size_t)i_ * p->rny[n] + j_];
                    const double nn = norm[(size_t)i * p->ny + j];
                    *w = nn <= 0 ? 0 : p->beta * *w / nn;
                }
            }
    free(norm);
}

/* get_result / set_result, PhaseDiverseCDI.c++:330-345 */
static void pd_get_result(orc_solver *f, double *r) { orc_get_transmission(f, r); }
static void pd_set_result(orc_solver *f, const double *r) { orc_set_transmission(f, r); }

/* add_to_object, PhaseDiverseCDI.c++:537-640 */
static void pd_add_to_object(orc_pd *p, int n)
{
    pd_get_result(p->frame[n], p->result[n]);
    pd_set_up_weights(p);
    const double xo = p->xpos[n], yo = p->ypos[n];
    const double *small = p->result[n], *w = p->weight[n];
    const int lnx = p->rnx[n], lny = p->rny[n], sc = p->scale;
    double *sub = zd(sc);
    for (int d = 0; d < sc; ++d) sub[d] = (d + 0.5 * ((sc + 1) % 2)) / ((double)sc);
    double *o = p->object;
    for (int i_ = 1; i_ < lnx - 1; ++i_)
        for (int j_ = 1; j_ < lny - 1; ++j_) {
            const double wt = w[(size_t)i_ * lny + j_];
            if (wt == 0) continue;
            const int i = pd_gx(p, i_, xo) * sc, j = pd_gy(p, j_, yo) * sc;
            if (!(i >= 0 && j >= 0 && i < p->nx && j < p->ny)) continue;
            const double *f00 = small + 2 * ((size_t)i_ * lny + j_);
            if (sc != 1) {
                const double *f10 = small + 2 * ((size_t)(i_ + 1) * lny + j_);
                const double *f01 = small + 2 * ((size_t)i_ * lny + j_ + 1);
                const double *f11 = small + 2 * ((size_t)(i_ + 1) * lny + j_ + 1);
                for (int di = 0; di < sc; ++di)
                    for (int dj = 0; dj < sc; ++dj) {
                        const double x = sub[di], y = sub[dj], x1 = 1 - x, y1 = 1 - y;
                        const double vr = f00[0] * (x1) * (y1) + f10[0] * x * (y1) + f01[0] * (x1) * y + f11[0] * x * y;
                        const double vi = f00[1] * (x1) * (y1) + f10[1] * x * (y1) + f01[1] * (x1) * y + f11[1] * x * y;
                        const int ni = (int)((i_ + 0.5 - xo - p->x_min) * sc + di);
                        const int nj = (int)((j_ + 0.5 - yo - p->y_min) * sc + dj);
                        /* the reference's flat index ni*ny + nj: a column past
                         * either edge lands in the neighbouring row; outside
                         * the whole array it writes out of bounds (skipped) */
                        const long long f = (long long)ni * p->ny + nj;
                        if (f < 0 || f >= (long long)p->nx * p->ny) continue;
                        double *t = o + 2 * f;
                        double nr = wt * vr + t[0];
                        double nim = wt * vi + t[1];
                        if (!p->parallel) {
                            nr -= wt * t[0];
                            nim -= wt * t[1];
                        }
                        t[0] = nr;
                        t[1] = nim;
                    }
            } else {
                double *t = o + 2 * ((size_t)i * p->ny + j);
                double nr = wt * f00[0] + t[0];
                double nim = wt * f00[1] + t[1];
                if (!p->parallel) {
                    nr -= wt * t[0];
                    nim -= wt * t[1];
                }
                t[0] = nr;
                t[1] = nim;
            }
        }
    free(sub);
}

/* update_from_object, PhaseDiverseCDI.c++:664-711 */
static void pd_update_from_object(orc_pd *p, int n)
{
    pd_set_up_weights(p);
    const double xo = p->xpos[n], yo = p->ypos[n];
    double *small = p->result[n];
    const double *w = p->weight[n];
    const int lnx = p->rnx[n], lny = p->rny[n], sc = p->scale;
    const double *o = p->object;
    for (int i_ = 0; i_ < lnx; ++i_)
        for (int j_ = 0; j_ < lny; ++j_) {
            if (w[(size_t)i_ * lny + j_] == 0) continue;
            const int i = pd_gx(p, i_, xo) * sc, j = pd_gy(p, j_, yo) * sc;
            if (!(i >= 0 && j >= 0 && i < p->nx && j < p->ny)) continue;
            double *s = small + 2 * ((size_t)i_ * lny + j_);
            if (sc != 1) {
                double re = 0, im = 0;
                for (int di = 0; di < sc; ++di)
                    for (int dj = 0; dj < sc; ++dj) {
                        /* flat index, as the reference reads (past the array: skipped) */
                        const long long f = (long long)(i + di) * p->ny + j + dj;
                        if (f >= (long long)p->nx * p->ny) continue;
                        re += o[2 * f];
                        im += o[2 * f + 1];
                    }
                const double norm = 1 / ((double)(sc * sc));
                s[0] = re * norm;
                s[1] = im * norm;
            } else {
                s[0] = o[2 * ((size_t)i * p->ny + j)];
                s[1] = o[2 * ((size_t)i * p->ny + j) + 1];
            }
        }
    pd_set_result(p->frame[n], small);
}

/* scale_object, PhaseDiverseCDI.c++:290-325 */
static void pd_scale_object(orc_pd *p, double factor)
{
    pd_set_up_weights(p);
    for (int i = 0; i < p->nx; ++i)
        for (int j = 0; j < p->ny; ++j) {
            int inside = 0;
            for (int n = 0; n < p->nframes; ++n) {
                const int i_ = pd_lx(p, i / p->scale, p->xpos[n]);
                const int j_ = pd_ly(p, j / p->scale, p->ypos[n]);
                if (i_ >= 0 && j_ >= 0 && i_ < p->rnx[n] && j_ < p->rny[n]) {
                    inside = p->weight[n][(size_t)i_ * p->rny[n] + j_] != 0;
                    if (inside) break;
                }
            }
            double *t = p->object + 2 * ((size_t)i * p->ny + j);
            if (!inside) {
                t[0] = 1.0;
                t[1] = 0.0;
            } else {
                t[0] = factor * t[0];
                t[1] = factor * t[1];
            }
        }
}

/* initialise_estimate, PhaseDiverseCDI.c++:163-177 */
void orc_pd_initialise_estimate(orc_pd *p)
{
    if (!p->object) return; /* no position yet (the reference dereferences null) */
    for (size_t k = 0; k < (size_t)p->nx * p->ny; ++k) {
        p->object[2 * k] = 1;
        p->object[2 * k + 1] = 0;
    }
    for (int n = 0; n < p->nframes; ++n) pd_add_to_object(p, n);
}

/* iterate, PhaseDiverseCDI.c++:180-230 (the reference also prints the
 * iteration count and each frame's error) */
void orc_pd_iterate(orc_pd *p)
{
    for (int n = 0; n < p->nframes; ++n) {
        pd_update_from_object(p, n);
        for (int k = 0; k < p->iterations_per_cycle; ++k) orc_iterate(p->frame[n]);
        if (!p->parallel) pd_add_to_object(p, n);
    }
    if (p->parallel) {
        pd_scale_object(p, 1 - p->beta);
        for (int n = 0; n < p->nframes; ++n) pd_add_to_object(p, n);
    }
}

void orc_pd_set_iterations_per_cycle(orc_pd *p, int n) { p->iterations_per_cycle = n; }
void orc_pd_set_feedback_parameter(orc_pd *p, double b) { p->beta = b; p->weights_set = 0; }
void orc_pd_set_amplification_factor(orc_pd *p, double g) { p->gamma = g; p->weights_set = 0; }
/* set_probe_scaling, PhaseDiverseCDI.h:214-226: returns 0 when n is too large */
int orc_pd_set_probe_scaling(orc_pd *p, int n, double alpha)
{
    int ok = n >= 0 && n < p->npos;
    if (ok) p->alpha[n] = alpha;
    p->weights_set = 0;
    return ok;
}
void orc_pd_get_size(orc_pd *p, int *nx, int *ny)
{
    *nx = p->object ? p->nx : 0;
    *ny = p->object ? p->ny : 0;
}
void orc_pd_get_transmission(orc_pd *p, double *out)
{
    memcpy(out, p->object, sizeof(double) * 2 * (size_t)p->nx * p->ny);
}
/* set_transmission, PhaseDiverseCDI.c++:81-101: returns 0 on a size mismatch */
int orc_pd_set_transmission(orc_pd *p, int nx, int ny, const double *t)
{
    if (!p->object) pd_realloc_object(p, nx, ny);
    if (nx != p->nx || ny != p->ny) return 0;
    memcpy(p->object, t, sizeof(double) * 2 * (size_t)nx * ny);
    return 1;
}
double orc_pd_get_x(orc_pd *p, int n) { return p->xpos[n]; }
double orc_pd_get_y(orc_pd *p, int n) { return p->ypos[n]; }

/* ---- image alignment (NADIA/src/utils.c:1151-1300) ---- */

/* real-to-complex / complex-to-real transforms in FFTW's layout: r2c keeps
 * columns 0..ny/2 of the transform of (x, 0); c2r extends by Hermitian
 * symmetry and keeps the real part of the backward transform (unnormalised) */
static void pd_r2c(const double *in, double *half, int nx, int ny)
{
    const int h = ny / 2 + 1;
    double *t = zd(2 * (size_t)nx * ny);
    for (size_t k = 0; k < (size_t)nx * ny; ++k) t[2 * k] = in[k];
    canon_ctxd *c = canon_ctx_created(nx, ny);
    canon_fft2d_execd(c, (canon_cd *)t, 1);
    canon_ctx_destroyd(c);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < h; ++y) {
            half[2 * ((size_t)x * h + y)] = t[2 * ((size_t)x * ny + y)];
            half[2 * ((size_t)x * h + y) + 1] = t[2 * ((size_t)x * ny + y) + 1];
        }
    free(t);
}

static void pd_c2r(const double *half, double *out, int nx, int ny)
{
    const int h = ny / 2 + 1;
    double *t = zd(2 * (size_t)nx * ny);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            double *d = t + 2 * ((size_t)x * ny + y);
            if (y < h) {
                d[0] = half[2 * ((size_t)x * h + y)];
                d[1] = half[2 * ((size_t)x * h + y) + 1];
            } else {
                const size_t k = (size_t)((nx - x) % nx) * h + (ny - y);
                d[0] = half[2 * k];
                d[1] = -half[2 * k + 1];
            }
        }
    canon_ctxd *c = canon_ctx_created(nx, ny);
    canon_fft2d_execd(c, (canon_cd *)t, 0);
    canon_ctx_destroyd(c);
    for (size_t k = 0; k < (size_t)nx * ny; ++k) out[k] = t[2 * k];
    free(t);
}

/* c2r(conj(r2c(a)) * r2c(b)) with Complex_2D::multiply's operation order
 * (Complex_2D.c++:203-228): the unnormalised cross-correlation */
static void pd_correlate(const double *a, const double *b, double *out, int nx, int ny)
{
    const int h = ny / 2 + 1;
    double *fa = zd(2 * (size_t)nx * h), *fb = zd(2 * (size_t)nx * h);
    pd_r2c(a, fa, nx, ny);
    pd_r2c(b, fb, nx, ny);
    for (size_t k = 0; k < (size_t)nx * h; ++k) {
        const double ar = fa[2 * k], ai = -1 * fa[2 * k + 1];
        const double br = fb[2 * k], bi = fb[2 * k + 1];
        const double nr = br * ar - bi * ai;
        const double ni = br * ai + bi * ar;
        fa[2 * k] = 1 * nr;
        fa[2 * k + 1] = 1 * ni;
    }
    pd_c2r(fa, out, nx, ny);
    free(fa);
    free(fb);
}

/* align, utils.c:1151-1300 (with its default overlap fraction 0.2 passed in) */
void orc_align(const double *first, int nx_1, int ny_1, const double *second, int nx_2, int ny_2,
               int *offset_x, int *offset_y, int min_x, int max_x, int min_y, int max_y,
               const double *first_w, const double *second_w, double overlap_fraction)
{
    const int nx = nx_1 > nx_2 ? nx_1 * 2 : nx_2 * 2;
    const int ny = ny_1 > ny_2 ? ny_1 * 2 : ny_2 * 2;
    if (min_x == max_x || min_y == max_y) {
        min_x = (int)(1 - nx / 2.0);
        max_x = (int)(nx / 2.0);
        min_y = (int)(1 - ny / 2.0);
        max_y = (int)(ny / 2.0);
    }
    const size_t N = (size_t)nx * ny;
    double *img1 = zd(N), *img2 = zd(N), *w1 = zd(N), *w2 = zd(N);
    double weight_sum = 0;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            if (!(i >= 0.5 * (nx - nx_1) && i < 0.5 * (nx + nx_1) && j >= 0.5 * (ny - ny_1) &&
                  j < 0.5 * (ny + ny_1)))
                continue;
            const int i_ = (int)(i - 0.5 * (nx - nx_1)), j_ = (int)(j - 0.5 * (ny - ny_1));
            const size_t k = (size_t)i * ny + j;
            if (!first_w || first_w[(size_t)i_ * ny_1 + j_] > 0) {
                img1[k] = first[(size_t)i_ * ny_1 + j_];
                w1[k] = 1.0;
            }
            if (i_ < nx_2 && j_ < ny_2 && (!second_w || second_w[(size_t)i_ * ny_2 + j_] > 0)) {
                img2[k] = second[(size_t)i_ * ny_2 + j_];
                w2[k] = 1.0;
            }
            if (nx_1 * ny_1 < nx_2 * ny_2)
                weight_sum += w1[k];
            else
                weight_sum += w2[k];
        }
    double *corr = zd(N), *overlap = zd(N);
    pd_correlate(img1, img2, corr, nx, ny);
    pd_correlate(w1, w2, overlap, nx, ny);
    double max = 0;
    const double overlap_factor = weight_sum * nx * ny;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            const size_t k = (size_t)i * ny + j;
            if (!(overlap[k] / overlap_factor > overlap_fraction)) continue;
            if (!(corr[k] / overlap[k] > max)) continue;
            int ti = -i, tj = -j;
            if (i >= nx / 2.0) ti = -i + nx;
            if (j >= ny / 2.0) tj = -j + ny;
            if (ti >= min_x && ti < max_x && tj >= min_y && tj < max_y) {
                max = corr[k] / overlap[k];
                *offset_x = ti;
                *offset_y = tj;
            }
        }
    free(img1); free(img2); free(w1); free(w2); free(corr); free(overlap);
}

/* interpolate(Double_2D, Double_2D), utils.c:1305-1352 (bilinear, border left 0) */
static void pd_interpolate(const double *a, int nx, int ny, double *big, int sc)
{
    const int bny = ny * sc;
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j) {
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

/* check_position, PhaseDiverseCDI.c++:395-447 */
static int pd_check_position(orc_pd *p, int n, double step, int min_x, int max_x, int min_y,
                             int max_y, int tries)
{
    const double x = p->xpos[n], y = p->ypos[n];
    if (step < 1.0 / p->scale) return 1;
    if (tries > 10 || x < (x + min_x) || x > (x + max_x) || y < (y + min_y) || y > (y + max_y))
        return 0;
    orc_solver *single = p->frame[n];
    double best_x = x, best_y = y, best_error = 100;
    const size_t on = 2 * (size_t)p->nx * p->ny, sn = 2 * (size_t)p->rnx[n] * p->rny[n];
    double *object_copy = zd(on), *single_copy = zd(sn);
    memcpy(object_copy, p->object, on * sizeof(double));
    memcpy(single_copy, p->result[n], sn * sizeof(double));
    p->beta = 0.5;
    p->weights_set = 0;
    for (int i = -1; i < 2; ++i)
        for (int j = -1; j < 2; ++j) {
            const double nx_ = x + i * step, ny_ = y + j * step;
            p->xpos[n] = nx_;
            p->ypos[n] = ny_;
            pd_add_to_object(p, n);
            pd_update_from_object(p, n);
            orc_iterate(single);
            if (orc_get_error(single) < best_error) {
                best_error = orc_get_error(single);
                best_x = nx_;
                best_y = ny_;
            }
            memcpy(p->object, object_copy, on * sizeof(double));
            pd_set_result(single, single_copy);
            memcpy(p->result[n], single_copy, sn * sizeof(double));
        }
    free(object_copy);
    free(single_copy);
    p->xpos[n] = best_x;
    p->ypos[n] = best_y;
    if (best_x == x && best_y == y) step = step / 2.0;
    if (!pd_check_position(p, n, step, min_x, max_x, min_y, max_y, ++tries)) {
        p->xpos[n] = x;
        p->ypos[n] = y;
        return 0;
    }
    p->beta = 1.0;
    p->weights_set = 0;
    return 1;
}

/* adjust_positions, PhaseDiverseCDI.c++:232-392; returns 0 for an unknown type */
int orc_pd_adjust_positions(orc_pd *p, int type, int forward, int min_x, int max_x, int min_y,
                            int max_y, double step_size)
{
    if (type != 0 && type != 1) return 0;
    const int parallel_c = p->parallel;
    double *saved_object = p->object;
    const int nx_c = p->nx, ny_c = p->ny, x_min_c = p->x_min, y_min_c = p->y_min;
    const double beta_c = p->beta;
    const int sc = p->scale;
    p->parallel = 0;
    int n = 1, limit = p->nframes;
    if (!forward) {
        n = p->nframes - 2;
        limit = -1;
    }
    double *temp_object = zd(2 * (size_t)p->nx * p->ny);
    for (size_t k = 0; k < (size_t)p->nx * p->ny; ++k) temp_object[2 * k] = 1;
    p->object = temp_object;
    p->beta = 1.0;
    p->weights_set = 0;
    const int first = forward ? 0 : p->nframes - 1;
    orc_iterate(p->frame[first]);
    pd_get_result(p->frame[first], p->result[first]);
    pd_add_to_object(p, first);
    while (n != limit) {
        const double bx = p->xpos[n], by = p->ypos[n];
        const int lnx = p->rnx[0], lny = p->rny[0];
        orc_iterate(p->frame[n]);
        pd_get_result(p->frame[n], p->result[n]);
        const int bnx = lnx * sc, bny = lny * sc;
        if (type == 0) { /* CROSS_CORRELATION */
            double *single = zd((size_t)lnx * lny), *others = zd((size_t)bnx * bny);
            for (int i = 0; i < bnx; ++i)
                for (int j = 0; j < bny; ++j) {
                    const int i_ = (int)(i - bx * sc - p->x_min * sc);
                    const int j_ = (int)(j - by * sc - p->y_min * sc);
                    if (i_ >= 0 && j_ >= 0 && i_ < p->nx && j_ < p->ny) {
                        const double m = mag_of(p->object + 2 * ((size_t)i_ * p->ny + j_));
                        if (m < 1) others[(size_t)i * bny + j] = 1 - m;
                    }
                    if (i < lnx && j < lny) {
                        const double m = mag_of(p->result[n] + 2 * ((size_t)i * p->rny[n] + j));
                        if (m < 1) single[(size_t)i * lny + j] = 1 - m;
                    }
                }
            double *single_int, *weight_int = zd((size_t)bnx * bny);
            orc_solver *f = p->frame[n];
            if (sc == 1) {
                single_int = single;
                memcpy(weight_int, f->support, sizeof(double) * (size_t)bnx * bny);
            } else {
                single_int = zd((size_t)bnx * bny);
                pd_interpolate(single, lnx, lny, single_int, sc);
                pd_interpolate(f->support, f->nx, f->ny, weight_int, sc);
            }
            int new_x = 0, new_y = 0;
            orc_align(single_int, bnx, bny, others, bnx, bny, &new_x, &new_y, min_x, max_x, min_y,
                      max_y, weight_int, others, 0.2);
            p->xpos[n] = bx + new_x / ((double)sc);
            p->ypos[n] = by + new_y / ((double)sc);
            if (single_int != single) free(single_int);
            free(single);
            free(others);
            free(weight_int);
        } else { /* MINIMUM_ERROR */
            double *temp = zd(2 * (size_t)bnx * bny);
            for (int i = 0; i < bnx; ++i)
                for (int j = 0; j < bny; ++j) {
                    const int i_ = (int)(i - bx * sc - p->x_min * sc);
                    const int j_ = (int)(j - by * sc - p->y_min * sc);
                    if (i_ >= 0 && j_ >= 0 && i_ < p->nx && j_ < p->ny) {
                        temp[2 * ((size_t)i * bny + j)] = p->object[2 * ((size_t)i_ * p->ny + j_)];
                        temp[2 * ((size_t)i * bny + j) + 1] = p->object[2 * ((size_t)i_ * p->ny + j_) + 1];
                    }
                }
            p->object = temp;
            p->nx = bnx;
            p->ny = bny;
            p->x_min = (int)(-p->xpos[n]);
            p->y_min = (int)(-p->ypos[n]);
            pd_check_position(p, n, step_size, min_x, max_x, min_y, max_y, 0);
            free(temp);
            p->object = temp_object;
            p->nx = nx_c;
            p->ny = ny_c;
            p->x_min = x_min_c;
            p->y_min = y_min_c;
        }
        p->weights_set = 0;
        pd_add_to_object(p, n);
        n += forward ? 1 : -1;
    }
    free(temp_object);
    p->object = saved_object;
    p->nx = nx_c;
    p->ny = ny_c;
    p->x_min = x_min_c;
    p->y_min = y_min_c;
    p->parallel = parallel_c;
    p->beta = beta_c;
    p->weights_set = 0;
    return 1;
}
