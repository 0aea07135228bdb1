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
