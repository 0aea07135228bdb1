// ref_driver.cpp -- TEST INFRASTRUCTURE (oracle). Not part of the product.
//
// A C entry layer over the reference's own classes (PlanarCDI, FresnelCDI,
// PolyCDI over BaseCDI), compiled by oracle/build_oracle.py together with the
// unmodified reference sources and the FFTW shim into oracle/_ref/*.so.  Its
// functions mirror the oracle restatement's (orc_*) so the tests can drive the
// reference, the restatement and the CUDA library with the same calls.
// Arrays are doubles, element (x,y) at x*ny+y, complex interleaved; they are
// converted to the build's precision (float by default, double with
// -DDOUBLE_PRECISION: NADIA/include/Complex_2D.h:511-515).
#include <cstdlib>
#include <cstring>
#include <string>
#include <Complex_2D.h>
#include <Double_2D.h>
#include <BaseCDI.h>
#include <PlanarCDI.h>
#include <FresnelCDI.h>
#include <FresnelCDI_WF.h>
#include <PolyCDI.h>
#include <TransmissionConstraint.h>
#include <PhaseDiverseCDI.h>
#include <vector>

namespace {

enum { KIND_PLANAR = 0, KIND_FRESNEL = 1, KIND_POLY = 2, KIND_FRESNEL_WF = 3 };

struct RefSolver {
    int kind, nx, ny;
    Complex_2D *esw;
    Complex_2D *wf;
    BaseCDI *cdi;
    // a transmission constraint and its regions (they must outlive the solver's use)
    TransmissionConstraint *tc = nullptr;
    std::vector<Double_2D *> regions;
    std::vector<ComplexConstraint *> constraints;
};

void to_real(Double_2D &d, const double *a, int nx, int ny)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) d.set(i, j, a[(size_t)i * ny + j]);
}

void to_cplx(Complex_2D &c, const double *a)
{
    int nx = c.get_size_x(), ny = c.get_size_y();
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            c.set_real(i, j, a[2 * ((size_t)i * ny + j)]);
            c.set_imag(i, j, a[2 * ((size_t)i * ny + j) + 1]);
        }
}

void from_cplx(const Complex_2D &c, double *a)
{
    int nx = c.get_size_x(), ny = c.get_size_y();
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            a[2 * ((size_t)i * ny + j)] = c.get_real(i, j);
            a[2 * ((size_t)i * ny + j) + 1] = c.get_imag(i, j);
        }
}

RefSolver *S(void *h) { return static_cast<RefSolver *>(h); }

} // namespace

extern "C" {

void *ref_planar_create(int nx, int ny, int n_best)
{
    RefSolver *s = new RefSolver();
    s->kind = KIND_PLANAR; s->nx = nx; s->ny = ny;
    s->esw = new Complex_2D(nx, ny);
    s->wf = 0;
    s->cdi = new PlanarCDI(*s->esw, n_best);
    return s;
}

void ref_set_transmission_constraint(void *h, int enforce_unity, int charge_flip, int flip_sign,
                                     int nregions, const double *regions, const double *alpha,
                                     const double *fixed_c)
{
    RefSolver *s = S(h);
    size_t n = (size_t)s->nx * s->ny;
    s->tc = new TransmissionConstraint();
    s->tc->set_enforce_unity(enforce_unity != 0);
    s->tc->set_charge_flipping(charge_flip != 0, flip_sign);
    for (int r = 0; r < nregions; ++r) {
        Double_2D *d = new Double_2D(s->nx, s->ny);
        to_real(*d, regions + r * n, s->nx, s->ny);
        ComplexConstraint *c = new ComplexConstraint(*d, alpha[2 * r], alpha[2 * r + 1]);
        if (fixed_c && fixed_c[r] == fixed_c[r]) c->set_fixed_c(fixed_c[r]);
        s->regions.push_back(d);
        s->constraints.push_back(c);
        s->tc->add_complex_constraint(*c);
    }
    s->cdi->set_complex_constraint(*s->tc);
}

void *ref_fresnel_wf_create(int nx, int ny, double wavelength, double zone_focal_length,
                            double focal_detector_length, double pixel, int n_best)
{
    RefSolver *s = new RefSolver();
    s->kind = KIND_FRESNEL_WF; s->nx = nx; s->ny = ny;
    s->esw = new Complex_2D(nx, ny);
    s->wf = 0;
    s->cdi = new FresnelCDI_WF(*s->esw, wavelength, zone_focal_length, focal_detector_length,
                               pixel, n_best);
    return s;
}

void ref_fresnel_wf_set_support(void *h, double z_diameter, double size)
{
    static_cast<FresnelCDI_WF *>(S(h)->cdi)->set_support(z_diameter, size);
}

void *ref_fresnel_create(int nx, int ny, const double *white_field, double wavelength,
                         double zfd, double zfs, double pixel, double norm, int n_best)
{
    RefSolver *s = new RefSolver();
    s->kind = KIND_FRESNEL; s->nx = nx; s->ny = ny;
    s->esw = new Complex_2D(nx, ny);
    s->wf = new Complex_2D(nx, ny);
    to_cplx(*s->wf, white_field);
    s->cdi = new FresnelCDI(*s->esw, *s->wf, wavelength, zfd, zfs, pixel, norm, n_best);
    return s;
}

void *ref_poly_create(int nx, int ny, double beta, int n_best)
{
    RefSolver *s = new RefSolver();
    s->kind = KIND_POLY; s->nx = nx; s->ny = ny;
    s->esw = new Complex_2D(nx, ny);
    s->wf = 0;
    s->cdi = new PolyCDI(*s->esw, beta, n_best, false);
    return s;
}

void ref_destroy(void *h)
{
    RefSolver *s = S(h);
    delete s->cdi;
    delete s->esw;
    delete s->wf;
    delete s->tc;
    for (ComplexConstraint *c : s->constraints) delete c;
    for (Double_2D *d : s->regions) delete d;
    delete s;
}

void ref_set_support(void *h, const double *a, int soften)
{
    Double_2D d(S(h)->nx, S(h)->ny);
    to_real(d, a, S(h)->nx, S(h)->ny);
    S(h)->cdi->set_support(d, soften != 0);
}

void ref_set_intensity(void *h, const double *a)
{
    Double_2D d(S(h)->nx, S(h)->ny);
    to_real(d, a, S(h)->nx, S(h)->ny);
    S(h)->cdi->set_intensity(d);
}

void ref_set_beam_stop(void *h, const double *a)
{
    Double_2D d(S(h)->nx, S(h)->ny);
    to_real(d, a, S(h)->nx, S(h)->ny);
    S(h)->cdi->set_beam_stop(d);
}

void ref_set_algorithm(void *h, int alg) { S(h)->cdi->set_algorithm(alg); }

void ref_set_custom_algorithm(void *h, const double *m)
{
    S(h)->cdi->set_custom_algorithm(m[0], m[1], m[2], m[3], m[4], m[5], m[6], m[7], m[8], m[9]);
}

void ref_set_relaxation_parameter(void *h, double b) { S(h)->cdi->set_relaxation_parameter(b); }

void ref_initialise_estimate(void *h, int seed) { S(h)->cdi->initialise_estimate(seed); }

void ref_set_esw(void *h, const double *a)
{
    Complex_2D c(S(h)->nx, S(h)->ny);
    to_cplx(c, a);
    S(h)->cdi->set_exit_surface_wave(c);
}

void ref_get_esw(void *h, double *a) { from_cplx(*S(h)->esw, a); }

void ref_iterate(void *h) { S(h)->cdi->iterate(); }

double ref_get_error(void *h) { return S(h)->cdi->get_error(); }

void ref_apply_shrinkwrap(void *h, double w, double t) { S(h)->cdi->apply_shrinkwrap(w, t); }

void ref_get_support(void *h, double *a)
{
    const Double_2D &d = S(h)->cdi->get_support();
    int nx = S(h)->nx, ny = S(h)->ny;
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) a[(size_t)i * ny + j] = d.get(i, j);
}

void ref_get_transmission(void *h, double *a)
{
    RefSolver *s = S(h);
    if (s->kind == KIND_FRESNEL) {
        Complex_2D t(s->nx, s->ny);
        static_cast<FresnelCDI *>(s->cdi)->get_transmission_function(t);
        from_cplx(t, a);
    } else {
        from_cplx(*s->esw, a);
    }
}

void ref_set_transmission(void *h, const double *a)
{
    RefSolver *s = S(h);
    Complex_2D t(s->nx, s->ny);
    to_cplx(t, a);
    if (s->kind == KIND_FRESNEL)
        static_cast<FresnelCDI *>(s->cdi)->set_transmission_function(t);
    else
        s->cdi->set_exit_surface_wave(t);
}

void ref_get_illumination_at_sample(void *h, double *a)
{
    RefSolver *s = S(h);
    if (s->kind == KIND_FRESNEL)
        from_cplx(static_cast<FresnelCDI *>(s->cdi)->get_illumination_at_sample(), a);
}

void ref_fresnel_auto_set_norm(void *h) { static_cast<FresnelCDI *>(S(h)->cdi)->auto_set_norm(); }

void ref_fresnel_set_norm(void *h, double n) { static_cast<FresnelCDI *>(S(h)->cdi)->set_norm(n); }

void ref_poly_set_spectrum(void *h, const double *wl_weight, int n)
{
    Double_2D d(n, 2);
    for (int i = 0; i < n; ++i) {
        d.set(i, 0, wl_weight[2 * i]);
        d.set(i, 1, wl_weight[2 * i + 1]);
    }
    static_cast<PolyCDI *>(S(h)->cdi)->set_spectrum(d);
}

void ref_poly_set_spectrum_file(void *h, const char *path)
{
    static_cast<PolyCDI *>(S(h)->cdi)->set_spectrum(std::string(path));
}

// PolyCDI::expand_wl on a field of fx x fy (PolyCDI.c++:296-334), then
// get_intensity (PolyCDI.h:244-246) into out (the solver's nx x ny)
void ref_poly_expand_wl(void *h, const double *field, int fx, int fy, double *out)
{
    PolyCDI *p = static_cast<PolyCDI *>(S(h)->cdi);
    Complex_2D c(fx, fy);
    to_cplx(c, field);
    p->expand_wl(c);
    Double_2D r = p->get_intensity();
    for (int i = 0; i < S(h)->nx; ++i)
        for (int j = 0; j < S(h)->ny; ++j) out[(size_t)i * S(h)->ny + j] = r.get(i, j);
}

int ref_get_best_result(void *h, int index, double *err, double *a)
{
    double e = 0;
    Complex_2D *c = S(h)->cdi->get_best_result(e, index);
    if (!c) return 0;
    *err = e;
    from_cplx(*c, a);
    return 1;
}

void ref_reset_best(void *h) { S(h)->cdi->reset_best(); }

void ref_propagate_to_detector(void *h, double *a)
{
    Complex_2D c(S(h)->nx, S(h)->ny);
    to_cplx(c, a);
    S(h)->cdi->propagate_to_detector(c);
    from_cplx(c, a);
}

void ref_propagate_from_detector(void *h, double *a)
{
    Complex_2D c(S(h)->nx, S(h)->ny);
    to_cplx(c, a);
    S(h)->cdi->propagate_from_detector(c);
    from_cplx(c, a);
}

void ref_scale_intensity(void *h, double *a)
{
    Complex_2D c(S(h)->nx, S(h)->ny);
    to_cplx(c, a);
    S(h)->cdi->scale_intensity(c);
    from_cplx(c, a);
}

void ref_apply_support(void *h, double *a)
{
    Complex_2D c(S(h)->nx, S(h)->ny);
    to_cplx(c, a);
    S(h)->cdi->apply_support(c);
    from_cplx(c, a);
}

void ref_project_intensity(void *h, double *a)
{
    Complex_2D c(S(h)->nx, S(h)->ny);
    to_cplx(c, a);
    S(h)->cdi->project_intensity(c);
    from_cplx(c, a);
}

void ref_get_intensity_autocorrelation(void *h, double *a)
{
    RefSolver *s = S(h);
    Double_2D d(s->nx, s->ny);
    static_cast<PlanarCDI *>(s->cdi)->get_intensity_autocorrelation(d);
    for (int i = 0; i < s->nx; ++i)
        for (int j = 0; j < s->ny; ++j) a[(size_t)i * s->ny + j] = d.get(i, j);
}

int ref_precision_bytes(void) { return (int)sizeof(((Double_2D *)0)->get(0, 0)); }

/* ---- PhaseDiverseCDI (NADIA/include/PhaseDiverseCDI.h) over RefSolver frames */

void *ref_pd_create(double beta, double gamma, int parallel, int granularity)
{
    return new PhaseDiverseCDI(beta, gamma, parallel != 0, granularity);
}

void ref_pd_destroy(void *pd) { delete static_cast<PhaseDiverseCDI *>(pd); }

void ref_pd_add_position(void *pd, void *frame, double x, double y, double alpha)
{
    static_cast<PhaseDiverseCDI *>(pd)->add_new_position(S(frame)->cdi, x, y, alpha);
}

void ref_pd_remove_positions(void *pd) { static_cast<PhaseDiverseCDI *>(pd)->remove_positions(); }

void ref_pd_initialise_estimate(void *pd)
{
    static_cast<PhaseDiverseCDI *>(pd)->initialise_estimate();
}

void ref_pd_iterate(void *pd) { static_cast<PhaseDiverseCDI *>(pd)->iterate(); }

void ref_pd_set_iterations_per_cycle(void *pd, int n)
{
    static_cast<PhaseDiverseCDI *>(pd)->set_iterations_per_cycle(n);
}

void ref_pd_set_feedback_parameter(void *pd, double b)
{
    static_cast<PhaseDiverseCDI *>(pd)->set_feedback_parameter(b);
}

void ref_pd_set_amplification_factor(void *pd, double g)
{
    static_cast<PhaseDiverseCDI *>(pd)->set_amplification_factor(g);
}

void ref_pd_set_probe_scaling(void *pd, int n, double alpha)
{
    static_cast<PhaseDiverseCDI *>(pd)->set_probe_scaling(n, alpha);
}

void ref_pd_get_size(void *pd, int *nx, int *ny)
{
    Complex_2D *o = static_cast<PhaseDiverseCDI *>(pd)->get_transmission();
    *nx = o ? o->get_size_x() : 0;
    *ny = o ? o->get_size_y() : 0;
}

void ref_pd_get_transmission(void *pd, double *a)
{
    from_cplx(*static_cast<PhaseDiverseCDI *>(pd)->get_transmission(), a);
}

void ref_pd_set_transmission(void *pd, int nx, int ny, const double *a)
{
    Complex_2D t(nx, ny);
    to_cplx(t, a);
    static_cast<PhaseDiverseCDI *>(pd)->set_transmission(t);
}

void ref_pd_adjust_positions(void *pd, int type, int forward, int min_x, int max_x, int min_y,
                             int max_y, double step_size)
{
    static_cast<PhaseDiverseCDI *>(pd)->adjust_positions(type, forward != 0, min_x, max_x, min_y,
                                                         max_y, step_size);
}

double ref_pd_get_x(void *pd, int n)
{
    return static_cast<PhaseDiverseCDI *>(pd)->get_final_x_position(n);
}

double ref_pd_get_y(void *pd, int n)
{
    return static_cast<PhaseDiverseCDI *>(pd)->get_final_y_position(n);
}

} // extern "C"
