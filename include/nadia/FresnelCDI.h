// FresnelCDI.h -- drop-in for the reference's FresnelCDI
// (NADIA/include/FresnelCDI.h:31-232): Fresnel (curved-beam) CDI on the GPU.
#ifndef NADIA_DROPIN_FRESNELCDI_H
#define NADIA_DROPIN_FRESNELCDI_H

#include "BaseCDI.h"

class FresnelCDI : public BaseCDI {
public:
    // FresnelCDI(initial_guess, white_field, ...) -- FresnelCDI.c++:20-44
    FresnelCDI(Complex_2D &initial_guess, Complex_2D &white_field, double beam_wavelength,
               double focal_detector_length, double focal_sample_length, double pixel_size,
               double normalisation = 1.0, int n_best = 0)
        : BaseCDI(initial_guess, n_best), illumination_at_sample(nx, ny)
    {
        std::vector<double> wf((size_t)2 * nx * ny);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                wf[2 * ((size_t)i * ny + j)] = white_field.get_real(i, j);
                wf[2 * ((size_t)i * ny + j) + 1] = white_field.get_imag(i, j);
            }
        nadia_solver *s = nullptr;
        auto make = [&](int prec) {
            return nadia_fresnel_create(nx, ny, prec, wf.data(), beam_wavelength,
                                        focal_detector_length, focal_sample_length, pixel_size,
                                        normalisation, n_best, &s);
        };
        int rc = make(precision_for(nx, ny));
        if (rc == NADIA_ERR_UNSUPPORTED) rc = make(NADIA_FP64);
        nadia_cxx::check(rc);
        adopt(s);
    }

    // FresnelCDI::auto_set_norm -- FresnelCDI.c++:129-148
    virtual void auto_set_norm() { nadia_cxx::check(nadia_fresnel_auto_set_norm(h)); }

    // FresnelCDI::set_norm -- FresnelCDI.c++:293-296
    void set_norm(double new_normalisation)
    {
        nadia_cxx::check(nadia_fresnel_set_norm(h, new_normalisation));
    }

    // FresnelCDI::set_normalisation -- FresnelCDI.h:187-189
    void set_normalisation(double normalisation)
    {
        nadia_cxx::check(nadia_fresnel_set_normalisation(h, normalisation));
    }

    // FresnelCDI::set_experimental_parameters -- FresnelCDI.c++:57-95
    void set_experimental_parameters(double beam_wavelength, double focal_detector_length,
                                     double focal_sample_length, double pixel_size)
    {
        nadia_cxx::check(nadia_fresnel_set_experimental_parameters(
            h, beam_wavelength, focal_detector_length, focal_sample_length, pixel_size));
    }

    // FresnelCDI::get_illumination_at_sample -- FresnelCDI.c++:285-296
    const Complex_2D &get_illumination_at_sample()
    {
        std::vector<double> d((size_t)2 * nx * ny);
        nadia_cxx::check(nadia_fresnel_get_illumination_at_sample(h, d.data()));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                illumination_at_sample.set_real(i, j, d[2 * ((size_t)i * ny + j)]);
                illumination_at_sample.set_imag(i, j, d[2 * ((size_t)i * ny + j) + 1]);
            }
        return illumination_at_sample;
    }

    // FresnelCDI::get_transmission_function(result, esw) -- FresnelCDI.c++:298-355.
    // Without esw it is computed on the GPU from the current estimate; with a
    // caller's esw the same per-pixel formula runs on the host.
    virtual void get_transmission_function(Complex_2D &result, Complex_2D *esw = 0)
    {
        if (!esw) {
            std::vector<double> d((size_t)2 * nx * ny);
            nadia_cxx::check(nadia_get_transmission(h, d.data()));
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j) {
                    result.set_real(i, j, d[2 * ((size_t)i * ny + j)]);
                    result.set_imag(i, j, d[2 * ((size_t)i * ny + j) + 1]);
                }
            return;
        }
        const Complex_2D &L = get_illumination_at_sample();
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                double lr = L.get_real(i, j), li = L.get_imag(i, j);
                double den = lr * lr + li * li;
                if (den != 0) {
                    double er = esw->get_real(i, j) + lr, ei = esw->get_imag(i, j) + li;
                    result.set_real(i, j, (lr * er + li * ei) / den);
                    result.set_imag(i, j, (lr * ei - li * er) / den);
                } else {
                    result.set_real(i, j, 1.0);
                    result.set_imag(i, j, 0.0);
                }
            }
    }

    // FresnelCDI::set_transmission_function(transmission, esw) --
    // FresnelCDI.c++:253-283: esw = T*L - L (into the estimate when esw is 0)
    virtual void set_transmission_function(Complex_2D &transmission, Complex_2D *esw = 0)
    {
        if (!esw) {
            std::vector<double> d((size_t)2 * nx * ny);
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j) {
                    d[2 * ((size_t)i * ny + j)] = transmission.get_real(i, j);
                    d[2 * ((size_t)i * ny + j) + 1] = transmission.get_imag(i, j);
                }
            upload_host_edits();
            nadia_cxx::check(nadia_set_transmission(h, d.data()));
            estimate_changed_on_device();
            return;
        }
        const Complex_2D &L = get_illumination_at_sample();
        // the reference's loop bounds are (nx, nx) (FresnelCDI.c++:270-271)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < nx && j < ny; ++j) {
                double lr = L.get_real(i, j), li = L.get_imag(i, j);
                double tr = transmission.get_real(i, j), ti = transmission.get_imag(i, j);
                esw->set_real(i, j, lr * tr - li * ti - lr);
                esw->set_imag(i, j, lr * ti + li * tr - li);
            }
    }

private:
    Complex_2D illumination_at_sample;
};

#endif
