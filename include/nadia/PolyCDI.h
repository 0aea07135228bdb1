// PolyCDI.h -- drop-in for the reference's PolyCDI
// (NADIA/include/PolyCDI.h:36-300): polychromatic CDI on the GPU, in the
// FP64 form (the FP32 form covers PlanarCDI and FresnelCDI).
#ifndef NADIA_DROPIN_POLYCDI_H
#define NADIA_DROPIN_POLYCDI_H

#include <cmath>
#include <string>
#include <vector>

#include "BaseCDI.h"

#define WL 0
#define WEIGHT 1

namespace nadia_cxx {

// The part of PolyCDI::set_spectrum (PolyCDI.c++:66-89) that the public
// expand_wl / get_intensity need on the host: the spectrum with its weights
// normalised to sum 1, the central wavelength (the first one of maximum
// weight) and the padding of each axis, (lambda_0 / lambda_c - 1) * n / 2
// truncated.  The same operations in the same order as the reference.
struct PolySpectrum {
    Double_2D spectrum;
    double lambdac = 0;
    int nlambda = 0, paddingx = 0, paddingy = 0;

    void set(const Double_2D &in, int nx, int ny)
    {
        spectrum = in;
        nlambda = spectrum.get_size_x();
        double maxweight = 0;
        double totweight = 0;
        for (int i = 0; i < nlambda; ++i) {
            if (spectrum.get(i, WEIGHT) > maxweight) {
                lambdac = spectrum.get(i, WL);
                maxweight = spectrum.get(i, WEIGHT);
            }
            totweight += spectrum.get(i, WEIGHT);
        }
        for (int i = 0; i < nlambda; ++i) spectrum.set(i, WEIGHT, spectrum.get(i, WEIGHT) / totweight);
        if (nlambda > 0) {
            paddingx = (int)((spectrum.get(0, WL) / lambdac - 1.0) * nx / 2);
            paddingy = (int)((spectrum.get(0, WL) / lambdac - 1.0) * ny / 2);
        }
    }
};

// PolyCDI::expand_wl (PolyCDI.c++:296-334) on the host: on the grid padded
// by (paddingx, paddingy), the intensity of the detector-plane field c summed
// over the wavelengths, each sampled at lf * (i - nx/2) + nx/2 (lf = lambda /
// lambda_c, coordinates truncated, points outside c skipped); the square
// root of the central nx x ny window goes to out.
inline void poly_expand_wl(const PolySpectrum &s, int nx, int ny, const Complex_2D &c,
                           Double_2D &out)
{
    const int px = s.paddingx, py = s.paddingy;
    if (px < 0 || py < 0) throw Failure(NADIA_ERR_INVALID, "negative PolyCDI padding");
    Double_2D pad(nx + 2 * px, ny + 2 * py);
    for (int sn = 0; sn < s.nlambda; ++sn) {
        const double lambda = s.spectrum.get(sn, WL);
        const double weightl = s.spectrum.get(sn, WEIGHT);
        const double lf = lambda / s.lambdac;
        for (int i = 0; i < nx + 2 * px; ++i)
            for (int j = 0; j < ny + 2 * py; ++j) {
                const double xval = lf * (i - nx / 2.0) + nx / 2.0;
                const double yval = lf * (j - ny / 2.0) + ny / 2.0;
                if (xval >= 0 && xval < c.get_size_x() && yval >= 0 && yval < c.get_size_y())
                    pad.set(i, j, pad.get(i, j) +
                                      weightl * std::pow(c.get_mag((int)xval, (int)yval), 2));
            }
    }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) out.set(i, j, std::sqrt(pad.get(i + px, j + py)));
}

} // namespace nadia_cxx

class PolyCDI : public BaseCDI {
public:
    // PolyCDI(initial_guess, beta, n_best, parallel) -- PolyCDI.c++:25-35.
    // As in the reference, beta is stored but does not reach the algorithm
    // weights (PolyCDI.h:53); `parallel` is accepted and ignored.
    PolyCDI(Complex_2D &initial_guess, double beta = 0.9, int n_best = 1, bool parallel = 0)
        : BaseCDI(initial_guess, n_best), intensity_sqrt_calc(nx, ny)
    {
        (void)parallel;
        nadia_solver *s = nullptr;
        nadia_cxx::check(nadia_poly_create(nx, ny, NADIA_FP64, beta, n_best, &s));
        adopt(s);
    }

    // PolyCDI::initialise_estimate -- PolyCDI.c++:102-126
    void initialise_estimate() { BaseCDI::initialise_estimate(0); }
    void initialise_estimate(int seed) { BaseCDI::initialise_estimate(seed); }

    // PolyCDI::set_spectrum(Double_2D) -- PolyCDI.c++:66-89: rows of
    // (wavelength, weight), longest wavelength first
    void set_spectrum(Double_2D spectrum_in)
    {
        const int nl = spectrum_in.get_size_x();
        std::vector<double> d((size_t)2 * nl);
        for (int i = 0; i < nl; ++i) {
            d[2 * i] = spectrum_in.get(i, WL);
            d[2 * i + 1] = spectrum_in.get(i, WEIGHT);
        }
        nadia_cxx::check(nadia_poly_set_spectrum(h, d.data(), nl));
        spec.set(spectrum_in, nx, ny);
    }

    // PolyCDI::set_spectrum(string) -- PolyCDI.c++:38-63
    void set_spectrum(std::string file_name)
    {
        nadia_cxx::check(nadia_poly_set_spectrum_file(h, file_name.c_str()));
        int nrows = 0;
        nadia_cxx::check(nadia_read_spec(file_name.c_str(), nullptr, 0, &nrows));
        std::vector<double> rows((size_t)2 * nrows);
        nadia_cxx::check(nadia_read_spec(file_name.c_str(), rows.data(), nrows, &nrows));
        Double_2D d(nrows, 2);
        for (int i = 0; i < nrows; ++i) {
            d.set(i, WL, rows[2 * i]);
            d.set(i, WEIGHT, rows[2 * i + 1]);
        }
        spec.set(d, nx, ny);
    }

    // PolyCDI::expand_wl (PolyCDI.c++:296-334): the polychromatic intensity
    // of a detector-plane field (for simulations: PolyCDI_simulation_example.c
    // propagates an object with propagate_to_detector first), computed on the
    // host in the build's precision; read it with get_intensity().  The
    // reconstruction's own expansion runs on the GPU inside iterate().
    void expand_wl(Complex_2D &c) { nadia_cxx::poly_expand_wl(spec, nx, ny, c, intensity_sqrt_calc); }

    // PolyCDI::get_intensity (PolyCDI.h:244-246): the square root of the
    // intensity the last expand_wl formed (zeros before the first)
    Double_2D get_intensity() { return intensity_sqrt_calc; }

    // PolyCDI::get_transmission (PolyCDI.h:210, declared without a
    // definition in the reference): the current estimate
    Complex_2D get_transmission()
    {
        Complex_2D t(nx, ny);
        std::vector<double> d((size_t)2 * nx * ny);
        nadia_cxx::check(nadia_get_transmission(h, d.data()));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                t.set_real(i, j, d[2 * ((size_t)i * ny + j)]);
                t.set_imag(i, j, d[2 * ((size_t)i * ny + j) + 1]);
            }
        return t;
    }

    // PolyCDI::set_transmission -- PolyCDI.h:220
    void set_transmission(Complex_2D &new_transmission) { set_exit_surface_wave(new_transmission); }

    // PolyCDI::sum_intensity (PolyCDI.c++:404-430): the sum over the fields
    // c[m] of eigen[m] * |c[m]|^2.  The reference never fills its mode
    // weights (eigen), so any non-empty list throws std::out_of_range there,
    // and here; an empty one gives zeros.
    Double_2D sum_intensity(std::vector<Complex_2D> &c)
    {
        Double_2D magnitude(nx, ny);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                double mag_total = 0;
                for (size_t mode = 0; mode < c.size(); ++mode)
                    mag_total += eigen.at(mode) * c.at(mode).get_mag(i, j) * c.at(mode).get_mag(i, j);
                magnitude.set(i, j, mag_total);
            }
        return magnitude;
    }

    // PolyCDI::set_iterations_per_cycle (PolyCDI.h:200-202): stored only;
    // PolyCDI::iterate never reads it in the reference either
    void set_iterations_per_cycle(int iterations) { iterations_per_cycle = iterations; }

private:
    nadia_cxx::PolySpectrum spec;
    Double_2D intensity_sqrt_calc;
    int iterations_per_cycle = 0;
    std::vector<double> eigen; // never filled, as in the reference
};

#endif
