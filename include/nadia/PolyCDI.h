// PolyCDI.h -- drop-in for the reference's PolyCDI
// (NADIA/include/PolyCDI.h:36-300): polychromatic CDI on the GPU, in the
// FP64 form (the FP32 form covers PlanarCDI and FresnelCDI).
#ifndef NADIA_DROPIN_POLYCDI_H
#define NADIA_DROPIN_POLYCDI_H

#include <string>

#include "BaseCDI.h"

#define WL 0
#define WEIGHT 1

class PolyCDI : public BaseCDI {
public:
    // PolyCDI(initial_guess, beta, n_best, parallel) -- PolyCDI.c++:25-35.
    // As in the reference, beta is stored but does not reach the algorithm
    // weights (PolyCDI.h:53); `parallel` is accepted and ignored.
    PolyCDI(Complex_2D &initial_guess, double beta = 0.9, int n_best = 1, bool parallel = 0)
        : BaseCDI(initial_guess, n_best)
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
    }

    // PolyCDI::set_spectrum(string) -- PolyCDI.c++:38-63
    void set_spectrum(std::string file_name)
    {
        nadia_cxx::check(nadia_poly_set_spectrum_file(h, file_name.c_str()));
    }

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
};

#endif
