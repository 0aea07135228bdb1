// PlanarCDI.h -- drop-in for the reference's PlanarCDI
// (NADIA/include/PlanarCDI.h:22-46): plane-wave CDI on the GPU.
#ifndef NADIA_DROPIN_PLANARCDI_H
#define NADIA_DROPIN_PLANARCDI_H

#include "BaseCDI.h"

class PlanarCDI : public BaseCDI {
public:
    // PlanarCDI(Complex_2D&, n_best) -- PlanarCDI.h:28-29
    PlanarCDI(Complex_2D &complex, unsigned int n_best = 0) : BaseCDI(complex, (int)n_best)
    {
        nadia_solver *s = nullptr;
        int rc = nadia_planar_create(nx, ny, precision_for(nx, ny), (int)n_best, &s);
        if (rc == NADIA_ERR_UNSUPPORTED) rc = nadia_planar_create(nx, ny, NADIA_FP64, (int)n_best, &s);
        nadia_cxx::check(rc);
        adopt(s);
    }

    // PlanarCDI::get_intensity_autocorrelation -- PlanarCDI.c++:23-35
    virtual void get_intensity_autocorrelation(Double_2D &autoc)
    {
        std::vector<double> d((size_t)nx * ny);
        nadia_cxx::check(nadia_get_intensity_autocorrelation(h, d.data()));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) autoc.set(i, j, d[(size_t)i * ny + j]);
    }
};

#endif
