// FresnelCDI_WF.h -- drop-in for the reference's FresnelCDI_WF
// (NADIA/include/FresnelCDI_WF.h): recovery of the detector-plane white field
// that FresnelCDI takes as its illumination, on the GPU: in the float build
// in the fused FP32 form where the grid has FP32 tiles (BaseCDI::precision_for),
// else in the FP64 form.  The estimate handed to the constructor is the
// detector-plane field.
#ifndef NADIA_DROPIN_FRESNELCDI_WF_H
#define NADIA_DROPIN_FRESNELCDI_WF_H

#include <iostream>

#include "BaseCDI.h"

class FresnelCDI_WF : public BaseCDI {
public:
    // FresnelCDI_WF(initial_guess, wavelength, zone_focal_length,
    // focal_detector_length, pixel_size, n_best) -- FresnelCDI_WF.c++:17-79
    FresnelCDI_WF(Complex_2D &initial_guess, double beam_wavelength, double zone_focal_length,
                  double focal_detector_length, double pixel_size, int n_best = 0)
        : BaseCDI(initial_guess, n_best)
    {
        nadia_solver *s = nullptr;
        nadia_cxx::check(nadia_fresnel_wf_create(nx, ny, precision_for(nx, ny), beam_wavelength,
                                                 zone_focal_length, focal_detector_length,
                                                 pixel_size, n_best, &s));
        adopt(s);
    }

    // FresnelCDI_WF::set_support(z_diameter, size) -- FresnelCDI_WF.c++:184-203
    // (hides BaseCDI::set_support, as in the reference)
    virtual void set_support(double z_diameter, double size = 1.01)
    {
        nadia_cxx::check(nadia_fresnel_wf_set_support(h, z_diameter, size));
    }

    // the algorithm is fixed (FresnelCDI_WF.h:147-181): warnings, as the reference
    void set_algorithm(int)
    {
        std::cout << "WARNING: Algorithm can not be set when performing Fresnel "
                  << "CDI white field recovery" << std::endl;
    }
    void print_algorithm()
    {
        std::cout << "Using the default Fresnel CDI "
                  << "white field recovery algorithm" << std::endl;
    }
    void set_relaxation_parameter(double)
    {
        std::cout << "WARNING: The relaxation parameter can not "
                  << "set when performing Fresnel white-field "
                  << "reconstruction" << std::endl;
    }
    void set_custom_algorithm(double, double, double, double, double, double, double, double,
                              double, double)
    {
        std::cout << "WARNING: Algorithm can not be set when performing Fresnel "
                  << "CDI white field recovery" << std::endl;
    }
};

#endif
