// fused32.h -- the FP32 engine of one reconstruction.
#pragma once

#include "common.h"

namespace nadia {

struct Solver;

class Fused32 {
public:
    explicit Fused32(Solver &s);
    ~Fused32();

    void upload_support(const double *h);
    void soften_support();
    void upload_intensity();
    void upload_beam_stop(const double *mask);
    void set_spectrum();
    void upload_illumination();
    void set_fresnel_geometry(double factor);
    // FresnelCDI_WF's zone-plate factors (FresnelCDI_WF.c++:31-79), per axis
    void set_wf_geometry();
    void scale_illumination(double f);
    void fresnel_initialise(const double *t);
    void fresnel_set_transmission(const double *t);
    void fresnel_get_transmission(double *t);
    // TransmissionConstraint's per-pixel part (charge flipping, unit
    // magnitude) inside the row pass's support projections
    // and its complex-constraint regions: map[k] = the region (1-based, 0:
    // none) of pixel k in the reference's order, prm = alpha1, alpha2, fixed
    // flag, fixed c_mean per region
    void set_constraint(bool on, bool unity, bool flip, int flip_sign, int nregions = 0,
                        const int *map = nullptr, const double *prm = nullptr);
    bool constrained() const;
    // the result a PhaseDiverseCDI exchanges (Fresnel: the transmission
    // function; else the estimate), natural order, double, on the device
    void transmission_to_device(double2 *dst);
    void transmission_from_device(const double2 *src);
    void get_illumination_at_sample(double *h);
    void set_x(const double *h);
    void get_x(double *h);
    void set_x_f32(const float *h);
    void get_x_f32(float *h);
    void copy_x_to(float2 *dst);
    void iterate(int count);
    void iterate_poly(int count);
    void shrinkwrap(double gauss_width, double threshold);
    void get_support(double *h);
    void single_op(int op, double *field);
    void autocorrelation(double *out);
    // raise NADIA_ERR_CUDA if a device-side wait of this reconstruction gave up
    void check_device_flag();

    struct Impl;
    Impl *impl;
};

} // namespace nadia
