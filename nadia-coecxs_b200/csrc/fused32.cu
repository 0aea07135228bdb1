// fused32.cu -- placeholder until the fused FP32 engine lands.
#include "fused32.h"
#include "solver.h"

namespace nadia {
struct Fused32::Impl {};
Fused32::Fused32(Solver &) : impl(nullptr)
{
    throw Error(NADIA_ERR_UNSUPPORTED, "FP32 path not built yet");
}
Fused32::~Fused32() {}
#define NOPE throw Error(NADIA_ERR_UNSUPPORTED, "FP32 path not built yet")
void Fused32::upload_support(const double *) { NOPE; }
void Fused32::soften_support() { NOPE; }
void Fused32::upload_intensity() { NOPE; }
void Fused32::upload_beam_stop(const double *) { NOPE; }
void Fused32::set_spectrum() { NOPE; }
void Fused32::upload_illumination() { NOPE; }
void Fused32::set_fresnel_geometry(double) { NOPE; }
void Fused32::scale_illumination(double) { NOPE; }
void Fused32::fresnel_initialise(const double *) { NOPE; }
void Fused32::fresnel_set_transmission(const double *) { NOPE; }
void Fused32::fresnel_get_transmission(double *) { NOPE; }
void Fused32::get_illumination_at_sample(double *) { NOPE; }
void Fused32::set_x(const double *) { NOPE; }
void Fused32::get_x(double *) { NOPE; }
void Fused32::set_x_f32(const float *) { NOPE; }
void Fused32::get_x_f32(float *) { NOPE; }
void Fused32::copy_x_to(float2 *) { NOPE; }
void Fused32::iterate(int) { NOPE; }
void Fused32::shrinkwrap(double, double) { NOPE; }
void Fused32::get_support(double *) { NOPE; }
void Fused32::single_op(int, double *) { NOPE; }
void Fused32::autocorrelation(double *) { NOPE; }
} // namespace nadia
