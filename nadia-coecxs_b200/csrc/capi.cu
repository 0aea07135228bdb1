// capi.cu -- the extern "C" entry points of libnadia_b200 (include/nadia_b200.h).
// Each converts exceptions into status codes and never exits the process.
#include <cstdlib>
#include <cstring>
#include <functional>
#include <new>
#include <string>
#include <vector>

#include "batch.h"
#include "fused32.h"
#include "fused32_impl.h"
#include "phase_diverse.h"
#include "server.h"
#include "solver.h"

using nadia::Error;
using nadia::Solver;

struct nadia_solver {
    Solver *s;
};

struct nadia_phase_diverse {
    nadia::PhaseDiverse *p;
};

namespace {

thread_local std::string g_last_error;

template <class F>
int guard(F &&f)
{
    // allocations outside a handle's call are ordered on the thread's own stream
    struct Reset {
        ~Reset() { nadia::t_alloc_stream = cudaStreamPerThread; }
    } reset;
    try {
        g_last_error.clear();
        nadia::t_alloc_stream = cudaStreamPerThread;
        f();
        return NADIA_OK;
    } catch (const Error &e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        g_last_error = "host allocation failed";
        return NADIA_ERR_NOMEM;
    } catch (const std::exception &e) {
        g_last_error = e.what();
        return NADIA_ERR_CUDA;
    }
}

Solver &S(nadia_solver *h)
{
    if (!h || !h->s) throw Error(NADIA_ERR_INVALID, "null handle");
    NADIA_CUDA(cudaSetDevice(h->s->device));
    nadia::t_alloc_stream = h->s->st; // buffers made during the call follow its stream
    return *h->s;
}

void need(const void *p, const char *what)
{
    if (!p) throw Error(NADIA_ERR_INVALID, std::string("null pointer: ") + what);
}

int create(int kind, int nx, int ny, int prec, int n_best, nadia_solver **out,
           const std::function<void(Solver &)> &init)
{
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        Solver *s = new Solver(kind, nx, ny, prec, n_best);
        try {
            if (init) init(*s);
        } catch (...) {
            delete s;
            throw;
        }
        *out = new nadia_solver{s};
    });
}

// FresnelCDI_WF overrides the algorithm setters with warnings
// (FresnelCDI_WF.h:147-181): its iteration is fixed
Solver &settable(nadia_solver *h)
{
    Solver &s = S(h);
    NADIA_REQUIRE(s.kind != NADIA_FRESNEL_WF, NADIA_ERR_UNSUPPORTED,
                  "the algorithm of a FresnelCDI_WF reconstruction can not be set");
    return s;
}

} // namespace

extern "C" {

const char *nadia_last_error(void) { return g_last_error.c_str(); }

const char *nadia_version(void) { return "nadia_b200 0.1 (sm_100a)"; }

int nadia_planar_create(int nx, int ny, int precision, int n_best, nadia_solver **out)
{
    return create(NADIA_PLANAR, nx, ny, precision, n_best, out, nullptr);
}

int nadia_fresnel_create(int nx, int ny, int precision, const double *white_field,
                         double beam_wavelength, double focal_detector_length,
                         double focal_sample_length, double pixel_size, double normalisation,
                         int n_best, nadia_solver **out)
{
    if (!white_field) {
        g_last_error = "null pointer: white_field";
        return NADIA_ERR_INVALID;
    }
    return create(NADIA_FRESNEL, nx, ny, precision, n_best, out, [&](Solver &s) {
        s.fresnel_init(white_field, beam_wavelength, focal_detector_length, focal_sample_length,
                       pixel_size, normalisation);
    });
}

int nadia_fresnel_wf_create(int nx, int ny, int precision, double beam_wavelength,
                            double zone_focal_length, double focal_detector_length,
                            double pixel_size, int n_best, nadia_solver **out)
{
    return create(NADIA_FRESNEL_WF, nx, ny, precision, n_best, out, [&](Solver &s) {
        s.fresnel_wf_init(beam_wavelength, zone_focal_length, focal_detector_length, pixel_size);
    });
}

int nadia_fresnel_wf_set_support(nadia_solver *h, double z_diameter, double size)
{
    return guard([&] { S(h).fresnel_wf_set_support(z_diameter, size); });
}

int nadia_set_transmission_constraint(nadia_solver *h, int enforce_unity, int charge_flip,
                                      int flip_sign, int nregions, const double *regions,
                                      const double *alpha, const double *fixed_c)
{
    return guard([&] {
        S(h).set_transmission_constraint(enforce_unity, charge_flip, flip_sign, nregions, regions,
                                         alpha, fixed_c);
    });
}

int nadia_set_transmission_custom(nadia_solver *h,
                                  void (*fn)(double *transmission, int nx, int ny, void *user),
                                  void *user)
{
    return guard([&] { S(h).set_transmission_custom(fn, user); });
}

int nadia_clear_transmission_constraint(nadia_solver *h)
{
    return guard([&] { S(h).clear_transmission_constraint(); });
}

int nadia_poly_create(int nx, int ny, int precision, double beta, int n_best,
                      nadia_solver **out)
{
    (void)beta; // PolyCDI.h:53 shadows BaseCDI::beta; the weights never see it
    return create(NADIA_POLY, nx, ny, precision, n_best, out, nullptr);
}

int nadia_destroy(nadia_solver *h)
{
    return guard([&] {
        if (!h) return;
        if (h->s) {
            NADIA_REQUIRE(h->s->pd_refs == 0, NADIA_ERR_STATE,
                          "the reconstruction is a frame of a phase-diverse reconstruction; "
                          "destroy that (or remove its positions) first");
            cudaSetDevice(h->s->device);
            delete h->s;
        }
        delete h;
    });
}

int nadia_get_size(const nadia_solver *h, int *nx, int *ny)
{
    return guard([&] {
        if (!h || !h->s) throw Error(NADIA_ERR_INVALID, "null handle");
        need(nx, "nx");
        need(ny, "ny");
        *nx = h->s->nx;
        *ny = h->s->ny;
    });
}

int nadia_set_support(nadia_solver *h, const double *a, int soften)
{
    return guard([&] { need(a, "support"); S(h).set_support(a, soften != 0); });
}

int nadia_set_intensity(nadia_solver *h, const double *a)
{
    return guard([&] { need(a, "intensity"); S(h).set_intensity(a); });
}

int nadia_set_beam_stop(nadia_solver *h, const double *a)
{
    return guard([&] { need(a, "mask"); S(h).set_beam_stop(a); });
}

int nadia_poly_set_spectrum(nadia_solver *h, const double *wl_weight, int nlambda)
{
    return guard([&] { need(wl_weight, "wl_weight"); S(h).set_spectrum(wl_weight, nlambda); });
}

int nadia_poly_set_spectrum_file(nadia_solver *h, const char *path)
{
    return guard([&] {
        need(path, "path");
        Solver &s = S(h);
        std::vector<double> sp = nadia::read_spec_file(path);
        s.set_spectrum(sp.data(), (int)(sp.size() / 2));
    });
}

int nadia_read_spec(const char *path, double *rows, int capacity, int *nrows)
{
    return guard([&] {
        need(path, "path");
        need(nrows, "nrows");
        NADIA_REQUIRE(capacity >= 0, NADIA_ERR_INVALID, "negative capacity");
        if (capacity > 0) need(rows, "rows");
        std::vector<double> sp = nadia::read_spec_file(path);
        const int n = (int)(sp.size() / 2);
        std::copy(sp.begin(), sp.begin() + 2 * (size_t)std::min(n, capacity), rows);
        *nrows = n;
    });
}

int nadia_convert_to_fp64(nadia_solver *h)
{
    return guard([&] { S(h).convert_to_fp64(); });
}

int nadia_get_precision(const nadia_solver *h, int *precision)
{
    return guard([&] {
        if (!h || !h->s) throw Error(NADIA_ERR_INVALID, "null handle");
        need(precision, "precision");
        *precision = h->s->prec;
    });
}

int nadia_poly_get_padding(const nadia_solver *h, int *px, int *py)
{
    return guard([&] {
        if (!h || !h->s) throw Error(NADIA_ERR_INVALID, "null handle");
        need(px, "px");
        need(py, "py");
        if (!h->s->has_spectrum) throw Error(NADIA_ERR_STATE, "no spectrum set");
        *px = h->s->px;
        *py = h->s->py;
    });
}

int nadia_set_algorithm(nadia_solver *h, int alg)
{
    return guard([&] { settable(h).set_algorithm(alg); });
}

int nadia_set_custom_algorithm(nadia_solver *h, const double m[10])
{
    return guard([&] { need(m, "m"); settable(h).set_custom(m); });
}

int nadia_set_relaxation_parameter(nadia_solver *h, double beta)
{
    return guard([&] { settable(h).set_relaxation_parameter(beta); });
}

int nadia_get_algorithm_structure(const nadia_solver *h, double w[5], int *algorithm)
{
    return guard([&] {
        if (!h || !h->s) throw Error(NADIA_ERR_INVALID, "null handle");
        need(w, "w");
        for (int i = 0; i < 5; ++i) w[i] = h->s->w[i];
        if (algorithm) *algorithm = h->s->algorithm;
    });
}

void nadia_custom_weights(const double m[10], double w[5])
{
    // BaseCDI.c++:245-249
    w[0] = m[0] + m[1] + m[2] + m[3];
    w[1] = -m[0] + m[4] + m[5] + m[6];
    w[2] = -m[2] - m[5] - m[7] + m[9];
    w[3] = -m[1] - m[4] + m[7] + m[8];
    w[4] = -m[3] - m[6] - m[8] - m[9];
}

int nadia_initialise_estimate(nadia_solver *h, int seed)
{
    return guard([&] { S(h).initialise_estimate(seed); });
}

int nadia_set_exit_surface_wave(nadia_solver *h, const double *a)
{
    return guard([&] { need(a, "esw"); S(h).set_esw(a); });
}

int nadia_get_exit_surface_wave(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "esw"); S(h).get_esw(a); });
}

int nadia_set_exit_surface_wave_f32(nadia_solver *h, const float *a)
{
    return guard([&] { need(a, "esw"); S(h).set_esw_f32(a); });
}

int nadia_get_exit_surface_wave_f32(nadia_solver *h, float *a)
{
    return guard([&] { need(a, "esw"); S(h).get_esw_f32(a); });
}

int nadia_iterate(nadia_solver *h, int iterations)
{
    nadia::Range range("nadia_iterate");
    return guard([&] { S(h).iterate(iterations); });
}

int nadia_get_error(nadia_solver *h, double *e)
{
    return guard([&] { need(e, "error"); *e = S(h).get_error(); });
}

int nadia_get_error_history(nadia_solver *h, double *e, int count)
{
    return guard([&] { need(e, "errors"); S(h).get_error_history(e, count); });
}

int nadia_apply_shrinkwrap(nadia_solver *h, double gauss_width, double threshold)
{
    nadia::Range range("nadia_apply_shrinkwrap");
    return guard([&] { S(h).apply_shrinkwrap(gauss_width, threshold); });
}

int nadia_get_support(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "support"); S(h).get_support(a); });
}

int nadia_get_best_result(nadia_solver *h, int index, double *error, double *esw)
{
    return guard([&] {
        need(error, "error");
        need(esw, "esw");
        S(h).get_best(index, error, esw);
    });
}

int nadia_reset_best(nadia_solver *h)
{
    return guard([&] { S(h).reset_best(); });
}

int nadia_get_transmission(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "transmission"); S(h).get_transmission(a); });
}

int nadia_set_transmission(nadia_solver *h, const double *a)
{
    return guard([&] { need(a, "transmission"); S(h).set_transmission(a); });
}

int nadia_fresnel_auto_set_norm(nadia_solver *h)
{
    return guard([&] { S(h).fresnel_auto_set_norm(); });
}

int nadia_fresnel_set_norm(nadia_solver *h, double nn)
{
    return guard([&] { S(h).fresnel_set_norm(nn); });
}

int nadia_fresnel_get_illumination_at_sample(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "illumination"); S(h).get_illumination_at_sample(a); });
}

int nadia_fresnel_set_experimental_parameters(nadia_solver *h, double wl, double zfd, double zfs,
                                              double pixel)
{
    return guard([&] {
        Solver &s = S(h);
        NADIA_REQUIRE(s.kind == NADIA_FRESNEL, NADIA_ERR_INVALID, "needs a FresnelCDI handle");
        s.fresnel_set_experimental_parameters(wl, zfd, zfs, pixel);
    });
}

int nadia_fresnel_set_normalisation(nadia_solver *h, double nn)
{
    return guard([&] {
        Solver &s = S(h);
        NADIA_REQUIRE(s.kind == NADIA_FRESNEL, NADIA_ERR_INVALID, "needs a FresnelCDI handle");
        s.norm = nn;
    });
}

int nadia_propagate_to_detector(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "field"); S(h).single_op(0, a); });
}

int nadia_propagate_from_detector(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "field"); S(h).single_op(1, a); });
}

int nadia_scale_intensity(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "field"); S(h).single_op(2, a); });
}

int nadia_apply_support(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "field"); S(h).single_op(3, a); });
}

int nadia_project_intensity(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "field"); S(h).single_op(4, a); });
}

int nadia_get_intensity_autocorrelation(nadia_solver *h, double *a)
{
    return guard([&] { need(a, "autoc"); S(h).autocorrelation(a); });
}

int nadia_fft2d(double *a, int nx, int ny, int forward)
{
    return guard([&] {
        need(a, "field");
        NADIA_REQUIRE(nx >= 1 && ny >= 1, NADIA_ERR_INVALID, "grid sizes must be positive");
        cudaStream_t st;
        NADIA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        try {
            nadia::plain::Fft2d fft;
            fft.init(nx, ny);
            nadia::DevBuf<double2> d((size_t)nx * ny);
            NADIA_CUDA(cudaMemcpyAsync(d.p, a, d.bytes(), cudaMemcpyHostToDevice, st));
            fft.exec(d.p, forward != 0, st);
            NADIA_CUDA(cudaMemcpyAsync(a, d.p, d.bytes(), cudaMemcpyDeviceToHost, st));
            NADIA_CUDA(cudaStreamSynchronize(st));
        } catch (...) {
            cudaStreamDestroy(st);
            throw;
        }
        cudaStreamDestroy(st);
    });
}

int nadia_synchronize(nadia_solver *h)
{
    return guard([&] { S(h).sync(); });
}

/* ---- PhaseDiverseCDI ------------------------------------------------------- */

namespace {
nadia::PhaseDiverse &P(nadia_phase_diverse *h)
{
    if (!h || !h->p) throw Error(NADIA_ERR_INVALID, "null phase-diverse handle");
    NADIA_CUDA(cudaSetDevice(h->p->device));
    nadia::t_alloc_stream = h->p->st;
    return *h->p;
}
} // namespace

int nadia_pd_create(double beta, double gamma, int parallel, int granularity,
                    nadia_phase_diverse **out)
{
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        nadia_phase_diverse *h = new nadia_phase_diverse{nullptr};
        try {
            h->p = new nadia::PhaseDiverse(beta, gamma, parallel != 0, granularity);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

int nadia_pd_destroy(nadia_phase_diverse *h)
{
    return guard([&] {
        if (!h) return;
        if (h->p) {
            cudaSetDevice(h->p->device);
            delete h->p;
        }
        delete h;
    });
}

int nadia_pd_add_position(nadia_phase_diverse *h, nadia_solver *frame, double x, double y,
                          double alpha)
{
    return guard([&] {
        nadia::PhaseDiverse &p = P(h);
        if (!frame || !frame->s) throw Error(NADIA_ERR_INVALID, "null frame handle");
        p.add_position(frame->s, x, y, alpha);
    });
}

int nadia_pd_remove_positions(nadia_phase_diverse *h)
{
    return guard([&] { P(h).remove_positions(); });
}

int nadia_pd_initialise_estimate(nadia_phase_diverse *h)
{
    return guard([&] { P(h).initialise_estimate(); });
}

int nadia_pd_iterate(nadia_phase_diverse *h, int cycles)
{
    return guard([&] {
        NADIA_REQUIRE(cycles >= 0, NADIA_ERR_INVALID, "negative cycle count");
        nadia::PhaseDiverse &p = P(h);
        for (int c = 0; c < cycles; ++c) p.iterate();
    });
}

int nadia_pd_set_iterations_per_cycle(nadia_phase_diverse *h, int iterations)
{
    return guard([&] {
        NADIA_REQUIRE(iterations >= 0, NADIA_ERR_INVALID, "negative iteration count");
        P(h).iterations_per_cycle = iterations;
    });
}

int nadia_pd_set_feedback_parameter(nadia_phase_diverse *h, double beta)
{
    return guard([&] { P(h).set_feedback_parameter(beta); });
}

int nadia_pd_set_amplification_factor(nadia_phase_diverse *h, double gamma)
{
    return guard([&] { P(h).set_amplification_factor(gamma); });
}

int nadia_pd_set_probe_scaling(nadia_phase_diverse *h, int n_probe, double alpha)
{
    return guard([&] {
        NADIA_REQUIRE(P(h).set_probe_scaling(n_probe, alpha), NADIA_ERR_RANGE,
                      "the probe number given is too large (set the scaling after "
                      "add_new_position)");
    });
}

int nadia_pd_get_size(const nadia_phase_diverse *h, int *nx, int *ny)
{
    return guard([&] {
        if (!h || !h->p) throw Error(NADIA_ERR_INVALID, "null phase-diverse handle");
        need(nx, "nx");
        need(ny, "ny");
        *nx = h->p->obj ? h->p->nx : 0;
        *ny = h->p->obj ? h->p->ny : 0;
    });
}

int nadia_pd_get_transmission(nadia_phase_diverse *h, double *out)
{
    return guard([&] {
        need(out, "out");
        P(h).get_transmission(out);
    });
}

int nadia_pd_set_transmission(nadia_phase_diverse *h, int nx, int ny, const double *t)
{
    return guard([&] {
        need(t, "t");
        P(h).set_transmission(nx, ny, t);
    });
}

int nadia_pd_adjust_positions(nadia_phase_diverse *h, int type, int forward, int min_x,
                              int max_x, int min_y, int max_y, double step_size)
{
    return guard([&] {
        P(h).adjust_positions(type, forward != 0, min_x, max_x, min_y, max_y, step_size);
    });
}

int nadia_pd_get_position(const nadia_phase_diverse *h, int n_probe, double *x, double *y)
{
    return guard([&] {
        if (!h || !h->p) throw Error(NADIA_ERR_INVALID, "null phase-diverse handle");
        need(x, "x");
        need(y, "y");
        NADIA_REQUIRE(n_probe >= 0 && n_probe < (int)h->p->xpos.size(), NADIA_ERR_RANGE,
                      "no such position");
        *x = h->p->xpos[n_probe];
        *y = h->p->ypos[n_probe];
    });
}

} // extern "C"

extern "C" int nadia_iterate_many(nadia_solver *const *solvers, int count, int iterations)
{
    nadia::Range range("nadia_iterate_many");
    return guard([&] {
        need(solvers, "solvers");
        std::vector<Solver *> v;
        for (int i = 0; i < count; ++i) v.push_back(&S(solvers[i]));
        nadia::iterate_many(v.data(), count, iterations);
    });
}

extern "C" int nadia_get_stream(nadia_solver *h, void **stream)
{
    return guard([&] {
        need(stream, "stream");
        *stream = (void *)S(h).st;
    });
}

extern "C" int nadia_pass_times(nadia_solver *const *solvers, int count, int reps, double out_us[3])
{
    return guard([&] {
        need(solvers, "solvers");
        need(out_us, "out_us");
        std::vector<Solver *> v;
        for (int i = 0; i < count; ++i) v.push_back(&S(solvers[i]));
        nadia::pass_times(v.data(), count, reps, out_us);
    });
}

extern "C" long long nadia_launch_count(void) { return nadia::g_launches.load(); }

namespace nadia {
namespace noalloc {
void shrinkwrap(const float *esw, float *support, int nx, int ny, double gauss_width,
                double threshold, cudaStream_t st);
}
} // namespace nadia

extern "C" int nadia_shrinkwrap_noalloc_f32(const float *esw_dev, float *support_dev, int nx,
                                            int ny, double gauss_width, double threshold,
                                            void *stream)
{
    return guard([&] {
        nadia::noalloc::shrinkwrap(esw_dev, support_dev, nx, ny, gauss_width, threshold,
                                   static_cast<cudaStream_t>(stream));
        nadia::g_launches += 5;
    });
}

// ---- serving (server.h) -----------------------------------------------------

struct nadia_server {
    nadia::Server *srv;
};

namespace {
nadia::Server &SV(nadia_server *h)
{
    if (!h || !h->srv) throw Error(NADIA_ERR_INVALID, "null server");
    return *h->srv;
}
} // namespace

extern "C" int nadia_server_create(unsigned long long budget_bytes, int max_active, int chunk,
                                   nadia_server **out)
{
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        std::unique_ptr<nadia::Server> s(new nadia::Server((size_t)budget_bytes, max_active, chunk));
        *out = new nadia_server{s.release()};
    });
}

extern "C" int nadia_server_submit(nadia_server *h, const nadia_request *req, long long *id)
{
    return guard([&] {
        need(req, "request");
        need(id, "id");
        *id = SV(h).submit(*req);
    });
}

extern "C" int nadia_server_wait(nadia_server *h, long long id, double timeout_s, int *done)
{
    return guard([&] {
        need(done, "done");
        *done = SV(h).wait(id, timeout_s) ? 1 : 0;
    });
}

extern "C" int nadia_server_result(nadia_server *h, long long id, double *esw, double *support,
                                   double *final_error, double times[3])
{
    return guard([&] { SV(h).result(id, esw, support, final_error, times); });
}

extern "C" int nadia_server_stats(nadia_server *h, long long out[12])
{
    return guard([&] {
        need(out, "out");
        SV(h).stats(out);
    });
}

extern "C" int nadia_server_destroy(nadia_server *h)
{
    return guard([&] {
        if (!h) return;
        delete h->srv;
        delete h;
    });
}

extern "C" int nadia_estimate_device_bytes(int kind, int nx, int ny, int precision, int n_best,
                                           int poly_pad_x, int poly_pad_y, int nlambda,
                                           unsigned long long *bytes)
{
    return guard([&] {
        need(bytes, "bytes");
        NADIA_REQUIRE(nx > 0 && ny > 0 && n_best >= 0 && poly_pad_x >= 0 && poly_pad_y >= 0 &&
                          nlambda >= 0,
                      NADIA_ERR_INVALID, "negative size");
        *bytes = nadia::footprint_bytes(kind, nx, ny, precision, n_best, nx + 2 * poly_pad_x,
                                        ny + 2 * poly_pad_y, nlambda);
    });
}

extern "C" long long nadia_device_bytes(void) { return nadia::g_device_bytes.load(); }

extern "C" int nadia_tuned_tiles(int nx, int ny, int fresnel, int batched, char *buf, int len)
{
    return guard([&] {
        need(buf, "buf");
        NADIA_REQUIRE(len > 0, NADIA_ERR_INVALID, "empty buffer");
        const char *mixed = getenv("NADIA_MIXED");
        if (batched && mixed && mixed[0] == '1' && nadia::f32::mix_variant(nx) &&
            nadia::f32::mix_variant(ny)) {
            // batched Planar/Fresnel grids of these lengths run with their classes' tiles
            const std::string t = "column pass: " + nadia::f32::mix_describe(nx) +
                                  "; row pass: " + nadia::f32::mix_describe(ny);
            snprintf(buf, (size_t)len, "%s", t.c_str());
            return;
        }
        const nadia::f32::Choice &c = nadia::f32::choose(nx, ny, fresnel != 0, batched ? 4 : 1);
        auto desc = [](const nadia::f32::TileVariant *v) {
            char t[160];
            snprintf(t, sizeof t, "n=%d threads=%d%s signals/tile=%d radices=%s%s%s", v->n, v->nt,
                     v->groups > 1 ? (v->groups == 4 ? " x4 groups" : " x2 groups") : "", v->L, v->radices,
                     v->single ? " persistent-TMA one stage"
                               : (v->persistent ? " persistent-TMA" : (v->ping ? " ping" : "")),
                     v->direct ? (v->ping && v->persistent ? " ping, sqrt(I) direct" : ", sqrt(I) direct") : "");
            return std::string(t);
        };
        char t[512];
        snprintf(t, sizeof t, "column pass: %s (%.1f us); row pass: %s (%.1f us)",
                 desc(c.col).c_str(), c.col_us, desc(c.row).c_str(), c.row_us);
        snprintf(buf, (size_t)len, "%s", t);
    });
}
