// BaseCDI.h -- drop-in for the reference's BaseCDI (NADIA/include/BaseCDI.h):
// the same class, method names and signatures, running the reconstruction
// on the GPU through libnadia_b200 (include/nadia_b200.h).
//
// Differences a caller can observe:
//   - the float build (default) runs the fused FP32 form when the grid is one
//     of its sizes (256, 512, 768, 1024, 1536, 2048, 4096 per axis) and the
//     FP64 form otherwise; -DDOUBLE_PRECISION runs the FP64 form, which
//     reproduces the reference's double build;
//   - failures throw nadia_cxx::Failure where the reference prints and exits;
//   - propagate_to_detector / propagate_from_detector / scale_intensity /
//     apply_support / project_intensity on a caller's field run in FP64 and
//     are not available on FP32 reconstructions;
//   - set_algorithm, set_custom_algorithm, set_relaxation_parameter and
//     print_algorithm are virtual, so FresnelCDI_WF's versions (a warning:
//     its algorithm is fixed) answer calls through a BaseCDI pointer too;
//   - a TransmissionConstraint's per-pixel part (charge flipping, unit
//     magnitude) runs inside the FP32 form's fused passes, its
//     complex-constraint regions in the FP32 form's split row pass; custom
//     functions run in the FP64 form, to which an FP32 reconstruction moves
//     when it gets one (as does an FP32 PolyCDI given any constraint).  The constraint is read when iterate() or
//     apply_support() next runs (changes to it after that are picked up at
//     the following call).
#ifndef NADIA_DROPIN_BASECDI_H
#define NADIA_DROPIN_BASECDI_H

#include <iostream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "Complex_2D.h"
#include "Double_2D.h"
#include "TransmissionConstraint.h"
#include "types.h"

#define NALGORITHMS 9
#define NTERMS 5
#define NVECTORS 10
enum { PSF, PFS, PS, PF, PI };
enum { ER, BIO, BOO, HIO, DM, SF, ASR, HPR, RAAR, CUSTOM };

class BaseCDI {
public:
    virtual ~BaseCDI()
    {
        if (h) {
            complex.fetch(); // leave the final estimate in the caller's field
            complex.owner = nullptr;
            complex.device_newer = complex.host_newer = false;
            nadia_destroy(h);
        }
    }

    // BaseCDI::set_complex_constraint (BaseCDI.h:471-473)
    virtual void set_complex_constraint(TransmissionConstraint &trans_constraint)
    {
        transmission_constraint = &trans_constraint;
        trans_constraint.push_to(h, nx, ny, true);
    }

    // BaseCDI::iterate (BaseCDI.c++:297-387): one iteration on the GPU
    virtual int iterate()
    {
        if (transmission_constraint) transmission_constraint->push_to(h, nx, ny);
        complex.push();
        nadia_cxx::check(nadia_iterate(h, 1));
        complex.device_newer = true;
        return SUCCESS;
    }

    // several iterations without returning to the host in between
    int iterate(int n)
    {
        if (transmission_constraint) transmission_constraint->push_to(h, nx, ny);
        complex.push();
        nadia_cxx::check(nadia_iterate(h, n));
        complex.device_newer = true;
        return SUCCESS;
    }

    virtual void initialise_estimate(int seed = 0)
    {
        complex.host_newer = false;
        nadia_cxx::check(nadia_initialise_estimate(h, seed));
        complex.device_newer = true;
    }

    Complex_2D *get_best_result(double &error, int index = 0)
    {
        if (index < 0 || index >= n_best) {
            std::cout << "index out of bounds in BaseCDI::get_best_result" << std::endl;
            return nullptr;
        }
        std::vector<double> d((size_t)2 * nx * ny);
        nadia_cxx::check(nadia_get_best_result(h, index, &error, d.data()));
        while ((int)best.size() <= index) best.emplace_back(new Complex_2D(nx, ny));
        Complex_2D &b = *best[index];
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                b.set_real(i, j, d[2 * ((size_t)i * ny + j)]);
                b.set_imag(i, j, d[2 * ((size_t)i * ny + j) + 1]);
            }
        return &b;
    }

    void set_support(const Double_2D &object_support, bool soften = false)
    {
        std::vector<double> d = to_double(object_support);
        nadia_cxx::check(nadia_set_support(h, d.data(), soften ? 1 : 0));
    }
    void set_intensity(const Double_2D &detector_intensity)
    {
        std::vector<double> d = to_double(detector_intensity);
        nadia_cxx::check(nadia_set_intensity(h, d.data()));
    }
    void set_beam_stop(const Double_2D &beam_stop_region)
    {
        std::vector<double> d = to_double(beam_stop_region);
        nadia_cxx::check(nadia_set_beam_stop(h, d.data()));
    }
    virtual void set_relaxation_parameter(double relaxation_parameter)
    {
        nadia_cxx::check(nadia_set_relaxation_parameter(h, relaxation_parameter));
    }
    int get_size_x() { return nx; }
    int get_size_y() { return ny; }

    const Complex_2D &get_exit_surface_wave()
    {
        complex.fetch();
        return complex;
    }
    void set_exit_surface_wave(Complex_2D &esw)
    {
        complex.copy(esw);
        complex.push();
    }

    virtual void set_algorithm(int alg) { nadia_cxx::check(nadia_set_algorithm(h, alg)); }
    virtual void set_custom_algorithm(double m1, double m2, double m3, double m4, double m5, double m6,
                              double m7, double m8, double m9, double m10)
    {
        const double m[10] = {m1, m2, m3, m4, m5, m6, m7, m8, m9, m10};
        nadia_cxx::check(nadia_set_custom_algorithm(h, m));
    }
    virtual void print_algorithm()
    {
        double w[5];
        int alg = 0;
        nadia_cxx::check(nadia_get_algorithm_structure(h, w, &alg));
        if (alg == ER)
            std::cout << "Currently using error-reduction: x(k+1) = Ps Pf x(k)" << std::endl;
        else
            std::cout << "Currently using the algorithm: x(k+1) = x(k) + (" << w[PSF] << "*PsPf + "
                      << w[PFS] << "*PfPs + " << w[PS] << "*Ps + " << w[PF] << "*Pf + " << w[PI]
                      << "*I)x(k)" << std::endl;
        std::cout << "Ps - support constraint, Pf - modulus constraint" << std::endl;
    }

    double get_error()
    {
        double e = 0;
        nadia_cxx::check(nadia_get_error(h, &e));
        return e;
    }

    static int getAlgFromName(std::string name)
    {
        static const std::map<std::string, int> m = {{"ER", ER},   {"BIO", BIO}, {"BOO", BOO},
                                                     {"HIO", HIO}, {"DM", DM},   {"SF", SF},
                                                     {"ASR", ASR}, {"HPR", HPR}, {"RAAR", RAAR}};
        auto it = m.find(name);
        return it == m.end() ? -1 : it->second;
    }

    virtual void apply_shrinkwrap(double gauss_width = 1.5, double threshold = 0.1)
    {
        complex.push();
        nadia_cxx::check(nadia_apply_shrinkwrap(h, gauss_width, threshold));
    }

    const Double_2D &get_support()
    {
        std::vector<double> d((size_t)nx * ny);
        nadia_cxx::check(nadia_get_support(h, d.data()));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) support.set(i, j, d[(size_t)i * ny + j]);
        return support;
    }

    virtual void apply_support(Complex_2D &c) { op(c, nadia_apply_support); }
    virtual void project_intensity(Complex_2D &c) { op(c, nadia_project_intensity); }
    virtual void scale_intensity(Complex_2D &c) { op(c, nadia_scale_intensity); }
    virtual void propagate_to_detector(Complex_2D &c) { op(c, nadia_propagate_to_detector); }
    virtual void propagate_from_detector(Complex_2D &c) { op(c, nadia_propagate_from_detector); }

    void set_fftw_type(int) {}

    void reset_best() { nadia_cxx::check(nadia_reset_best(h)); }

    // the C handle, for calls that have no method here (batching, history)
    nadia_solver *handle() { return h; }

protected:
    friend class PhaseDiverseCDI;

    // hand pending host-side changes (edited estimate, constraint) to the GPU
    void prepare_device()
    {
        if (transmission_constraint) transmission_constraint->push_to(h, nx, ny);
        complex.push();
    }

    BaseCDI(Complex_2D &c, int n_best_)
        : complex(c), nx(c.get_size_x()), ny(c.get_size_y()), n_best(n_best_), support(nx, ny)
    {
    }

    // the estimate was replaced on the GPU; the caller's field fetches it on
    // its next access
    void estimate_changed_on_device()
    {
        complex.host_newer = false;
        complex.device_newer = true;
    }
    void upload_host_edits() { complex.push(); }

    // bind the caller's field to a freshly created handle
    void adopt(nadia_solver *handle)
    {
        h = handle;
        if (complex.owner)
            throw nadia_cxx::Failure(NADIA_ERR_STATE, "the field already belongs to a reconstruction");
        complex.owner = h;
        complex.host_newer = true; // upload the caller's starting field
        complex.device_newer = false;
        complex.push();
    }

    static int precision_for(int nx, int ny)
    {
#ifdef DOUBLE_PRECISION
        (void)nx;
        (void)ny;
        return NADIA_FP64;
#else
        auto ok = [](int n) {
            return n == 256 || n == 512 || n == 768 || n == 1024 || n == 1536 || n == 2048 ||
                   n == 4096;
        };
        return ok(nx) && ok(ny) ? NADIA_FP32 : NADIA_FP64;
#endif
    }

    template <class V>
    static std::vector<double> to_double(const V &d)
    {
        std::vector<double> out((size_t)d.get_size_x() * d.get_size_y());
        for (int i = 0; i < d.get_size_x(); ++i)
            for (int j = 0; j < d.get_size_y(); ++j) out[(size_t)i * d.get_size_y() + j] = d.get(i, j);
        return out;
    }

    void op(Complex_2D &c, int (*f)(nadia_solver *, double *))
    {
        std::vector<double> d((size_t)2 * nx * ny);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                d[2 * ((size_t)i * ny + j)] = c.get_real(i, j);
                d[2 * ((size_t)i * ny + j) + 1] = c.get_imag(i, j);
            }
        nadia_cxx::check(f(h, d.data()));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                c.set_real(i, j, d[2 * ((size_t)i * ny + j)]);
                c.set_imag(i, j, d[2 * ((size_t)i * ny + j) + 1]);
            }
    }

    Complex_2D &complex;
    int nx, ny;
    int n_best;
    TransmissionConstraint *transmission_constraint = nullptr;
    nadia_solver *h = nullptr;
    Double_2D support;
    std::vector<std::unique_ptr<Complex_2D>> best;
};

#endif
