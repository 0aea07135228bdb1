// PhaseDiverseCDI.h -- drop-in for the reference's PhaseDiverseCDI
// (NADIA/include/PhaseDiverseCDI.h, NADIA/src/PhaseDiverseCDI.c++):
// phase-diverse / ptychographic reconstruction over several FresnelCDI (or
// other BaseCDI) frames, run on the GPU through nadia_pd_* (include/nadia_b200.h).
//
// Differences a caller can observe:
//   - frames keep their form (the float build's FP32 frames stay FP32, the
//     object is FP64); an FP32 PolyCDI frame moves to the FP64 form when added;
//   - get_transmission returns a copy of the object, refreshed by each call;
//     edits to it reach the reconstruction through set_transmission;
//   - frames must outlive this object (as in the reference), and the library
//     refuses to destroy a frame while it is part of one;
//   - failures throw nadia_cxx::Failure where the reference prints and exits.
#ifndef NADIA_DROPIN_PHASEDIVERSECDI_H
#define NADIA_DROPIN_PHASEDIVERSECDI_H

#include <iostream>
#include <memory>
#include <vector>

#include "BaseCDI.h"
#include "Complex_2D.h"

class PhaseDiverseCDI {
public:
    enum { CROSS_CORRELATION, MINIMUM_ERROR };

    // PhaseDiverseCDI(beta, gamma, parallel, granularity) -- PhaseDiverseCDI.c++:17-33
    PhaseDiverseCDI(double beta = 1.0, double gamma = 1.0, bool parallel = false,
                    int granularity = 1)
    {
        nadia_cxx::check(nadia_pd_create(beta, gamma, parallel ? 1 : 0, granularity, &h));
    }
    ~PhaseDiverseCDI()
    {
        if (h) nadia_pd_destroy(h);
    }
    PhaseDiverseCDI(const PhaseDiverseCDI &) = delete;
    PhaseDiverseCDI &operator=(const PhaseDiverseCDI &) = delete;

    // add_new_position -- PhaseDiverseCDI.c++:104-160
    void add_new_position(BaseCDI *local, double x = 0, double y = 0, double alpha = 1)
    {
        local->prepare_device();
        int rc = nadia_pd_add_position(h, local->handle(), x, y, alpha);
        if (rc == NADIA_ERR_UNSUPPORTED) { // an FP32 PolyCDI frame
            nadia_cxx::check(nadia_convert_to_fp64(local->handle()));
            rc = nadia_pd_add_position(h, local->handle(), x, y, alpha);
        }
        nadia_cxx::check(rc);
        frames.push_back(local);
        std::cout << "Added position " << frames.size() - 1 << std::endl;
    }

    // remove_positions -- PhaseDiverseCDI.c++:60-66
    void remove_positions()
    {
        nadia_cxx::check(nadia_pd_remove_positions(h));
        frames.clear();
    }

    // initialise_estimate -- PhaseDiverseCDI.c++:163-177
    void initialise_estimate()
    {
        before();
        nadia_cxx::check(nadia_pd_initialise_estimate(h));
        after();
    }

    // iterate -- PhaseDiverseCDI.c++:180-230, with its messages
    void iterate()
    {
        static int total_iterations = 0;
        std::cout << "Iteration " << total_iterations << std::endl;
        before();
        nadia_cxx::check(nadia_pd_iterate(h, 1));
        after();
        std::vector<double> err(iterations_per_cycle > 0 ? iterations_per_cycle : 1);
        for (size_t i = 0; i < frames.size(); ++i) {
            if (iterations_per_cycle <= 0) break;
            nadia_cxx::check(nadia_get_error_history(frames[i]->handle(), err.data(),
                                                     iterations_per_cycle));
            for (int j = 0; j < iterations_per_cycle; ++j)
                std::cout << "Error for frame " << i << " is " << err[j] << std::endl;
        }
        total_iterations++;
    }

    void set_iterations_per_cycle(int iterations)
    {
        nadia_cxx::check(nadia_pd_set_iterations_per_cycle(h, iterations));
        iterations_per_cycle = iterations;
    }
    void set_feedback_parameter(double beta)
    {
        nadia_cxx::check(nadia_pd_set_feedback_parameter(h, beta));
    }
    void set_amplification_factor(double gamma)
    {
        nadia_cxx::check(nadia_pd_set_amplification_factor(h, gamma));
    }
    void set_probe_scaling(int n_probe, double alpha)
    {
        if (nadia_pd_set_probe_scaling(h, n_probe, alpha) != NADIA_OK)
            std::cout << "In PhaseDiverseCDI::set_probe_scaling, "
                      << "the probe number given is too large. "
                      << "Are you trying to set the value of alpha "
                      << "before calling add_new_position?" << std::endl;
    }

    // get_transmission -- PhaseDiverseCDI.c++:77-79 (a copy, see above)
    Complex_2D *get_transmission()
    {
        int nx = 0, ny = 0;
        nadia_cxx::check(nadia_pd_get_size(h, &nx, &ny));
        if (nx == 0) return nullptr;
        std::vector<double> d((size_t)2 * nx * ny);
        nadia_cxx::check(nadia_pd_get_transmission(h, d.data()));
        if (!object || object->get_size_x() != nx || object->get_size_y() != ny)
            object.reset(new Complex_2D(nx, ny));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                object->set_real(i, j, d[2 * ((size_t)i * ny + j)]);
                object->set_imag(i, j, d[2 * ((size_t)i * ny + j) + 1]);
            }
        return object.get();
    }

    // set_transmission -- PhaseDiverseCDI.c++:81-101
    void set_transmission(Complex_2D &new_transmission)
    {
        const int nx = new_transmission.get_size_x(), ny = new_transmission.get_size_y();
        std::vector<double> d((size_t)2 * nx * ny);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                d[2 * ((size_t)i * ny + j)] = new_transmission.get_real(i, j);
                d[2 * ((size_t)i * ny + j) + 1] = new_transmission.get_imag(i, j);
            }
        if (nadia_pd_set_transmission(h, nx, ny, d.data()) != NADIA_OK)
            std::cout << "Can not set the transmission function in "
                      << "PhaseDiverseCDI because the complex array "
                      << "given does not have the same dimensions as "
                      << "the current transmission function" << std::endl;
    }

    // adjust_positions -- PhaseDiverseCDI.c++:232-392
    void adjust_positions(int type = CROSS_CORRELATION, bool forwards = true, int x_min = -50,
                          int x_max = +50, int y_min = -50, int y_max = +50,
                          double step_size = 4)
    {
        if (type != CROSS_CORRELATION && type != MINIMUM_ERROR) {
            std::cerr << "The alignment type given to"
                      << " PhaseDiverseCDI::adjust_positions is not"
                      << " a known type. Please consider using"
                      << " PhaseDiverseCDI::CROSS_CORRELATION or "
                      << " PhaseDiverseCDI::MINIMUM_ERROR." << std::endl;
            return;
        }
        before();
        nadia_cxx::check(nadia_pd_adjust_positions(h, type, forwards ? 1 : 0, x_min, x_max,
                                                   y_min, y_max, step_size));
        after();
    }

    double get_final_x_position(int n_probe) { return position(n_probe, true); }
    double get_final_y_position(int n_probe) { return position(n_probe, false); }

private:
    nadia_phase_diverse *h = nullptr;
    std::vector<BaseCDI *> frames;
    std::unique_ptr<Complex_2D> object;
    int iterations_per_cycle = 1;

    void before()
    {
        for (BaseCDI *f : frames) f->prepare_device();
    }
    void after()
    {
        for (BaseCDI *f : frames) f->estimate_changed_on_device();
    }
    double position(int n, bool x)
    {
        double px = 0, py = 0;
        nadia_cxx::check(nadia_pd_get_position(h, n, &px, &py));
        return x ? px : py;
    }
};

#endif
