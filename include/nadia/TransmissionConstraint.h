// TransmissionConstraint.h -- drop-in for the reference's ComplexConstraint and
// TransmissionConstraint (NADIA/include/TransmissionConstraint.h): the
// constraint object a caller builds and hands to set_complex_constraint.  The
// reconstruction applies it on the GPU (FP32 or FP64 form) after every support
// projection; apply_constraint here is the same operation on the host for
// callers that apply it to a field of their own.
#ifndef NADIA_DROPIN_TRANSMISSIONCONSTRAINT_H
#define NADIA_DROPIN_TRANSMISSIONCONSTRAINT_H

#include <cmath>
#include <cstdint>
#include <iostream>
#include <vector>

#include "Complex_2D.h"
#include "Double_2D.h"

// ComplexConstraint (TransmissionConstraint.h:27-130): a region whose
// magnitude and phase are coupled through c_mean
class ComplexConstraint {
protected:
    double alpha1, alpha2;
    Double_2D *region;
    double c_mean = 0;
    bool fixed_c = false;

public:
    ComplexConstraint(Double_2D &region_, double alpha1_, double alpha2_)
        : alpha1(alpha1_), alpha2(alpha2_), region(&region_)
    {
    }
    void set_fixed_c(double c)
    {
        fixed_c = true;
        c_mean = c;
    }
    void set_c_mean(double c)
    {
        if (!fixed_c) c_mean = c;
    }
    double get_c_mean() { return c_mean; }
    bool is_c_fixed() const { return fixed_c; }
    void set_alpha1(double a) { alpha1 = a; }
    void set_alpha2(double a) { alpha2 = a; }
    double get_alpha1() const { return alpha1; }
    double get_alpha2() const { return alpha2; }
    double get_new_mag(double old_mag, double old_phase)
    {
        return exp((1 - alpha1) * log(old_mag) + alpha1 * c_mean * old_phase);
    }
    double get_new_phase(double old_mag, double old_phase)
    {
        return (1 - alpha2) * old_phase + alpha2 * log(old_mag) / c_mean;
    }
    Double_2D *get_region() { return region; }
};

// TransmissionConstraint (TransmissionConstraint.h:200-375)
class TransmissionConstraint {
protected:
    std::vector<ComplexConstraint *> complex_constraint_list;
    bool do_enforce_unity = true;
    bool do_charge_flip = true;
    int flip_sign = 1;
    void (*custom_constraint)(Complex_2D &) = nullptr;

public:
    TransmissionConstraint() {}
    virtual ~TransmissionConstraint() {}

    void delete_complex_constraint_regions()
    {
        while (!complex_constraint_list.empty()) {
            delete complex_constraint_list.back();
            complex_constraint_list.pop_back();
        }
    }
    virtual void add_complex_constraint(ComplexConstraint &c) { complex_constraint_list.push_back(&c); }
    void set_charge_flipping(bool enable, int sign = 1)
    {
        do_charge_flip = enable;
        flip_sign = sign > 0 ? 1 : -1;
    }
    void set_enforce_unity(bool enable) { do_enforce_unity = enable; }
    void set_custom_constraint(void (*f)(Complex_2D &transmission)) { custom_constraint = f; }

    // TransmissionConstraint::apply_constraint (TransmissionConstraint.c++:76-172)
    virtual void apply_constraint(Complex_2D &t)
    {
        const int nx = t.get_size_x(), ny = t.get_size_y();
        std::vector<int> map = region_map(nx, ny);
        const int R = (int)complex_constraint_list.size();
        if (R > 0) {
            std::vector<double> lnA(R, 0.0), ph(R, 0.0);
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j) {
                    const int r = map[(size_t)i * ny + j];
                    if (r > 0) {
                        ph[r - 1] += fabs(t.get_phase(i, j));
                        lnA[r - 1] += fabs(log(t.get_mag(i, j)));
                    }
                }
            for (int r = 0; r < R; ++r) complex_constraint_list[r]->set_c_mean(lnA[r] / ph[r]);
        }
        if (R > 0 || do_charge_flip || do_enforce_unity)
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j) {
                    const double phase_old = t.get_phase(i, j);
                    double mag_old = t.get_mag(i, j);
                    const int r = map[(size_t)i * ny + j];
                    if (r > 0) {
                        ComplexConstraint *c = complex_constraint_list[r - 1];
                        const double mag_new = c->get_new_mag(mag_old, phase_old);
                        const double phase_new = c->get_new_phase(mag_old, phase_old);
                        t.set_mag(i, j, mag_new);
                        t.set_phase(i, j, phase_new);
                        mag_old = mag_new;
                    }
                    if (do_charge_flip && flip_sign * t.get_imag(i, j) > 0)
                        t.set_imag(i, j, -1 * t.get_imag(i, j));
                    if (do_enforce_unity && mag_old > 1) t.set_mag(i, j, 1);
                }
        if (custom_constraint) (*custom_constraint)(t);
    }

    // hand the constraint to a reconstruction of the C ABI (again only when
    // a setting, a region object or the custom function changed since the
    // last hand-over to the same reconstruction; set force after a region's
    // mask was edited in place)
    void push_to(nadia_solver *h, int nx, int ny, bool force = false)
    {
        const int R = (int)complex_constraint_list.size();
        std::vector<double> sig = {(double)do_enforce_unity, (double)do_charge_flip,
                                   (double)flip_sign, (double)R,
                                   (double)(uintptr_t)custom_constraint, (double)(uintptr_t)h};
        for (ComplexConstraint *c : complex_constraint_list) {
            sig.push_back((double)(uintptr_t)c->get_region());
            sig.push_back(c->get_alpha1());
            sig.push_back(c->get_alpha2());
            sig.push_back(c->is_c_fixed() ? c->get_c_mean() : -1.0);
            sig.push_back((double)c->is_c_fixed());
        }
        if (!force && sig == pushed_) return;
        pushed_ = sig;
        std::vector<double> regions((size_t)R * nx * ny), alpha(2 * (size_t)R), fixed(R);
        for (int r = 0; r < R; ++r) {
            ComplexConstraint *c = complex_constraint_list[r];
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j)
                    regions[((size_t)r * nx + i) * ny + j] = c->get_region()->get(i, j);
            alpha[2 * r] = c->get_alpha1();
            alpha[2 * r + 1] = c->get_alpha2();
            fixed[r] = c->is_c_fixed() ? c->get_c_mean() : NAN;
        }
        // custom functions run in the FP64 form (the per-pixel part and the
        // regions also run in the FP32 form)
        if (custom_constraint) nadia_cxx::check(nadia_convert_to_fp64(h));
        int rc = nadia_set_transmission_constraint(
            h, do_enforce_unity, do_charge_flip, flip_sign, R, R ? regions.data() : nullptr,
            R ? alpha.data() : nullptr, R ? fixed.data() : nullptr);
        if (rc == NADIA_ERR_UNSUPPORTED) { // e.g. an FP32 PolyCDI
            nadia_cxx::check(nadia_convert_to_fp64(h));
            rc = nadia_set_transmission_constraint(
                h, do_enforce_unity, do_charge_flip, flip_sign, R, R ? regions.data() : nullptr,
                R ? alpha.data() : nullptr, R ? fixed.data() : nullptr);
        }
        nadia_cxx::check(rc);
        nadia_cxx::check(nadia_set_transmission_custom(h, custom_constraint ? &trampoline : nullptr,
                                                       this));
    }

private:
    std::vector<double> pushed_; // what was last handed over

    // a pixel belongs to the first region that claims it (TransmissionConstraint.c++:20-73)
    std::vector<int> region_map(int nx, int ny)
    {
        std::vector<int> map((size_t)nx * ny, 0);
        for (size_t r = 0; r < complex_constraint_list.size(); ++r) {
            Double_2D *reg = complex_constraint_list[r]->get_region();
            for (int i = 0; i < nx; ++i)
                for (int j = 0; j < ny; ++j)
                    if (reg->get(i, j) > 0 && map[(size_t)i * ny + j] == 0)
                        map[(size_t)i * ny + j] = (int)r + 1;
        }
        return map;
    }

    static void trampoline(double *t, int nx, int ny, void *user)
    {
        TransmissionConstraint *self = static_cast<TransmissionConstraint *>(user);
        Complex_2D c(nx, ny);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                c.set_real(i, j, t[2 * ((size_t)i * ny + j)]);
                c.set_imag(i, j, t[2 * ((size_t)i * ny + j) + 1]);
            }
        (*self->custom_constraint)(c);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                t[2 * ((size_t)i * ny + j)] = c.get_real(i, j);
                t[2 * ((size_t)i * ny + j) + 1] = c.get_imag(i, j);
            }
    }
};

#endif
