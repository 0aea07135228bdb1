// A caller written against the reference's C++ classes (PlanarCDI,
// FresnelCDI, PolyCDI, Complex_2D, Double_2D), compiled unchanged against the
// drop-in headers in include/nadia.  It runs the same call sequences as
// tests/scenarios.py (planar_mixed, fresnel_mixed, poly_mixed) plus the flow of
// the reference's PlanarCDI example (ER/HIO/ER cycles with shrinkwrap, the
// estimate read back every 10 iterations), reading inputs from and writing
// results to raw little-endian float64 files in a directory.
//
//   cdi_program <planar|fresnel|poly|example|wf|tc|pd> <nx> <ny> <dir> [padding]
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include <Complex_2D.h>
#include <Double_2D.h>
#include <FresnelCDI.h>
#include <FresnelCDI_WF.h>
#include <PhaseDiverseCDI.h>
#include <PlanarCDI.h>
#include <PolyCDI.h>

static std::string dir;

static std::vector<double> load(const std::string &name, size_t n)
{
    std::vector<double> v(n);
    std::ifstream f(dir + "/" + name, std::ios::binary);
    if (!f.read((char *)v.data(), n * sizeof(double))) {
        std::cerr << "cannot read " << name << std::endl;
        std::exit(2);
    }
    return v;
}

static void save(const std::string &name, const std::vector<double> &v)
{
    std::ofstream f(dir + "/" + name, std::ios::binary);
    f.write((const char *)v.data(), v.size() * sizeof(double));
}

static Double_2D real_2d(const std::string &name, int nx, int ny)
{
    std::vector<double> v = load(name, (size_t)nx * ny);
    Double_2D d(nx, ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) d.set(i, j, v[(size_t)i * ny + j]);
    return d;
}

static void complex_2d(const std::string &name, Complex_2D &c)
{
    int nx = c.get_size_x(), ny = c.get_size_y();
    std::vector<double> v = load(name, (size_t)2 * nx * ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            c.set_real(i, j, v[2 * ((size_t)i * ny + j)]);
            c.set_imag(i, j, v[2 * ((size_t)i * ny + j) + 1]);
        }
}

static void save_complex(const std::string &name, const Complex_2D &c)
{
    int nx = c.get_size_x(), ny = c.get_size_y();
    std::vector<double> v((size_t)2 * nx * ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            v[2 * ((size_t)i * ny + j)] = c.get_real(i, j);
            v[2 * ((size_t)i * ny + j) + 1] = c.get_imag(i, j);
        }
    save(name, v);
}

static void save_real(const std::string &name, const Double_2D &d)
{
    int nx = d.get_size_x(), ny = d.get_size_y();
    std::vector<double> v((size_t)nx * ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) v[(size_t)i * ny + j] = d.get(i, j);
    save(name, v);
}

static int planar(int nx, int ny)
{
    Complex_2D object_estimate(nx, ny);
    PlanarCDI planar(object_estimate, 2);
    planar.set_support(real_2d("support.bin", nx, ny));
    planar.set_intensity(real_2d("intensity.bin", nx, ny));
    planar.set_beam_stop(real_2d("beam_stop.bin", nx, ny));
    planar.initialise_estimate(3);
    save_complex("init.bin", object_estimate);
    std::vector<double> errs;
    for (int i = 0; i < 3; ++i) {
        planar.iterate();
        errs.push_back(planar.get_error());
    }
    planar.set_relaxation_parameter(0.7);
    planar.set_algorithm(HIO);
    for (int it = 0; it < 24; ++it) {
        planar.iterate();
        errs.push_back(planar.get_error());
        if (it % 8 == 7) planar.apply_shrinkwrap(1.5, 0.1);
    }
    planar.set_relaxation_parameter(0.8);
    planar.set_algorithm(RAAR);
    for (int i = 0; i < 10; ++i) {
        planar.iterate();
        errs.push_back(planar.get_error());
    }
    planar.set_algorithm(ER);
    for (int i = 0; i < 6; ++i) {
        planar.iterate();
        errs.push_back(planar.get_error());
    }
    save("errors.bin", errs);
    save_complex("esw.bin", object_estimate);
    save_real("support_out.bin", planar.get_support());
    double best_err = 0;
    Complex_2D *best = planar.get_best_result(best_err, 1);
    save_complex("best.bin", *best);
    save("best_err.bin", std::vector<double>(1, best_err));
    if (planar.get_best_result(best_err, 2) != NULL) return 3;
    return 0;
}

static int fresnel(int nx, int ny)
{
    std::vector<double> p = load("params.bin", 4);
    Complex_2D white_field(nx, ny);
    complex_2d("white_field.bin", white_field);
    Complex_2D object_estimate(nx, ny);
    FresnelCDI proj(object_estimate, white_field, p[0], p[1], p[2], p[3], 0.97);
    proj.set_support(real_2d("support.bin", nx, ny));
    proj.set_intensity(real_2d("intensity.bin", nx, ny));
    proj.auto_set_norm();
    proj.initialise_estimate(2);
    save_complex("init.bin", object_estimate);
    save_complex("illum.bin", proj.get_illumination_at_sample());
    std::vector<double> errs;
    for (int i = 0; i < 8; ++i) {
        proj.iterate();
        errs.push_back(proj.get_error());
    }
    proj.set_algorithm(HIO);
    for (int it = 0; it < 12; ++it) {
        proj.iterate();
        errs.push_back(proj.get_error());
        if (it == 6) proj.apply_shrinkwrap(2, 0.1);
    }
    save("errors.bin", errs);
    save_complex("esw.bin", object_estimate);
    Complex_2D trans(nx, ny);
    proj.get_transmission_function(trans);
    save_complex("transmission.bin", trans);
    // the host form of the same formula, on a copy of the estimate
    Complex_2D esw_copy(object_estimate);
    Complex_2D trans_host(nx, ny);
    proj.get_transmission_function(trans_host, &esw_copy);
    save_complex("transmission_host.bin", trans_host);
    save_real("support_out.bin", proj.get_support());
    return 0;
}

static int poly(int nx, int ny, int padding)
{
    (void)padding;
    std::vector<double> nl = load("spectrum_n.bin", 1);
    int nlambda = (int)nl[0];
    Double_2D spectrum = real_2d("spectrum.bin", nlambda, 2);
    Complex_2D object_estimate(nx, ny);
    PolyCDI poly(object_estimate, 0.9, 1);
    poly.set_support(real_2d("support.bin", nx, ny));
    poly.set_intensity(real_2d("intensity.bin", nx, ny));
    poly.set_spectrum(spectrum);
    poly.initialise_estimate(7);
    std::vector<double> errs;
    for (int i = 0; i < 3; ++i) {
        poly.iterate();
        errs.push_back(poly.get_error());
    }
    poly.set_algorithm(HIO);
    for (int it = 0; it < 8; ++it) {
        poly.iterate();
        errs.push_back(poly.get_error());
        if (it == 4) poly.apply_shrinkwrap(1.5, 0.1);
    }
    save("errors.bin", errs);
    save_complex("esw.bin", object_estimate);
    save_real("support_out.bin", poly.get_support());
    return 0;
}

// PlanarCDI with a TransmissionConstraint: tests/scenarios.py's
// planar_constrained with ER only
static int constrained(int nx, int ny)
{
    Complex_2D object_estimate(nx, ny);
    PlanarCDI planar(object_estimate);
    planar.set_support(real_2d("support.bin", nx, ny));
    planar.set_intensity(real_2d("intensity.bin", nx, ny));
    std::vector<double> p = load("tc_params.bin", 9); // (alpha1, alpha2, fixed c or NaN) x 3
    Double_2D r0 = real_2d("region0.bin", nx, ny), r1 = real_2d("region1.bin", nx, ny),
              r2 = real_2d("region2.bin", nx, ny);
    ComplexConstraint c0(r0, p[0], p[1]), c1(r1, p[3], p[4]), c2(r2, p[6], p[7]);
    if (p[5] == p[5]) c1.set_fixed_c(p[5]);
    TransmissionConstraint tc;
    tc.set_enforce_unity(true);
    tc.set_charge_flipping(true, -1);
    tc.add_complex_constraint(c0);
    tc.add_complex_constraint(c1);
    tc.add_complex_constraint(c2);
    planar.set_complex_constraint(tc);
    planar.initialise_estimate(3);
    std::vector<double> errs;
    for (int it = 0; it < 12; ++it) {
        planar.iterate();
        errs.push_back(planar.get_error());
    }
    save("errors.bin", errs);
    save_complex("esw.bin", object_estimate);
    return 0;
}

// FresnelCDI_WF: the sequence of tests/scenarios.py's fresnel_wf_mixed
static int white_field(int nx, int ny)
{
    std::vector<double> p = load("params.bin", 5);
    Complex_2D wf(nx, ny);
    FresnelCDI_WF proj(wf, p[0], p[1], p[2], p[3]);
    proj.set_support(p[4]);
    proj.set_intensity(real_2d("intensity.bin", nx, ny));
    proj.initialise_estimate(0);
    save_complex("init.bin", wf);
    save_real("support0.bin", proj.get_support());
    proj.set_algorithm(HIO); // prints the reference's warning and changes nothing
    std::vector<double> errs;
    const int iterations = 12;
    for (int it = 0; it < iterations; ++it) {
        proj.iterate();
        errs.push_back(proj.get_error());
        if (it == iterations / 2) proj.apply_shrinkwrap(1.5, 0.1);
    }
    save("errors.bin", errs);
    save_complex("esw.bin", wf);
    save_real("support_out.bin", proj.get_support());
    return 0;
}

// PhaseDiverseCDI over three FresnelCDI frames (tests/scenarios.py
// phase_diverse_mixed with adjust="cc"): params.bin holds wavelength,
// focus-to-detector, pixel, then per frame focus-to-sample, x, y, dx, dy
static int phase_diverse(int nx, int ny)
{
    const int frames = 3;
    std::vector<double> p = load("params.bin", 3 + 5 * frames);
    Double_2D support = real_2d("support.bin", nx, ny);
    std::vector<Complex_2D *> esw;
    std::vector<FresnelCDI *> proj;
    PhaseDiverseCDI pd(1.0, 1.0, false, 1);
    for (int k = 0; k < frames; ++k) {
        esw.push_back(new Complex_2D(nx, ny));
        Complex_2D wf(nx, ny);
        complex_2d("white_field" + std::to_string(k) + ".bin", wf);
        const double *f = &p[3 + 5 * k];
        proj.push_back(new FresnelCDI(*esw.back(), wf, p[0], p[1], f[0], p[2], 1.0));
        proj.back()->set_support(support);
        proj.back()->set_intensity(real_2d("intensity" + std::to_string(k) + ".bin", nx, ny));
        proj.back()->initialise_estimate(k + 1);
    }
    for (int k = 0; k < frames; ++k) {
        const double *f = &p[3 + 5 * k];
        pd.add_new_position(proj[k], f[1] + f[3], f[2] + f[4]);
    }
    pd.set_iterations_per_cycle(2);
    pd.initialise_estimate();
    pd.adjust_positions(PhaseDiverseCDI::CROSS_CORRELATION, true, -6, 6, -6, 6);
    for (int c = 0; c < 3; ++c) pd.iterate();
    save_complex("object.bin", *pd.get_transmission());
    std::vector<double> pos;
    for (int k = 0; k < frames; ++k) {
        pos.push_back(pd.get_final_x_position(k));
        pos.push_back(pd.get_final_y_position(k));
        save_complex("frame" + std::to_string(k) + ".bin", *esw[k]);
    }
    save("positions.bin", pos);
    return 0;
}

// the flow of the reference's PlanarCDI example, two short cycles
static int example(int nx, int ny)
{
    Double_2D data = real_2d("intensity.bin", nx, ny);
    Double_2D support = real_2d("support.bin", nx, ny);
    Complex_2D object_estimate(nx, ny);
    PlanarCDI planar(object_estimate, 4);
    planar.set_support(support);
    planar.set_intensity(data);
    planar.initialise_estimate(0);
    Double_2D result(nx, ny);
    object_estimate.get_2d(MAG, result);
    std::vector<double> errs, mags;
    planar.set_algorithm(ER);
    const int er1 = 10, hio = 20, er2 = 10, out_every = 10, shrink = 10;
    for (int a = 0; a < 2; ++a) {
        for (int i = 0; i < er1; ++i) {
            planar.iterate();
            errs.push_back(planar.get_error());
            if (i % out_every == 0) {
                object_estimate.get_2d(MAG, result);
                mags.push_back(result.get_sum());
            }
            if (i % shrink == shrink - 1) planar.apply_shrinkwrap(1.5, 0.1);
        }
        planar.set_relaxation_parameter(0.5);
        planar.set_algorithm(HIO);
        for (int i = er1; i < er1 + hio; ++i) {
            planar.iterate();
            errs.push_back(planar.get_error());
            if (i % out_every == 0) {
                object_estimate.get_2d(MAG, result);
                mags.push_back(result.get_sum());
            }
            if (i % shrink == shrink - 1) planar.apply_shrinkwrap(2.0, 0.1);
        }
        planar.set_algorithm(ER);
        for (int i = er1 + hio; i < er1 + hio + er2; ++i) {
            planar.iterate();
            errs.push_back(planar.get_error());
            if (i % shrink == shrink - 1) planar.apply_shrinkwrap(2.0, 0.1);
        }
    }
    save("errors.bin", errs);
    save("mags.bin", mags);
    save_complex("esw.bin", object_estimate);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 5) {
        std::cerr << "usage: cdi_program <planar|fresnel|poly|example> nx ny dir [padding]" << std::endl;
        return 1;
    }
    std::string mode = argv[1];
    int nx = std::atoi(argv[2]), ny = std::atoi(argv[3]);
    dir = argv[4];
    try {
        if (mode == "planar") return planar(nx, ny);
        if (mode == "fresnel") return fresnel(nx, ny);
        if (mode == "poly") return poly(nx, ny, argc > 5 ? std::atoi(argv[5]) : 0);
        if (mode == "example") return example(nx, ny);
        if (mode == "wf") return white_field(nx, ny);
        if (mode == "tc") return constrained(nx, ny);
        if (mode == "pd") return phase_diverse(nx, ny);
    } catch (const nadia_cxx::Failure &e) {
        std::cerr << "failure " << e.code << ": " << e.what() << std::endl;
        return 4;
    }
    std::cerr << "unknown mode " << mode << std::endl;
    return 1;
}
