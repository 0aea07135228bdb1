// CDI_reconstruction -- the reconstruction tool of the reference
// (NADIA/tools/CDI_reconstruction.c) on the GPU drop-in classes.
//
//   CDI_reconstruction <config file> [planar|fresnel|fresnel_wf|poly] [seed]
//
// The configuration keys, the files read and written, their names and
// formats, and the order of the steps are those of the reference tool
// (CDI_reconstruction.c:94-410): the algorithm / iterations lists run in
// turn, a magnitude image is written every output_iterations iterations,
// shrink-wrap runs after iteration i when i % shrinkwrap_iterations ==
// shrinkwrap_iterations - 1, the final estimate goes to
// <output_file_name_prefix>.cplx (fresnel_wf: white_field_reco_file_name)
// and, for fresnel, the transmission function to transmission_function.cplx.
// A starting_point_file_name (.cplx) replaces initialise_estimate, which
// makes a run restartable from any .cplx it wrote.
//
// The iterations between two of those events run as one call of
// BaseCDI::iterate(n): the estimate stays on the GPU and is read back only
// for the images and the final files.  info_level 2 (print the error of
// every iteration) runs them one by one.
//
// Built twice: the float build (fused FP32 form on its grid sizes, FP64
// otherwise) and -DDOUBLE_PRECISION (FP64 form, the reference's double build).
// partial and partchar (PartialCDI, PartialCharCDI) are not part of this
// library; asking for them prints so and exits 1.  The diffraction image of
// output_diffraction_estimate is named <prefix>_diffraction_<i>.<type>; the
// reference appends that name to the magnitude image's name.  An
// output_iterations of 0 writes no images (the reference divides by it).
#include <cstdlib>
#include <iostream>
#include <list>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "BaseCDI.h"
#include "Complex_2D.h"
#include "Config.h"
#include "Double_2D.h"
#include "FresnelCDI.h"
#include "FresnelCDI_WF.h"
#include "PlanarCDI.h"
#include "PolyCDI.h"
#include "io.h"

namespace {

enum { OUTPUT_MINIMAL = 0, OUTPUT_ITER = 1, OUTPUT_ERROR = 2 };

const char *const kTypes[] = {"planar", "fresnel", "fresnel_wf", "partial", "partchar", "poly"};

void usage()
{
    std::cout << "Usage: " << std::endl
              << std::endl
              << "CDI_reconstruction <config filename> <reco_type> <seed>" << std::endl
              << std::endl
              << "where <reco_type> may be: planar, fresnel, fresnel_wf, partial, partchar or poly"
              << std::endl
              << "<seed> should be an integer" << std::endl
              << std::endl
              << "<reco_type> and <seed> do not need to be specified: "
              << "<reco_type> defaults to planar and <seed> to 0." << std::endl;
}

// one entry of the algorithm / iterations lists
struct Stage {
    std::string algorithm;
    int iterations;
};

struct Run {
    int pixels_x = 0, pixels_y = 0;
    int output_iterations = 0;
    int output_level = OUTPUT_MINIMAL;
    bool output_diffraction = false, log_diffraction = false, log_object = false;
    int shrinkwrap_iterations = 0;
    double shrinkwrap_gauss_width = 0, shrinkwrap_threshold = 0;
    std::string output_file_type, starting_point, data_file, support_file, prefix, output_file;
    std::vector<Stage> stages;
};

std::string image_name(const Run &r, const char *what, int i)
{
    std::ostringstream s;
    s << r.prefix << what << i << "." << r.output_file_type;
    return s.str();
}

// the last iteration of the run of iterations starting at i that ends at an
// event: a stage boundary, an image, a shrink-wrap or a printed error
int chunk_end(const Run &r, int i, int stage_end)
{
    if (r.output_level == OUTPUT_ERROR) return i;
    int e = stage_end - 1;
    if (r.output_iterations != 0) {
        const int k = std::abs(r.output_iterations);
        const int next = (i % k == 0) ? i : i + (k - i % k);
        if (next < e) e = next;
    }
    if (r.shrinkwrap_iterations > 0) {
        const int k = r.shrinkwrap_iterations;
        const int next = i + (k - 1 - i % k);
        if (next < e) e = next;
    }
    return e;
}

int reconstruct(int argc, char *argv[])
{
    if (argc == 1) {
        std::cout << std::endl << "No config file given, ";
        usage();
        return 0;
    }
    const std::string config_file = argv[1];
    std::string reco_type = "planar";
    int seed = 0;
    if (argc <= 2)
        std::cout << "No reconstruction type given... using planar" << std::endl;
    else
        reco_type = argv[2];
    if (argc <= 3)
        std::cout << "No seed value given... using the default (0)" << std::endl;
    else
        seed = std::atoi(argv[3]);
    if (argc > 4) {
        std::cout << std::endl << "Wrong number of arguments given. ";
        usage();
        return 0;
    }

    Config c(config_file);
    if (c.getStatus() == FAILURE) {
        std::cout << "Could not open the file " << config_file << ". Exiting" << std::endl;
        return 0;
    }

    Run r;
    r.output_iterations = (int)c.getDouble("output_iterations");
    std::unique_ptr<std::list<std::string>> algorithms(c.getStringList("algorithm"));
    std::unique_ptr<std::list<int>> iterations(c.getIntList("iterations"));
    r.pixels_x = c.getInt("pixels_x");
    r.pixels_y = c.getInt("pixels_y");
    if (c.getStatus() == FAILURE) {
        std::cout << "Problem reading the configuration file. Exiting" << std::endl;
        return 0;
    }
    if (algorithms->size() != iterations->size()) {
        std::cout << "The number of algorithms and the number "
                  << "of iterations do not match. Exiting" << std::endl;
        return 0;
    }
    {
        auto it = iterations->begin();
        for (const std::string &a : *algorithms) r.stages.push_back({a, *it++});
    }

    // optional keys (0 / "" when absent, as in the reference)
    r.output_level = c.getInt("info_level");
    r.output_diffraction = c.getInt("output_diffraction_estimate") != 0;
    r.log_diffraction = c.getInt("use_log_scale_for_diffraction") != 0;
    r.log_object = c.getInt("use_log_scale_for_object") != 0;
    r.shrinkwrap_iterations = c.getInt("shrinkwrap_iterations");
    r.shrinkwrap_gauss_width = c.getDouble("shrinkwrap_gauss_width");
    r.shrinkwrap_threshold = c.getDouble("shrinkwrap_threshold");
    r.output_file_type = c.getString("output_file_type");

    Complex_2D object_estimate(r.pixels_x, r.pixels_y);
    r.starting_point = c.getString("starting_point_file_name");
    if (!r.starting_point.empty() && !read_cplx(r.starting_point, object_estimate)) {
        std::cout << "Can not process the file " << r.starting_point << ".. exiting" << std::endl;
        return 1;
    }

    r.data_file = c.getString("data_file_name");
    r.support_file = c.getString("support_file_name");
    r.prefix = c.getString("output_file_name_prefix");
    r.output_file = r.prefix + ".cplx";

    std::unique_ptr<Complex_2D> white_field;
    std::unique_ptr<BaseCDI> proj;
    if (reco_type == "planar") {
        proj.reset(new PlanarCDI(object_estimate));
    } else if (reco_type == "fresnel") {
        const double wavelength = c.getDouble("beam_wavelength");
        const double focal_detector = c.getDouble("focal_detector_length");
        const double focal_sample = c.getDouble("focal_sample_length");
        const double pixel = c.getDouble("pixel_size");
        const double normalisation = c.getDouble("normalisation");
        white_field.reset(new Complex_2D(r.pixels_x, r.pixels_y));
        if (!read_cplx(c.getString("white_field_reco_file_name"), *white_field)) {
            std::cout << "failed to read white-field data .. exiting" << std::endl;
            return 1;
        }
        std::cout << white_field->get_value(0, 0, MAG_SQ) << std::endl;
        proj.reset(new FresnelCDI(object_estimate, *white_field, wavelength, focal_detector,
                                  focal_sample, pixel, normalisation));
    } else if (reco_type == "fresnel_wf") {
        const double wavelength = c.getDouble("beam_wavelength");
        const double zone_focal = c.getDouble("zone_focal_length");
        const double focal_detector = c.getDouble("focal_detector_length");
        const double pixel = c.getDouble("pixel_size");
        proj.reset(new FresnelCDI_WF(object_estimate, wavelength, zone_focal, focal_detector, pixel));
        // the white-field recovery has its own files, a fixed algorithm and
        // no shrink-wrap
        r.output_file = c.getString("white_field_reco_file_name");
        r.data_file = c.getString("white_field_data_file_name");
        r.support_file = c.getString("white_field_support_file_name");
        r.stages = {{"ER", c.getInt("wf_iterations")}};
        r.shrinkwrap_iterations = 0;
    } else if (reco_type == "poly") {
        const std::string spectrum = c.getString("spectrum_file_name");
        PolyCDI *p = new PolyCDI(object_estimate);
        proj.reset(p);
        p->set_spectrum(spectrum);
    } else if (reco_type == "partial" || reco_type == "partchar") {
        std::cout << "the reconstruction type " << reco_type
                  << " (partially coherent illumination) is not part of this library" << std::endl;
        return 1;
    } else {
        std::cout << "the reconstruction type specified (" << reco_type << ") is "
                  << "unrecognised. Please use: ";
        for (int k = 0; k < 6; ++k) std::cout << kTypes[k] << (k < 4 ? ", " : k < 5 ? ", or " : "");
        std::cout << std::endl;
        return 1;
    }

    Double_2D data;
    read_image(r.data_file, data, r.pixels_x, r.pixels_y);
    if (r.pixels_x != data.get_size_x() || r.pixels_y != data.get_size_y()) {
        std::cout << "Dimensions of the data to not match those given ... exiting" << std::endl;
        return 1;
    }
    Double_2D support;
    read_image(r.support_file, support, r.pixels_x, r.pixels_y);
    if (r.pixels_x != support.get_size_x() || r.pixels_y != support.get_size_y()) {
        std::cout << "Dimensions of the support to not match ... exiting" << std::endl;
        return 1;
    }
    proj->set_support(support);
    proj->set_intensity(data);
    if (r.starting_point.empty()) proj->initialise_estimate(seed);

    Double_2D result(r.pixels_x, r.pixels_y);
    int i = 0;
    for (const Stage &st : r.stages) {
        if (r.output_level != OUTPUT_MINIMAL)
            std::cout << "Switching to the " << st.algorithm << " algorithm" << std::endl;
        const int alg = BaseCDI::getAlgFromName(st.algorithm);
        if (alg == -1) {
            std::cout << "Could not find reconstruction algorithm with the name " << st.algorithm
                      << ". Exiting" << std::endl;
            return 0;
        }
        proj->set_algorithm(alg);
        const int stage_end = i + st.iterations;
        while (i < stage_end) {
            const int e = chunk_end(r, i, stage_end);
            if (r.output_level != OUTPUT_MINIMAL)
                for (int k = i; k <= e; ++k) std::cout << "Iteration " << k << std::endl;
            proj->iterate(e - i + 1);
            i = e;
            if (r.output_level == OUTPUT_ERROR && i > 0)
                std::cout << "Error for iteration " << (i - 1) << " is " << proj->get_error()
                          << std::endl;
            if (r.output_iterations != 0 && i % r.output_iterations == 0) {
                object_estimate.get_2d(MAG, result);
                write_image(image_name(r, "_", i), result, r.log_object);
                if (r.output_diffraction) {
                    std::unique_ptr<Complex_2D> temp(object_estimate.clone());
                    proj->propagate_to_detector(*temp);
                    temp->get_2d(MAG_SQ, result);
                    write_image(image_name(r, "_diffraction_", i), result, r.log_diffraction);
                }
            }
            if (r.shrinkwrap_iterations != 0 &&
                i % r.shrinkwrap_iterations == r.shrinkwrap_iterations - 1) {
                proj->apply_shrinkwrap(r.shrinkwrap_gauss_width, r.shrinkwrap_threshold);
                std::cout << "Applying shrink-wrap at iteration " << i << std::endl;
            }
            ++i;
        }
    }

    write_cplx(r.output_file, object_estimate);
    if (reco_type == "fresnel") {
        static_cast<FresnelCDI *>(proj.get())->get_transmission_function(object_estimate);
        write_cplx("transmission_function.cplx", object_estimate);
    }
    return 0;
}

} // namespace

int main(int argc, char *argv[])
{
    try {
        return reconstruct(argc, argv);
    } catch (const nadia_cxx::Failure &e) {
        std::cout << e.what() << ". Exiting now.." << std::endl;
        return 1;
    }
}
