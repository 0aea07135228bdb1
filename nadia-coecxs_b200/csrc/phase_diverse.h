// phase_diverse.h -- PhaseDiverseCDI (NADIA/include/PhaseDiverseCDI.h,
// NADIA/src/PhaseDiverseCDI.c++) on the GPU: several reconstructions
// ("frames", FP64 Solvers) placed at (x, y) on one global object.  The object,
// every frame's last result and the blending weights live on the device; the
// blending (add_to_object), the read-back into a frame (update_from_object),
// the parallel-mode rescale and the position search's image work are kernels
// (phase_diverse.cu, compiled with --fmad=false, one IEEE operation sequence
// per pixel as the reference's double build).  Frame work runs on the frame's
// own stream and the object work on this object's stream, joined by events,
// so in parallel mode the frames iterate concurrently.  The weights
// (set_up_weights) are computed on the host in the reference's order from
// each frame's support and illumination and uploaded when they change.
#pragma once

#include <vector>

#include "solver.h"

namespace nadia {

struct PhaseDiverse {
    enum { CROSS_CORRELATION = 0, MINIMUM_ERROR = 1 };

    // declared first: destroyed after every buffer below, whose releases are
    // ordered on this stream
    int device = 0;
    OwnedStream own_st;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;

    double beta, gamma;
    bool parallel;
    int scale;
    int iterations_per_cycle = 1;
    bool weights_set = false;

    // frames since the last remove_positions (singleCDI); the per-position
    // vectors below keep every position ever added, indexed as in the
    // reference (remove_positions clears the frames only)
    std::vector<Solver *> frames;
    std::vector<double> xpos, ypos, alpha;
    std::vector<int> rnx, rny;
    std::vector<DevBuf<double2>> result; // single_result
    std::vector<DevBuf<double>> weight;  // weights
    // alpha * (|illumination| / max)^gamma, 0 outside the support: the part
    // of each weight that needs the host's pow, kept until its inputs change
    struct Base {
        const Solver *frame = nullptr;
        unsigned long long version = ~0ull;
        double gamma = 0, alpha = 0;
        std::vector<double> h;
        DevBuf<double> d;
    };
    std::vector<Base> base;

    // the current object: the owned global one, or a temporary during the
    // position search (adjust_positions swaps it as the reference does)
    DevBuf<double2> object_buf;
    double2 *obj = nullptr;
    int nx = 0, ny = 0, x_min = 0, y_min = 0;

    DevBuf<unsigned long long> d_count;
    DevBuf<double> d_best;      // argmax partials: (ratio, index) pairs
    DevBuf<char> d_frames;      // frame table of scale_object

    PhaseDiverse(double beta, double gamma, bool parallel, int granularity);
    ~PhaseDiverse();

    void add_position(Solver *frame, double x, double y, double alpha);
    void remove_positions();
    void initialise_estimate();
    void iterate();
    void set_feedback_parameter(double b);
    void set_amplification_factor(double g);
    bool set_probe_scaling(int n, double a);
    void get_transmission(double *h);
    void set_transmission(int nx, int ny, const double *h);
    void adjust_positions(int type, bool forward, int min_x, int max_x, int min_y, int max_y,
                          double step_size);
    // wait for everything this object queued (on its stream and the frames')
    void sync();

private:
    void join(cudaStream_t from, cudaStream_t to);
    void to_frame(int n) { join(st, frames[n]->st); }
    void to_object(int n) { join(frames[n]->st, st); }
    void rejoin_frames();
    void realloc_object(int nx, int ny);
    void set_up_weights();
    void get_result(int n, double2 *dst);
    void set_result(int n, const double2 *src);
    void add_to_object(int n);
    void update_from_object(int n);
    void scale_object(double factor);
    bool check_position(int n, double step, int min_x, int max_x, int min_y, int max_y,
                        int tries);
    void align(const double *first, int nx1, int ny1, const double *second, int nx2, int ny2,
               int &offset_x, int &offset_y, int min_x, int max_x, int min_y, int max_y,
               const double *first_w, const double *second_w, double overlap_fraction);
};

} // namespace nadia
