// server.h -- a request loop over many reconstructions on one GPU:
// diffraction patterns arrive at any time, are admitted while an HBM budget
// and a slot limit allow, keep their estimate, support and intensity resident
// on the device, and step together (iterate_many) until each has run its
// iterations; results wait on the host until collected.  A few host worker
// threads build admitted reconstructions (device buffers, inputs, initial
// estimate) and read finished ones back, while one stepping thread keeps the
// GPU busy with the others.
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "solver.h"

namespace nadia {

// Device bytes a reconstruction holds once all of its lazily made buffers
// exist (the admission charge).  pad_nx/pad_ny: PolyCDI's padded grid.
size_t footprint_bytes(int kind, int nx, int ny, int prec, int n_best, int pad_nx, int pad_ny,
                       int nlambda);

class Server {
public:
    Server(size_t budget_bytes, int max_active, int chunk);
    ~Server();

    long long submit(const nadia_request &r);
    // true when the request has finished (or failed) within timeout_s
    bool wait(long long id, double timeout_s);
    // copies the result out and forgets the request; throws the request's
    // own error if it failed
    void result(long long id, double *esw, double *support, double *final_error,
                double times[3]);
    void stats(long long out[12]);

private:
    enum State { QUEUED, ACTIVE, DONE, FAILED };
    struct Record {
        long long id = 0;
        nadia_request req{};
        std::vector<double> intensity, support, beam_stop, spectrum, white_field;
        size_t bytes = 0;
        std::unique_ptr<Solver> solver;
        int done_iters = 0;
        State state = QUEUED;
        int code = NADIA_OK;
        std::string message;
        std::vector<double> esw, sup_out;
        double final_error = 0;
        double t_arrive = 0, t_admit = 0, t_done = 0;
    };

    void run();
    void prepare_loop();
    bool can_admit() const;
    void start(Record &r);
    void finish(Record &r);
    void fail(Record &r, int code, const std::string &msg);
    int next_event(const Record &r) const;
    double now() const;

    int device_ = 0;
    size_t budget_;
    int max_active_, chunk_;
    std::chrono::steady_clock::time_point t0_;

    std::mutex mu_;
    std::condition_variable cv_admit_, cv_ready_, cv_done_;
    std::deque<Record *> queue_;                           // submitted, not admitted
    std::vector<Record *> ready_;                          // admitted and prepared
    std::deque<Record *> done_;    // iterations queued, waiting for their readback
    std::map<long long, std::unique_ptr<Record>> records_;
    std::vector<Record *> active_; // stepped; touched by the stepping thread only
    int slots_ = 0;                // admitted and not yet finished
    size_t bytes_in_use_ = 0, peak_bytes_ = 0;
    long long next_id_ = 1, completed_ = 0, failed_ = 0, steps_ = 0, admitted_ = 0;
    // host microseconds: stepping thread stepping / waiting for work; worker
    // threads preparing / reading back
    long long us_step_ = 0, us_idle_ = 0, us_prepare_ = 0, us_readback_ = 0;
    bool stop_ = false;
    std::thread worker_;
    std::vector<std::thread> preparers_;
};

} // namespace nadia
