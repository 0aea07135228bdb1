// server.cu -- the request loop (server.h) and the admission charge of one
// reconstruction.
//
// Admission is in arrival order: a request waits while the slot limit or
// the HBM budget would be exceeded, and later ones wait behind it.  Admitted
// requests are prepared by host worker threads (device buffers, inputs,
// initial estimate, each on the reconstruction's own stream) and handed to
// the stepping thread, which steps every active reconstruction together with
// iterate_many for the same number of iterations: the chunk size, shortened
// so that no request passes its next shrinkwrap or its last iteration.
// Finished requests go back to the worker threads, which copy them out and
// release their device memory, freeing their slot and budget for the next
// admission; arrivals therefore
// overlap with the work of the requests already on the GPU.
//
// Every request is stepped only through iterate_many, whose tile choice does
// not depend on the other members of a batch, so a request's result is the
// same whether it ran alone or among others.
#include "server.h"

#include <algorithm>
#include <cstring>

#include "batch.h"
#include "fused32.h"
#include "fused32_impl.h"

namespace nadia {

size_t footprint_bytes(int kind, int nx, int ny, int prec, int n_best, int pad_nx, int pad_ny,
                       int nlambda)
{
    const size_t n = (size_t)nx * ny;
    // error value, error history, reduction scratch, maxima (solver.cu)
    size_t b = 8 + 8 * (size_t)Solver::kRing + 8 * (2 * (size_t)plain::kRedBlocks + 64) + 16;
    if (prec == NADIA_FP64) {
        b += n * (16 + 8 + 8 + 8 + 8); // x, support, sqrt(I), blur result, scratch
        if (kind != NADIA_FRESNEL_WF) b += 4 * 16 * n; // the combine's projection terms at most
        b += 8 * n;                    // beam stop
        b += 16 * (size_t)(nx + ny);   // transform twiddles
        if ((nx | ny) & 1) b += 16 * n; // odd grids: the quadrant swap's gather target
        b += 8 * 64;                   // blur kernel table
        b += (size_t)n_best * 16 * n;
        if (kind == NADIA_FRESNEL) b += 16 * n + 16 * n + 16 * (size_t)(nx / 2) * (ny / 2);
        if (kind == NADIA_FRESNEL_WF) b += 16 * (size_t)(nx / 2) * (ny / 2);
        if (kind == NADIA_POLY)
            b += 16 * (size_t)nlambda + 16 * (size_t)pad_nx * pad_ny + 8 * n +
                 16 * (size_t)(pad_nx + pad_ny);
    } else {
        b += n * (8 + 8 + 4 + 4);                     // P, x, support, sqrt(I)
        // partials (one per column tile; FresnelCDI_WF one per row tile),
        // counter, flag, slot pointer
        b += 8 * (size_t)(kind == NADIA_FRESNEL_WF ? std::max(nx, ny / 2) : ny / 2) + 8 + 4 + 2 * 8;
        b += sizeof(f32::Slot);
        const size_t tiles = ((size_t)(nx + 31) / 32) * ((ny + 31) / 32);
        b += 2 * 4 * n + 4 * (std::max<size_t>(tiles, 592) + 2); // shrinkwrap scratch
        b += (size_t)n_best * 8 * n;
        if (kind == NADIA_FRESNEL) b += 8 * n + 8 * n + 8 * (size_t)(nx + ny);
        if (kind == NADIA_FRESNEL_WF) b += 8 * (size_t)(nx + ny); // per-axis zone-plate factors
        if (kind == NADIA_POLY) {
            const size_t m = (size_t)pad_nx * pad_ny;
            b += 8 * m + 4 * m;                                  // padded work array, |Psi|^2
            b += 4 * (size_t)nlambda * (nx + ny + 1);            // gather tables, weights
            b += 8 * 1184 + 4 * n;                               // error partials, ratio
        }
    }
    return b;
}

namespace {

constexpr int kPreparers = 8; // host worker threads (prepare and read back requests)

// PolyCDI's padding from its spectrum (PolyCDI.c++:66-89)
void poly_padding(const double *sp, int nl, int nx, int ny, int *px, int *py)
{
    double maxweight = 0, lc = 0;
    for (int i = 0; i < nl; i++)
        if (sp[2 * i + 1] > maxweight) {
            lc = sp[2 * i];
            maxweight = sp[2 * i + 1];
        }
    NADIA_REQUIRE(maxweight > 0, NADIA_ERR_INVALID, "spectrum has no positive weight");
    *px = (int)((sp[0] / lc - 1.0) * nx / 2);
    *py = (int)((sp[0] / lc - 1.0) * ny / 2);
    NADIA_REQUIRE(*px >= 0 && *py >= 0, NADIA_ERR_INVALID,
                  "negative padding: list the longest wavelength first");
}

std::vector<double> copy_of(const double *p, size_t n)
{
    return p ? std::vector<double>(p, p + n) : std::vector<double>();
}

} // namespace

Server::Server(size_t budget_bytes, int max_active, int chunk)
    : budget_(budget_bytes), max_active_(max_active), chunk_(chunk)
{
    NADIA_REQUIRE(max_active >= 1, NADIA_ERR_INVALID, "max_active must be at least 1");
    NADIA_REQUIRE(chunk >= 1, NADIA_ERR_INVALID, "chunk must be at least 1");
    NADIA_CUDA(cudaGetDevice(&device_));
    t0_ = std::chrono::steady_clock::now();
    const int np = std::max(1, std::min(kPreparers, max_active));
    worker_ = std::thread([this] { run(); });
    for (int i = 0; i < np; ++i) preparers_.emplace_back([this] { prepare_loop(); });
}

Server::~Server()
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_admit_.notify_all();
    cv_ready_.notify_all();
    for (auto &t : preparers_)
        if (t.joinable()) t.join();
    if (worker_.joinable()) worker_.join();
    // what never reached the stepping thread or its readback
    std::vector<Record *> left;
    {
        std::lock_guard<std::mutex> lk(mu_);
        left.assign(ready_.begin(), ready_.end());
        left.insert(left.end(), done_.begin(), done_.end());
        ready_.clear();
        done_.clear();
    }
    for (Record *r : left) fail(*r, NADIA_ERR_STATE, "the server stopped");
}

double Server::now() const
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
}

long long Server::submit(const nadia_request &q)
{
    NADIA_REQUIRE(q.kind >= NADIA_PLANAR && q.kind <= NADIA_POLY, NADIA_ERR_INVALID,
                  "unknown kind");
    NADIA_REQUIRE(q.precision == NADIA_FP32 || q.precision == NADIA_FP64, NADIA_ERR_INVALID,
                  "unknown precision");
    NADIA_REQUIRE(q.nx >= 2 && q.ny >= 2, NADIA_ERR_INVALID, "grid too small");
    NADIA_REQUIRE(q.intensity && q.support, NADIA_ERR_INVALID,
                  "a request needs an intensity and a support");
    NADIA_REQUIRE(q.iterations >= 0 && q.shrinkwrap_every >= 0, NADIA_ERR_INVALID,
                  "negative iteration count");
    NADIA_REQUIRE(q.kind != NADIA_POLY || (q.spectrum && q.nlambda >= 1), NADIA_ERR_INVALID,
                  "a PolyCDI request needs a spectrum");
    NADIA_REQUIRE(q.kind != NADIA_FRESNEL || q.white_field, NADIA_ERR_INVALID,
                  "a FresnelCDI request needs a white field");
    std::unique_ptr<Record> r(new Record);
    const size_t n = (size_t)q.nx * q.ny;
    r->req = q;
    r->intensity = copy_of(q.intensity, n);
    r->support = copy_of(q.support, n);
    r->beam_stop = copy_of(q.beam_stop, n);
    r->spectrum = copy_of(q.kind == NADIA_POLY ? q.spectrum : nullptr, 2 * (size_t)q.nlambda);
    r->white_field = copy_of(q.kind == NADIA_FRESNEL ? q.white_field : nullptr, 2 * n);
    int px = 0, py = 0;
    if (q.kind == NADIA_POLY) poly_padding(r->spectrum.data(), q.nlambda, q.nx, q.ny, &px, &py);
    r->bytes = footprint_bytes(q.kind, q.nx, q.ny, q.precision, 0, q.nx + 2 * px, q.ny + 2 * py,
                               q.nlambda);
    NADIA_REQUIRE(r->bytes <= budget_, NADIA_ERR_NOMEM,
                  "the request needs more device memory than the whole budget");
    long long id;
    {
        std::lock_guard<std::mutex> lk(mu_);
        NADIA_REQUIRE(!stop_, NADIA_ERR_STATE, "the server is stopping");
        id = next_id_++;
        r->id = id;
        r->t_arrive = now();
        queue_.push_back(r.get());
        records_[id] = std::move(r);
    }
    cv_admit_.notify_all();
    return id;
}

bool Server::wait(long long id, double timeout_s)
{
    std::unique_lock<std::mutex> lk(mu_);
    auto it = records_.find(id);
    NADIA_REQUIRE(it != records_.end(), NADIA_ERR_INVALID, "unknown request id");
    Record *r = it->second.get();
    auto done = [&] { return r->state == DONE || r->state == FAILED; };
    if (timeout_s < 0) {
        cv_done_.wait(lk, done);
        return true;
    }
    return cv_done_.wait_for(lk, std::chrono::duration<double>(timeout_s), done);
}

void Server::result(long long id, double *esw, double *support, double *final_error,
                    double times[3])
{
    std::unique_ptr<Record> r;
    {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = records_.find(id);
        NADIA_REQUIRE(it != records_.end(), NADIA_ERR_INVALID, "unknown request id");
        NADIA_REQUIRE(it->second->state == DONE || it->second->state == FAILED, NADIA_ERR_STATE,
                      "the request has not finished");
        r = std::move(it->second);
        records_.erase(it);
    }
    if (times) {
        times[0] = r->t_admit - r->t_arrive;
        times[1] = r->t_done - r->t_admit;
        times[2] = r->t_done - r->t_arrive;
    }
    if (r->state == FAILED) throw Error(r->code, r->message);
    if (esw) std::memcpy(esw, r->esw.data(), r->esw.size() * sizeof(double));
    if (support) std::memcpy(support, r->sup_out.data(), r->sup_out.size() * sizeof(double));
    if (final_error) *final_error = r->final_error;
}

void Server::stats(long long out[12])
{
    std::lock_guard<std::mutex> lk(mu_);
    out[8] = us_step_;
    out[9] = us_idle_;
    out[10] = us_prepare_;
    out[11] = us_readback_;
    out[0] = (long long)queue_.size();
    out[1] = slots_;
    out[2] = completed_;
    out[3] = failed_;
    out[4] = (long long)bytes_in_use_;
    out[5] = (long long)peak_bytes_;
    out[6] = steps_;
    out[7] = admitted_;
}

// iterations until the request's next shrinkwrap or its end
int Server::next_event(const Record &r) const
{
    int d = r.req.iterations - r.done_iters;
    const int k = r.req.shrinkwrap_every;
    if (k > 0) d = std::min(d, k - r.done_iters % k);
    return d;
}

void Server::start(Record &r)
{
    const nadia_request &q = r.req;
    r.solver.reset(new Solver(q.kind, q.nx, q.ny, q.precision, 0));
    Solver &s = *r.solver;
    AllocScope scope(s.st);
    if (q.kind == NADIA_FRESNEL)
        s.fresnel_init(r.white_field.data(), q.wavelength, q.focal_detector_length,
                       q.focal_sample_length, q.pixel_size, q.normalisation);
    s.set_support(r.support.data(), false);
    s.set_intensity(r.intensity.data());
    if (!r.beam_stop.empty()) s.set_beam_stop(r.beam_stop.data());
    if (q.kind == NADIA_POLY) s.set_spectrum(r.spectrum.data(), q.nlambda);
    if (q.kind == NADIA_FRESNEL && q.fresnel_auto_norm) s.fresnel_auto_set_norm();
    s.initialise_estimate(q.seed);
    // BaseCDI::set_relaxation_parameter takes effect at the next algorithm
    // change (BaseCDI.h:264-267); the handle starts as ER
    s.set_relaxation_parameter(q.beta);
    s.set_algorithm(q.algorithm);
    // the inputs are on the device; the host copies are no longer needed
    std::vector<double>().swap(r.intensity);
    std::vector<double>().swap(r.beam_stop);
    std::vector<double>().swap(r.white_field);
}

void Server::finish(Record &r)
{
    Solver &s = *r.solver;
    AllocScope scope(s.st);
    r.final_error = s.get_error();
    r.esw.resize(2 * s.n);
    s.get_esw(r.esw.data());
    r.sup_out.resize(s.n);
    s.get_support(r.sup_out.data());
    r.solver.reset();
    {
        std::lock_guard<std::mutex> lk(mu_);
        bytes_in_use_ -= r.bytes;
        --slots_;
        r.t_done = now();
        r.state = DONE;
        ++completed_;
    }
    cv_admit_.notify_all();
}

void Server::fail(Record &r, int code, const std::string &msg)
{
    r.solver.reset();
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (r.state == ACTIVE) {
            bytes_in_use_ -= r.bytes;
            --slots_;
        }
        r.code = code;
        r.message = msg;
        r.t_done = now();
        if (r.t_admit == 0) r.t_admit = r.t_done;
        r.state = FAILED;
        ++failed_;
    }
    cv_admit_.notify_all();
    cv_done_.notify_all();
}

bool Server::can_admit() const
{
    return !queue_.empty() && slots_ < max_active_ &&
           bytes_in_use_ + queue_.front()->bytes <= budget_;
}

// worker thread: read back a finished request, or admit the next request
// that fits, build it and hand it to the stepping thread
void Server::prepare_loop()
{
    cudaSetDevice(device_);
    for (;;) {
        Record *r = nullptr;
        bool readback = false;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_admit_.wait(lk, [&] { return stop_ || !done_.empty() || can_admit(); });
            if (stop_) return;
            if (!done_.empty()) { // finishing first: it frees a slot and budget
                r = done_.front();
                done_.pop_front();
                readback = true;
            }
        }
        if (readback) {
            const double t0 = now();
            try {
                finish(*r);
            } catch (const Error &e) {
                fail(*r, e.code, e.what());
            } catch (const std::exception &e) {
                fail(*r, NADIA_ERR_CUDA, e.what());
            }
            {
                std::lock_guard<std::mutex> lk(mu_);
                us_readback_ += (long long)(1e6 * (now() - t0));
            }
            cv_done_.notify_all();
            continue;
        }
        {
            std::unique_lock<std::mutex> lk(mu_);
            if (stop_) return;
            if (!can_admit()) continue;
            r = queue_.front();
            queue_.pop_front();
            bytes_in_use_ += r->bytes;
            peak_bytes_ = std::max(peak_bytes_, bytes_in_use_);
            ++slots_;
            r->state = ACTIVE;
            r->t_admit = now();
            ++admitted_;
        }
        cv_admit_.notify_all(); // another worker may admit the next one
        const double t0 = now();
        try {
            start(*r);
        } catch (const Error &e) {
            fail(*r, e.code, e.what());
            continue;
        } catch (const std::exception &e) {
            fail(*r, NADIA_ERR_CUDA, e.what());
            continue;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            us_prepare_ += (long long)(1e6 * (now() - t0));
            ready_.push_back(r);
        }
        cv_ready_.notify_all();
    }
}

// stepping thread
void Server::run()
{
    cudaSetDevice(device_);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(mu_);
            const double t0 = now();
            if (active_.empty()) cv_ready_.wait(lk, [&] { return stop_ || !ready_.empty(); });
            us_idle_ += (long long)(1e6 * (now() - t0));
            if (stop_) break;
            active_.insert(active_.end(), ready_.begin(), ready_.end());
            ready_.clear();
        }
        if (active_.empty()) continue;

        int c = chunk_;
        std::vector<Solver *> handles;
        for (Record *r : active_) {
            c = std::min(c, next_event(*r));
            handles.push_back(r->solver.get());
        }
        std::vector<Record *> keep;
        const double t0 = now();
        try {
            Range range("nadia_server_step");
            if (c > 0) iterate_many(handles.data(), (int)handles.size(), c);
            for (Record *r : active_) {
                r->done_iters += c;
                const int k = r->req.shrinkwrap_every;
                if (k > 0 && r->done_iters % k == 0 && c > 0)
                    r->solver->apply_shrinkwrap(r->req.shrinkwrap_sigma, r->req.shrinkwrap_threshold);
            }
            // finished requests go to the worker threads for their readback
            // (which waits for their streams) while this thread steps the rest
            std::vector<Record *> finished;
            for (Record *r : active_)
                (r->done_iters >= r->req.iterations ? finished : keep).push_back(r);
            {
                std::lock_guard<std::mutex> lk(mu_);
                ++steps_;
                us_step_ += (long long)(1e6 * (now() - t0));
                done_.insert(done_.end(), finished.begin(), finished.end());
            }
            if (!finished.empty()) cv_admit_.notify_all();
        } catch (const Error &e) {
            // a failure inside a shared step fails every request in it
            for (Record *r : active_)
                if (r->state == ACTIVE) fail(*r, e.code, e.what());
            keep.clear();
        } catch (const std::exception &e) {
            for (Record *r : active_)
                if (r->state == ACTIVE) fail(*r, NADIA_ERR_CUDA, e.what());
            keep.clear();
        }
        active_.swap(keep);
        cv_done_.notify_all();
    }
    // stopping: release what is still on the device, fail what is queued
    for (Record *r : active_) fail(*r, NADIA_ERR_STATE, "the server stopped");
    active_.clear();
    std::vector<Record *> left;
    {
        std::lock_guard<std::mutex> lk(mu_);
        left.assign(queue_.begin(), queue_.end());
        queue_.clear();
    }
    for (Record *r : left) fail(*r, NADIA_ERR_STATE, "the server stopped");
}

} // namespace nadia
