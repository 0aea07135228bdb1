// batch.cu -- several reconstructions stepped together (nadia_iterate_many).
//
// FP32 handles are grouped by grid size and geometry.  Each group runs one
// launch per pass for all of its members (gridDim.y = members), the groups
// run concurrently on forked streams, and a whole block of iterations is
// captured once as a CUDA graph and replayed.  Handles the fused form cannot
// batch (FP64, PolyCDI, n-best bookkeeping, algorithms with a PfPs term) are
// stepped one by one on their own streams.
#include <algorithm>
#include <cstdlib>
#include <atomic>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "batch.h"
#include "fused32.h"
#include "fused32_impl.h"
#include "solver.h"

namespace nadia {

std::atomic<long long> g_launches{0};

namespace {

constexpr int kGraphIters = 16;
constexpr int kBatchClass = 4; // tuner class of batched groups (fused32.cu: choose)
constexpr size_t kMaxPlans = 8;

struct Group {
    int nx = 0, ny = 0;
    bool fresnel = false;
    const f32::Choice *choice = nullptr;
    // PolyCDI groups (same grid and padding): the padded-grid passes
    const f32::PolyVariant *pcol = nullptr, *prow = nullptr;
    int pcols = 0, rtiles = 0;
    int launches_per_iter() const { return pcol ? 4 : 2; }
    std::vector<Solver *> members;
    DevBuf<f32::Slot *> ptrs;
    const float2 *twx = nullptr, *twy = nullptr;
    cudaStream_t st = nullptr; // side stream (null for the first group)
};

// The members of several grid sizes whose lengths all have a mixed-length
// class: one column launch per kind (PlanarCDI, FresnelCDI) and one row
// launch per iteration for all of them, whatever their sizes.
struct MixList {
    DevBuf<f32::MixItem> items;
    DevBuf<int> bounds;
    int ctas = 0;
};
struct Mixed {
    std::vector<Solver *> members;
    DevBuf<f32::Slot *> ptrs;
    MixList col[2], row; // col[1]: FresnelCDI members
    bool empty() const { return members.empty(); }
    void launch(cudaStream_t s) const
    {
        for (int k = 0; k < 2; ++k)
            f32::mix_launch_col(k == 1, col[k].items.p, col[k].bounds.p, col[k].ctas, ptrs.p, s);
        f32::mix_launch_row(row.items.p, row.bounds.p, row.ctas, ptrs.p, (int)members.size(), s);
    }
    int launches() const { return (col[0].ctas > 0) + (col[1].ctas > 0) + (row.ctas > 0); }
};

struct Plan {
    std::vector<unsigned long long> key;
    Mixed mixed;
    std::vector<Group> groups;
    cudaStream_t st = nullptr;               // batch stream (first member's)
    std::vector<cudaEvent_t> fork, join;     // per side stream
    cudaGraphExec_t exec = nullptr;
    ~Plan()
    {
        if (exec) cudaGraphExecDestroy(exec);
        for (auto &g : groups)
            if (g.st) cudaStreamDestroy(g.st);
        // group 0 runs on the batch stream and has no events of its own;
        // destroying a null event would leave an error for the next check
        for (auto e : fork)
            if (e) cudaEventDestroy(e);
        for (auto e : join)
            if (e) cudaEventDestroy(e);
    }

    void launch_block(int iters)
    {
        // fork side streams off the batch stream
        for (size_t i = 0; i < groups.size(); ++i) {
            if (!groups[i].st) continue;
            NADIA_CUDA(cudaEventRecord(fork[i], st));
            NADIA_CUDA(cudaStreamWaitEvent(groups[i].st, fork[i], 0));
        }
        for (int it = 0; it < iters; ++it) mixed.launch(st);
        for (auto &g : groups) {
            cudaStream_t s = g.st ? g.st : st;
            const int n = (int)g.members.size();
            for (int it = 0; it < iters; ++it) {
                if (g.pcol) {
                    g.pcol->col_fwd(g.ptrs.p, n, g.pcols, s, g.twx);
                    g.pcol->col_inv(g.ptrs.p, n, g.pcols, s, g.twx);
                    g.prow->row(f32::kRowFull, g.ptrs.p, n, g.rtiles, s, g.twy);
                } else {
                    g.choice->col->col(g.fresnel, g.ptrs.p, n, g.nx, g.ny, g.twx, s);
                    g.choice->row->row(f32::kRowFull, g.ptrs.p, n, g.nx, g.ny, g.twy, s);
                }
            }
        }
        for (size_t i = 0; i < groups.size(); ++i) {
            if (!groups[i].st) continue;
            NADIA_CUDA(cudaEventRecord(join[i], groups[i].st));
            NADIA_CUDA(cudaStreamWaitEvent(st, join[i], 0));
        }
    }

    long long launches_per_iter() const
    {
        long long l = mixed.launches();
        for (const auto &g : groups) l += g.launches_per_iter();
        return l;
    }
};

std::mutex g_mu;
std::list<std::unique_ptr<Plan>> g_plans; // most recently used first

bool batchable(const Solver &s)
{
    return s.prec == NADIA_FP32 && s.n_best == 0 && !s.tc.active && s.kind != NADIA_FRESNEL_WF &&
           (s.kind != NADIA_POLY || s.f32->impl->pcol != nullptr) &&
           (s.algorithm == NADIA_ER || s.w[PFS] == 0);
}

// With NADIA_MIXED=1 in the environment when a batch is first stepped,
// Planar/Fresnel reconstructions whose column length (nx) and row length (ny)
// both have a mixed-length class run with their class's tile configuration,
// alone or not: in the mixed passes when the call holds several such sizes,
// in that configuration's single-length passes otherwise; either way the
// same arithmetic, so a reconstruction's result never depends on the other
// handles of a call.  Otherwise (the default: faster on B200) every size
// group runs the batched tuner choice for its grid, the same alone or not.
bool mixable(const Solver &s)
{
    const char *env = getenv("NADIA_MIXED");
    if (!(env && env[0] == '1')) return false;
    return s.kind != NADIA_POLY && f32::mix_variant(s.nx) && f32::mix_variant(s.ny);
}

void upload_list(MixList &l, std::vector<f32::MixItem> &items, cudaStream_t st)
{
    if (items.empty()) return;
    std::vector<int> bounds;
    l.ctas = std::min<int>(f32::mix_ctas(), (int)items.size());
    f32::mix_order(items, bounds, l.ctas);
    l.items.alloc(items.size());
    l.bounds.alloc(bounds.size());
    NADIA_CUDA(cudaMemcpyAsync(l.items.p, items.data(), items.size() * sizeof(f32::MixItem),
                               cudaMemcpyHostToDevice, st));
    NADIA_CUDA(cudaMemcpyAsync(l.bounds.p, bounds.data(), bounds.size() * sizeof(int),
                               cudaMemcpyHostToDevice, st));
    // the host vectors are pageable: finish the copies before they go
    NADIA_CUDA(cudaStreamSynchronize(st));
}

// the work lists: every column tile (by kind) and every row tile of every
// member, ordered by class and cut into per-CTA ranges
void build_mixed(Mixed &m, cudaStream_t st)
{
    std::vector<f32::MixItem> col[2], row;
    std::vector<f32::Slot *> hp;
    for (size_t k = 0; k < m.members.size(); ++k) {
        Solver *s = m.members[k];
        const int cc = f32::mix_class_of(s->nx), rc = f32::mix_class_of(s->ny);
        const int ct = s->ny / f32::mix_tile(cc), rt = s->nx / f32::mix_tile(rc);
        auto &cl = col[s->kind == NADIA_FRESNEL ? 1 : 0];
        for (int t = 0; t < ct; ++t) cl.push_back({(int)k, t, cc, 0});
        for (int t = 0; t < rt; ++t) row.push_back({(int)k, t, rc, 0});
        hp.push_back(s->f32->impl->slot.p);
    }
    m.ptrs.alloc(hp.size());
    NADIA_CUDA(cudaMemcpyAsync(m.ptrs.p, hp.data(), hp.size() * sizeof(f32::Slot *),
                               cudaMemcpyHostToDevice, st));
    for (int k = 0; k < 2; ++k) upload_list(m.col[k], col[k], st);
    upload_list(m.row, row, st);
}

// the fixed choice of a mixable grid: its classes' single-length variants
const f32::Choice &class_choice(int nx, int ny)
{
    static std::mutex mu;
    static std::map<std::pair<int, int>, f32::Choice> cache;
    std::lock_guard<std::mutex> lock(mu);
    f32::Choice &c = cache[{nx, ny}];
    if (!c.col) {
        c.col = f32::mix_variant(nx);
        c.row = f32::mix_variant(ny);
        c.col->prepare();
        c.row->prepare();
    }
    return c;
}
} // namespace

void iterate_many(Solver *const *solvers, int count, int iterations)
{
    NADIA_REQUIRE(count >= 0 && iterations >= 0, NADIA_ERR_INVALID, "negative count");
    std::vector<Solver *> fused, other;
    for (int i = 0; i < count; ++i) {
        NADIA_REQUIRE(solvers[i] != nullptr, NADIA_ERR_INVALID, "null handle in batch");
        for (int j = 0; j < i; ++j)
            NADIA_REQUIRE(solvers[j] != solvers[i], NADIA_ERR_INVALID, "handle listed twice");
        (batchable(*solvers[i]) ? fused : other).push_back(solvers[i]);
    }
    for (Solver *s : other) s->iterate(iterations);
    if (fused.empty() || iterations == 0) return;

    std::lock_guard<std::mutex> lock(g_mu);
    std::vector<unsigned long long> key;
    for (Solver *s : fused) key.push_back(s->uid);
    Plan *plan = nullptr;
    for (auto it = g_plans.begin(); it != g_plans.end(); ++it)
        if ((*it)->key == key) {
            g_plans.splice(g_plans.begin(), g_plans, it);
            plan = g_plans.front().get();
            break;
        }
    if (!plan) {
        std::unique_ptr<Plan> p(new Plan);
        p->key = key;
        p->st = fused[0]->st;
        // the plan's buffers are ordered on its stream (a member's, which
        // outlives the plan: plans go before their members' streams do)
        AllocScope scope(p->st);
        std::map<std::tuple<int, int, int, int, int>, size_t> index;
        // mixable members of more than one grid size share the mixed passes
        std::vector<Solver *> mix;
        for (Solver *s : fused)
            if (mixable(*s)) mix.push_back(s);
        bool several = false;
        for (Solver *s : mix)
            several |= s->nx != mix[0]->nx || s->ny != mix[0]->ny;
        for (Solver *s : fused) {
            if (several && mixable(*s)) {
                p->mixed.members.push_back(s);
                continue;
            }
            // PolyCDI members of a group share the padding too
            auto k = std::make_tuple(s->nx, s->ny, s->kind, s->kind == NADIA_POLY ? s->px : 0,
                                     s->kind == NADIA_POLY ? s->py : 0);
            auto f = index.find(k);
            if (f == index.end()) {
                index[k] = p->groups.size();
                p->groups.emplace_back();
                Group &g = p->groups.back();
                g.nx = s->nx;
                g.ny = s->ny;
                g.fresnel = s->kind == NADIA_FRESNEL;
                g.members.push_back(s);
            } else {
                p->groups[f->second].members.push_back(s);
            }
        }
        p->fork.resize(p->groups.size(), nullptr);
        p->join.resize(p->groups.size(), nullptr);
        for (size_t i = 0; i < p->groups.size(); ++i) {
            Group &g = p->groups[i];
            if (g.members[0]->kind == NADIA_POLY) {
                // the padded-grid variants the members picked (the same for all)
                const Fused32::Impl &I0 = *g.members[0]->f32->impl;
                g.pcol = I0.pcol;
                g.prow = I0.prow;
                g.pcols = I0.pcols;
                g.rtiles = I0.nx / I0.prow->L;
                g.twx = I0.twx;
                g.twy = I0.twy;
            } else {
                // the batched tuning class for every group, whatever its size, so a
                // handle's arithmetic does not depend on the other handles of the
                // call; mixable grids use their classes' configuration
                g.choice = mixable(*g.members[0]) ? &class_choice(g.nx, g.ny)
                                                  : &f32::choose(g.nx, g.ny, g.fresnel, kBatchClass);
                g.twx = f32::twiddle_table(g.nx);
                g.twy = f32::twiddle_table(g.ny);
            }
            std::vector<f32::Slot *> hp;
            for (Solver *s : g.members) hp.push_back(s->f32->impl->slot.p);
            g.ptrs.alloc(hp.size());
            NADIA_CUDA(cudaMemcpyAsync(g.ptrs.p, hp.data(), hp.size() * sizeof(f32::Slot *),
                                       cudaMemcpyHostToDevice, p->st));
            // the first group shares the batch stream unless the mixed
            // passes run there
            if (i > 0 || !p->mixed.empty()) {
                NADIA_CUDA(cudaStreamCreateWithFlags(&g.st, cudaStreamNonBlocking));
                NADIA_CUDA(cudaEventCreateWithFlags(&p->fork[i], cudaEventDisableTiming));
                NADIA_CUDA(cudaEventCreateWithFlags(&p->join[i], cudaEventDisableTiming));
            }
        }
        if (!p->mixed.empty()) {
            f32::mix_prepare();
            build_mixed(p->mixed, p->st);
        }
        g_plans.emplace_front(std::move(p));
        while (g_plans.size() > kMaxPlans) g_plans.pop_back();
        plan = g_plans.front().get();
    }

    // order the batch after each member's queued work; set the members'
    // descriptors for the variants this batch uses; prime stale work arrays
    cudaEvent_t ev;
    NADIA_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    for (Solver *s : fused) {
        if (s->st == plan->st) continue;
        NADIA_CUDA(cudaEventRecord(ev, s->st));
        NADIA_CUDA(cudaStreamWaitEvent(plan->st, ev, 0));
    }
    for (Solver *s : plan->mixed.members) {
        Fused32::Impl &I = *s->f32->impl;
        I.check_algorithm();
        I.use_ncol(s->ny / f32::mix_tile(f32::mix_class_of(s->nx)));
        I.push_slot_async(plan->st);
        if (!I.p_valid) I.prime(plan->st);
    }
    for (auto &g : plan->groups)
        for (Solver *s : g.members) {
            Fused32::Impl &I = *s->f32->impl;
            I.check_algorithm();
            if (g.choice) I.use_choice(g.choice);
            I.push_slot_async(plan->st);
            if (!I.p_valid) I.prime(plan->st);
        }
    int left = iterations;
    if (left >= kGraphIters) {
        if (!plan->exec) {
            cudaGraph_t graph = nullptr;
            NADIA_CUDA(cudaStreamBeginCapture(plan->st, cudaStreamCaptureModeThreadLocal));
            plan->launch_block(kGraphIters);
            NADIA_CUDA(cudaStreamEndCapture(plan->st, &graph));
            NADIA_CUDA(cudaGraphInstantiate(&plan->exec, graph, 0));
            cudaGraphDestroy(graph);
        }
        while (left >= kGraphIters) {
            NADIA_CUDA(cudaGraphLaunch(plan->exec, plan->st));
            g_launches += kGraphIters * plan->launches_per_iter();
            left -= kGraphIters;
        }
    }
    if (left > 0) {
        plan->launch_block(left);
        g_launches += left * plan->launches_per_iter();
    }
    NADIA_CUDA(cudaGetLastError());
    NADIA_CUDA(cudaEventRecord(ev, plan->st));
    for (Solver *s : fused) {
        s->iters += iterations;
        s->f32->impl->q_valid = false; // only PfPs iterations carry Q (never batched)
        if (s->st != plan->st) NADIA_CUDA(cudaStreamWaitEvent(s->st, ev, 0));
    }
    NADIA_CUDA(cudaEventDestroy(ev));
}

// Device time of one column pass and one row pass (microseconds, mean of
// `reps` launches with CUDA events on the launching stream) for the batch.
void pass_times(Solver *const *solvers, int count, int reps, double out_us[3])
{
    NADIA_REQUIRE(count >= 1 && reps >= 1, NADIA_ERR_INVALID, "bad count");
    for (int i = 0; i < count; ++i)
        NADIA_REQUIRE(batchable(*solvers[i]) && solvers[i]->nx == solvers[0]->nx &&
                          solvers[i]->ny == solvers[0]->ny && solvers[i]->kind == solvers[0]->kind &&
                          solvers[i]->px == solvers[0]->px && solvers[i]->py == solvers[0]->py,
                      NADIA_ERR_INVALID, "pass timing needs FP32 handles of one size and kind");
    // run one iteration through the batch path so the plan and graph exist
    iterate_many(solvers, count, 1);
    Plan *plan = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        plan = g_plans.front().get();
    }
    cudaStream_t st = plan->st;
    cudaEvent_t e[4];
    for (auto &x : e) NADIA_CUDA(cudaEventCreate(&x));
    float t[3] = {0, 0, 0};
    if (!plan->mixed.empty()) {
        // the members run in the mixed-length passes
        const Mixed &m = plan->mixed;
        for (int r = 0; r < reps; ++r) {
            NADIA_CUDA(cudaEventRecord(e[0], st));
            for (int k = 0; k < 2; ++k)
                f32::mix_launch_col(k == 1, m.col[k].items.p, m.col[k].bounds.p, m.col[k].ctas,
                                    m.ptrs.p, st);
            NADIA_CUDA(cudaEventRecord(e[1], st));
            NADIA_CUDA(cudaEventRecord(e[2], st));
            f32::mix_launch_row(m.row.items.p, m.row.bounds.p, m.row.ctas, m.ptrs.p,
                                (int)m.members.size(), st);
            NADIA_CUDA(cudaEventRecord(e[3], st));
            NADIA_CUDA(cudaEventSynchronize(e[3]));
            for (int k = 0; k < 3; ++k) {
                float ms = 0;
                NADIA_CUDA(cudaEventElapsedTime(&ms, e[k], e[k + 1]));
                t[k] += ms;
            }
        }
        g_launches += (long long)m.launches() * reps;
        for (auto &x : e) cudaEventDestroy(x);
        out_us[0] = 1000.0 * t[0] / reps;
        out_us[1] = 0;
        out_us[2] = 1000.0 * t[2] / reps;
        for (Solver *s : m.members) s->iters += reps;
        return;
    }
    Group &g = plan->groups[0];
    const int n = (int)g.members.size();
    for (int r = 0; r < reps; ++r) {
        NADIA_CUDA(cudaEventRecord(e[0], st));
        if (g.pcol) {
            g.pcol->col_fwd(g.ptrs.p, n, g.pcols, st, g.twx);
            NADIA_CUDA(cudaEventRecord(e[1], st));
            g.pcol->col_inv(g.ptrs.p, n, g.pcols, st, g.twx);
            NADIA_CUDA(cudaEventRecord(e[2], st));
            g.prow->row(f32::kRowFull, g.ptrs.p, n, g.rtiles, st, g.twy);
        } else {
            g.choice->col->col(g.fresnel, g.ptrs.p, n, g.nx, g.ny, g.twx, st);
            NADIA_CUDA(cudaEventRecord(e[1], st));
            NADIA_CUDA(cudaEventRecord(e[2], st));
            g.choice->row->row(f32::kRowFull, g.ptrs.p, n, g.nx, g.ny, g.twy, st);
        }
        NADIA_CUDA(cudaEventRecord(e[3], st));
        NADIA_CUDA(cudaEventSynchronize(e[3]));
        for (int k = 0; k < 3; ++k) {
            float ms = 0;
            NADIA_CUDA(cudaEventElapsedTime(&ms, e[k], e[k + 1]));
            t[k] += ms;
        }
    }
    g_launches += (long long)reps * g.launches_per_iter();
    for (auto &x : e) cudaEventDestroy(x);
    if (!g.pcol) t[1] = 0; // no second column pass
    for (int k = 0; k < 3; ++k) out_us[k] = 1000.0 * t[k] / reps;
    for (Solver *s : g.members) s->iters += reps;
}

void forget_batches_with(unsigned long long uid)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_plans.remove_if([&](const std::unique_ptr<Plan> &p) {
        return std::find(p->key.begin(), p->key.end(), uid) != p->key.end();
    });
}

} // namespace nadia
