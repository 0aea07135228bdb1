// batch.h -- stepping several reconstructions together, and launch accounting.
#pragma once

#include <atomic>

namespace nadia {

struct Solver;

// kernels of this library launched so far (graph replays count their kernels)
extern std::atomic<long long> g_launches;

void iterate_many(Solver *const *solvers, int count, int iterations);
void pass_times(Solver *const *solvers, int count, int reps, double out_us[3]);
void forget_batches_with(unsigned long long uid);

} // namespace nadia
