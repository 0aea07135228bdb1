// fused32_v2048.cu -- the FP32 tile variants of transform length 2048.
// Swizzles from tests/swizzle_search.py (conflict-free exchanges).
#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

void add_variants_2048(std::vector<TileVariant> &v)
{
    v.push_back(make_variant<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_variant<2048, 256, 4, 2, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_variant<2048, 1024, 4, 1, Swizzle<4, 5, 3, 2>, 8, 8, 8, 4>("8.8.8.4"));
    v.push_back(make_variant<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_variant<2048, 1024, 8, 1, Swizzle<4, 6, 3, 2>, 16, 16, 8>("16.16.8"));
    v.push_back(make_persistent<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_persistent<2048, 256, 4, 2, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_persistent<2048, 1024, 4, 1, Swizzle<4, 5, 3, 2>, 8, 8, 8, 4>("8.8.8.4"));
    v.push_back(make_persistent<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_ping<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_ping<2048, 1024, 4, 1, Swizzle<4, 5, 3, 2>, 8, 8, 8, 4>("8.8.8.4"));
    v.push_back(make_ping<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    // two CTAs per SM: one-stage column tiles of 32 values a thread, row tiles of two rows
    v.push_back(make_persistent_single<2048, 256, 4, 2, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_persistent_single<2048, 256, 4, 2, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_persistent_row<2048, 256, 2, 2, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_persistent_row<2048, 256, 2, 2, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    // column passes reading sqrt(I) from global memory: one stage, two CTAs per
    // SM; or two stages with ping-pong exchanges (one barrier per exchange)
    v.push_back(make_persistent_direct<2048, 256, 4, 2, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_persistent_ping<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_persistent_ping<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_persistent_ping<2048, 1024, 4, 1, Swizzle<4, 5, 3, 2>, 8, 8, 8, 4>("8.8.8.4"));
    // column passes with one sqrt(I) stage refilled after each modulus and
    // ping-pong exchanges (one barrier per exchange)
    v.push_back(make_persistent_mstage<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_persistent_mstage<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    // column passes in two independent groups of 256 threads (half panels)
    v.push_back(make_grouped_col<2048, 256, 2, 2, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_grouped_col<2048, 256, 2, 2, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    // row passes in independent groups: four of 128 threads (one row each) or
    // two of 256 (two rows each), every group with its own pipeline
    v.push_back(make_grouped_row<2048, 128, 1, 4, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_grouped_row<2048, 128, 1, 4, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    v.push_back(make_grouped_row<2048, 256, 2, 2, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16"));
    v.push_back(make_grouped_row<2048, 256, 2, 2, Swizzle<4, 5, 7, 1>, 16, 16, 8>("16.16.8"));
    // the best column and row shapes with every twiddle loaded from the table
    v.push_back(make_persistent_tw<2048, 512, 4, 1, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16 tw"));
    v.push_back(make_grouped_row_tw<2048, 128, 1, 4, Swizzle<4, 5, 7, 1>, 8, 16, 16>("8.16.16 tw"));
    // column passes that stage sqrt(I) (and the white field) by cp.async
    v.push_back(make_staged_ping<2048, 1024, 4, 1, Swizzle<4, 5, 3, 2>, 8, 8, 8, 4>("8.8.8.4 staged"));
    v.push_back(make_staged<2048, 1024, 4, 1, Swizzle<4, 5, 3, 2>, 8, 8, 8, 4>("8.8.8.4 staged"));
}

} // namespace f32
} // namespace nadia
