// fused32_v768.cu -- the FP32 tile variants of transform length 768.
// Swizzles from tests/swizzle_search.py (conflict-free exchanges).
#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

void add_variants_768(std::vector<TileVariant> &v)
{
    v.push_back(make_variant<768, 256, 8, 2, Swizzle<4, 6, 3, 2>, 8, 8, 4, 3>("8.8.4.3"));
    v.push_back(make_variant<768, 128, 4, 4, Swizzle<4, 0, 7, 1>, 8, 8, 4, 3>("8.8.4.3"));
    v.push_back(make_variant<768, 256, 4, 2, Swizzle<4, 6, 3, 2>, 4, 4, 4, 4, 3>("4.4.4.4.3"));
    v.push_back(make_persistent<768, 256, 8, 2, Swizzle<4, 6, 3, 2>, 8, 8, 4, 3>("8.8.4.3"));
    v.push_back(make_persistent<768, 128, 4, 4, Swizzle<4, 0, 7, 1>, 8, 8, 4, 3>("8.8.4.3"));
    v.push_back(make_persistent<768, 256, 4, 2, Swizzle<4, 6, 3, 2>, 4, 4, 4, 4, 3>("4.4.4.4.3"));
    v.push_back(make_ping<768, 256, 8, 2, Swizzle<4, 6, 3, 2>, 8, 8, 4, 3>("8.8.4.3"));
    // the tile configuration of this length's class in the mixed-length passes
    v.push_back(make_persistent<768, 512, 8, 1, Swizzle<4, 5, 3, 2>, 12, 4, 4, 4>("12.4.4.4"));
    // column passes that stage sqrt(I) (and the white field) by cp.async
    v.push_back(make_staged<768, 128, 4, 4, Swizzle<4, 0, 7, 1>, 8, 8, 4, 3>("8.8.4.3 staged"));
    v.push_back(make_staged<768, 256, 8, 2, Swizzle<4, 6, 3, 2>, 8, 8, 4, 3>("8.8.4.3 staged"));
}

} // namespace f32
} // namespace nadia
