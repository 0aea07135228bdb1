// fused32_v1536.cu -- the FP32 tile variants of transform length 1536.
// Swizzles from tests/swizzle_search.py (conflict-free exchanges).
#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

void add_variants_1536(std::vector<TileVariant> &v)
{
    v.push_back(make_variant<1536, 256, 4, 2, Swizzle<4, 5, 7, 1>, 8, 8, 8, 3>("8.8.8.3"));
    v.push_back(make_variant<1536, 512, 4, 1, Swizzle<4, 5, 3, 2>, 4, 4, 4, 4, 2, 3>("4.4.4.4.2.3"));
    v.push_back(make_persistent<1536, 256, 4, 2, Swizzle<4, 5, 7, 1>, 8, 8, 8, 3>("8.8.8.3"));
    v.push_back(make_persistent<1536, 512, 4, 1, Swizzle<4, 5, 3, 2>, 4, 4, 4, 4, 2, 3>("4.4.4.4.2.3"));
    v.push_back(make_ping<1536, 256, 4, 2, Swizzle<4, 5, 7, 1>, 8, 8, 8, 3>("8.8.8.3"));
    // the tile configuration of this length's class in the mixed-length passes
    v.push_back(make_persistent<1536, 512, 4, 1, Swizzle<4, 0, 3, 2>, 12, 4, 4, 4, 2>("12.4.4.4.2"));
    // column passes that stage sqrt(I) (and the white field) by cp.async
    v.push_back(make_staged_ping<1536, 256, 4, 2, Swizzle<4, 5, 7, 1>, 8, 8, 8, 3>("8.8.8.3 staged"));
    v.push_back(make_staged<1536, 256, 4, 2, Swizzle<4, 5, 7, 1>, 8, 8, 8, 3>("8.8.8.3 staged"));
}

} // namespace f32
} // namespace nadia
