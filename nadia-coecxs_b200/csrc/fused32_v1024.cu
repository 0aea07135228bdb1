// fused32_v1024.cu -- the FP32 tile variants of transform length 1024.
// Swizzles from tests/swizzle_search.py (conflict-free exchanges).
#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

void add_variants_1024(std::vector<TileVariant> &v)
{
    v.push_back(make_variant<1024, 256, 4, 2, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4"));
    v.push_back(make_variant<1024, 128, 4, 4, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4"));
    v.push_back(make_variant<1024, 512, 4, 2, Swizzle<4, 5, 3, 2>, 8, 8, 4, 4>("8.8.4.4"));
    v.push_back(make_variant<1024, 512, 8, 1, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4"));
    v.push_back(make_persistent<1024, 256, 4, 2, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4"));
    v.push_back(make_persistent<1024, 128, 4, 4, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4"));
    v.push_back(make_persistent<1024, 512, 4, 2, Swizzle<4, 5, 3, 2>, 8, 8, 4, 4>("8.8.4.4"));
    v.push_back(make_persistent<1024, 512, 8, 1, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4"));
    v.push_back(make_ping<1024, 256, 4, 2, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4"));
    v.push_back(make_ping<1024, 512, 4, 2, Swizzle<4, 5, 3, 2>, 8, 8, 4, 4>("8.8.4.4"));
    // column passes that stage sqrt(I) (and the white field) by cp.async
    v.push_back(make_staged_ping<1024, 256, 4, 2, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4 staged"));
    v.push_back(make_staged<1024, 256, 4, 2, Swizzle<4, 6, 3, 2>, 16, 16, 4>("16.16.4 staged"));
}

} // namespace f32
} // namespace nadia
