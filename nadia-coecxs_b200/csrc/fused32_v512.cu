// fused32_v512.cu -- the FP32 tile variants of transform length 512.
// Swizzles from tests/swizzle_search.py (conflict-free exchanges).
#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

void add_variants_512(std::vector<TileVariant> &v)
{
    v.push_back(make_variant<512, 256, 8, 2, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4"));
    v.push_back(make_variant<512, 128, 4, 4, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4"));
    v.push_back(make_variant<512, 256, 4, 3, Swizzle<4, 0, 7, 1>, 8, 8, 8>("8.8.8"));
    v.push_back(make_persistent<512, 256, 8, 2, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4"));
    v.push_back(make_persistent<512, 128, 4, 4, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4"));
    v.push_back(make_persistent<512, 256, 4, 3, Swizzle<4, 0, 7, 1>, 8, 8, 8>("8.8.8"));
    v.push_back(make_ping<512, 256, 8, 2, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4"));
    // the tile configuration of this length's class in the mixed-length passes
    v.push_back(make_persistent<512, 512, 16, 1, Swizzle<4, 7, 3, 2>, 8, 8, 8>("8.8.8"));
    // column passes that stage sqrt(I) (and the white field) by cp.async
    v.push_back(make_staged<512, 256, 8, 2, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4 staged"));
    v.push_back(make_staged<512, 128, 4, 4, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4 staged"));
}

} // namespace f32
} // namespace nadia
