// fused32_v256.cu -- the FP32 tile variants of transform length 256.
// Swizzles from tests/swizzle_search.py (conflict-free exchanges).
#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

void add_variants_256(std::vector<TileVariant> &v)
{
    v.push_back(make_variant<256, 256, 16, 2, Swizzle<4, 8, 3, 2>, 16, 16>("16.16"));
    v.push_back(make_variant<256, 128, 8, 4, Swizzle<4, 7, 3, 2>, 16, 16>("16.16"));
    v.push_back(make_variant<256, 256, 8, 3, Swizzle<4, 6, 3, 2>, 8, 8, 4>("8.8.4"));
    v.push_back(make_persistent<256, 256, 16, 2, Swizzle<4, 8, 3, 2>, 16, 16>("16.16"));
    v.push_back(make_persistent<256, 128, 8, 4, Swizzle<4, 7, 3, 2>, 16, 16>("16.16"));
    v.push_back(make_persistent<256, 256, 8, 3, Swizzle<4, 6, 3, 2>, 8, 8, 4>("8.8.4"));
    v.push_back(make_ping<256, 256, 16, 2, Swizzle<4, 8, 3, 2>, 16, 16>("16.16"));
}

} // namespace f32
} // namespace nadia
