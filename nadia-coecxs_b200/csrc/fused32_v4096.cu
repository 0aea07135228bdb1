// fused32_v4096.cu -- the FP32 tile variants of transform length 4096.
// Swizzles from tests/swizzle_search.py (conflict-free exchanges).
#include "fused32_kernels.cuh"

namespace nadia {
namespace f32 {

void add_variants_4096(std::vector<TileVariant> &v)
{
    v.push_back(make_variant<4096, 1024, 4, 1, Swizzle<4, 5, 7, 1>, 16, 16, 16>("16.16.16"));
    v.push_back(make_variant<4096, 512, 4, 1, Swizzle<4, 5, 7, 1>, 16, 16, 16>("16.16.16"));
}

} // namespace f32
} // namespace nadia
