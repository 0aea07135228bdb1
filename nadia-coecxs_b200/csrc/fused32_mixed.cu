// fused32_mixed.cu -- the length classes of the mixed-length persistent
// passes and their launchers (see fused32_mixed.cuh).
//
// Classes (512 threads a CTA): transform length, signals per tile, radices;
// swizzles from tests/swizzle_search.py.  Every tile holds at most 8192
// values, so both stages of the column pass (P and sqrt(I)) and of the row
// pass (P, plus x and the support) fit in shared memory.
#include "fused32_mixed.cuh"

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

namespace nadia {
namespace f32 {

constexpr int kMixNT = 512;

// mix_class<N, L, Swizzle, radices...>: one length class, as a column-map and
// a row-map tile configuration
template <int N, int L, class SW, int... Rs>
struct mix_class {
    using Col = TileCfg<N, kMixNT, L, kColMap, Radices<Rs...>, SW, 1>;
    using Row = TileCfg<N, kMixNT, L, kRowMap, Radices<Rs...>, SW, 1>;
};

using Mix2048 = mix_class<2048, 4, Swizzle<4, 5, 7, 1>, 8, 16, 16>;
using Mix1536 = mix_class<1536, 4, Swizzle<4, 0, 3, 2>, 12, 4, 4, 4, 2>;
using Mix1024 = mix_class<1024, 8, Swizzle<4, 6, 3, 2>, 16, 16, 4>;
using Mix768 = mix_class<768, 8, Swizzle<4, 5, 3, 2>, 12, 4, 4, 4>;
using Mix512 = mix_class<512, 16, Swizzle<4, 7, 3, 2>, 8, 8, 8>;

using ColFam = MixFamily<Mix2048::Col, Mix1536::Col, Mix1024::Col, Mix768::Col, Mix512::Col>;
using RowFam = MixFamily<Mix2048::Row, Mix1536::Row, Mix1024::Row, Mix768::Row, Mix512::Row>;

static const char *const kMixRadices[] = {"8.16.16", "12.4.4.4.2", "16.16.4", "12.4.4.4", "8.8.8"};

int mix_class_of(int n) { return ColFam::class_of(n); }
int mix_tile(int cls) { return ColFam::tile(cls); }
int mix_len(int cls) { return ColFam::len(cls); }
int mix_threads() { return kMixNT; }

std::string mix_describe(int n)
{
    const int c = mix_class_of(n);
    if (c < 0) return std::string();
    char t[160];
    snprintf(t, sizeof t, "n=%d threads=%d signals/tile=%d radices=%s mixed-length persistent-TMA",
             n, kMixNT, ColFam::tile(c), kMixRadices[c]);
    return std::string(t);
}

namespace {
MixTw tables()
{
    MixTw t{};
    for (int c = 0; c < ColFam::K; ++c) t.t[c] = twiddle_table(ColFam::len(c));
    return t;
}

// estimated work of one tile of a class: values x passes
double tile_cost(int cls)
{
    static const int passes[] = {3, 5, 3, 4, 3};
    return (double)ColFam::len(cls) * ColFam::tile(cls) * passes[cls];
}
} // namespace

int mix_ctas() { return sm_count(); }

// Orders the items by class (stable: member order within a class) and cuts
// the list into `ctas` contiguous ranges of about equal estimated work;
// bounds gets ctas + 1 entries.
void mix_order(std::vector<MixItem> &items, std::vector<int> &bounds, int ctas)
{
    std::stable_sort(items.begin(), items.end(),
                     [](const MixItem &a, const MixItem &b) { return a.cls < b.cls; });
    double total = 0;
    for (const auto &m : items) total += tile_cost(m.cls);
    bounds.assign(ctas + 1, (int)items.size());
    bounds[0] = 0;
    double acc = 0;
    int b = 1;
    for (size_t i = 0; i < items.size() && b < ctas; ++i) {
        acc += tile_cost(items[i].cls);
        while (b < ctas && acc >= total * b / ctas) bounds[b++] = (int)i + 1;
    }
}

// The persistent single-length variant with a class's tile configuration:
// a batch of one grid size runs it (the same arithmetic as the class in the
// mixed passes, without the other classes' code)
const TileVariant *mix_variant(int n)
{
    const int c = mix_class_of(n);
    if (c < 0) return nullptr;
    for (const auto &v : variants(n))
        if (v.persistent && !v.single && !v.direct && v.col && v.row && v.nt == kMixNT &&
            v.L == ColFam::tile(c) && std::string(v.radices) == kMixRadices[c])
            return &v;
    return nullptr;
}

void mix_prepare()
{
    NADIA_CUDA(cudaFuncSetAttribute(kp_colm<ColFam, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)mix_col_smem<ColFam>()));
    NADIA_CUDA(cudaFuncSetAttribute(kp_colm<ColFam, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)mix_col_smem<ColFam>()));
    NADIA_CUDA(cudaFuncSetAttribute(kp_rowm<RowFam>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)mix_row_smem<RowFam>()));
    tables(); // the twiddle tables exist before any capture
}

void mix_launch_col(bool fresnel, const MixItem *items, const int *bounds, int ctas,
                    const Slot *const *slots, cudaStream_t st)
{
    if (ctas <= 0) return;
    if (fresnel)
        kp_colm<ColFam, true><<<ctas, kMixNT, mix_col_smem<ColFam>(), st>>>(items, bounds, slots, tables());
    else
        kp_colm<ColFam, false><<<ctas, kMixNT, mix_col_smem<ColFam>(), st>>>(items, bounds, slots, tables());
}

void mix_launch_row(const MixItem *items, const int *bounds, int ctas, const Slot *const *slots,
                    int nslots, cudaStream_t st)
{
    if (ctas <= 0) return;
    kp_rowm<RowFam><<<ctas, kMixNT, mix_row_smem<RowFam>(), st>>>(items, bounds, slots, nslots,
                                                                 tables());
}

} // namespace f32
} // namespace nadia
