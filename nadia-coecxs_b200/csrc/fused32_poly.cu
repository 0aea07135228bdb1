// fused32_poly.cu -- the FP32 PolyCDI form: tile shapes of the padded grid
// sizes, the set-up done by set_spectrum, and the iteration (the kernels and
// their design are in fused32_poly.cuh).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>

#include "batch.h"
#include "fused32.h"
#include "fused32_poly.cuh"
#include "solver.h"

namespace nadia {
namespace f32 {

// Padded sizes with PolyCDI tiles: 256 and 512 (small cases) and 1080, the
// 1024 x 1024 detector padded by 28 on each side (1080 = 6*6*6*5, so every
// radix divides the 30 values a thread holds).  A 1080-point tile needs
// about 168 registers a thread, so an SM holds 288 such threads: as one CTA
// of 8 signals, or as two independent CTAs of 4 signals and 144 threads
// (four and a half warps), whose global loads and barriers overlap each
// other's arithmetic.  Swizzles from tests/swizzle_search.py.
const std::vector<PolyVariant> &poly_variants(int n)
{
    static const std::map<int, std::vector<PolyVariant>> reg = [] {
        std::map<int, std::vector<PolyVariant>> r;
        r[256].push_back(make_poly<256, 256, 8, 3, Swizzle<4, 6, 3, 2>, 8, 8, 4>("8.8.4"));
        r[512].push_back(make_poly<512, 256, 8, 2, Swizzle<4, 6, 3, 2>, 16, 8, 4>("16.8.4"));
        r[1080].push_back(make_poly<1080, 144, 4, 2, Swizzle<7, 0, 7, 1>, 6, 6, 6, 5>("6.6.6.5"));
        r[1080].push_back(
            make_poly<1080, 144, 4, 2, Swizzle<7, 0, 7, 1>, 6, 6, 6, 5>("6.6.6.5 direct", false));
        r[1080].push_back(
            make_poly<1080, 288, 8, 1, Swizzle<4, 0, 1, 2>, 6, 6, 6, 5>("6.6.6.5 direct", false));
        return r;
    }();
    static const std::vector<PolyVariant> none;
    auto it = reg.find(n);
    return it == reg.end() ? none : it->second;
}

} // namespace f32

using namespace f32;

namespace {

// the first variant whose tiles divide `tiles_of` (column tiles run over the
// padded columns, row tiles over the estimate's rows); NADIA_POLY_TILE=k
// starts the search at the k-th registered shape of the size
const PolyVariant *pick(int n, int tiles_of)
{
    const auto &vs = poly_variants(n);
    const char *e = std::getenv("NADIA_POLY_TILE");
    const size_t first = e ? (size_t)std::max(0, std::atoi(e)) : 0;
    for (size_t k = first < vs.size() ? first : 0; k < vs.size(); ++k)
        if (tiles_of % vs[k].L == 0) return &vs[k];
    return nullptr;
}

} // namespace

// PolyCDI::set_spectrum (PolyCDI.c++:66-89) on the FP32 form: the padded
// grid, the |Psi|^2 buffer and the gather tables of expand_wl
// (PolyCDI.c++:296-334): for wavelength l and unpadded row i (padded row
// i + px) the sampled row is ga = (int)(lf*(i + px - nx/2) + nx/2) with
// lf = lambda_l / lambda_c, or none when outside [0, mx); likewise columns
// (gb).  The tables hold the row and column parts of the sample's address
// in q's panel layout (k_poly_expand).
void Fused32::set_spectrum()
{
    Impl &I = *impl;
    Solver &S = I.S;
    const int mx = S.nx + 2 * S.px, my = S.ny + 2 * S.py;
    const PolyVariant *pc = pick(mx, my), *pr = pick(my, S.nx);
    NADIA_REQUIRE(pc && pr, NADIA_ERR_UNSUPPORTED,
                  "the FP32 PolyCDI form supports padded grids of 256, 512 and 1080 per axis "
                  "(for example 1024 padded by 28); use NADIA_FP64 for others");
    NADIA_REQUIRE(mx % 4 == 0 && my % 4 == 0, NADIA_ERR_UNSUPPORTED, "padded grid not a multiple of 4");
    pc->prepare();
    pr->prepare();
    NADIA_CUDA(cudaStreamSynchronize(S.st));
    if (I.graph_exec) { // captured for the previous padded grid
        cudaGraphExecDestroy(I.graph_exec);
        I.graph_exec = nullptr;
    }
    I.mx = mx;
    I.my = my;
    I.pcol = pc;
    I.prow = pr;
    I.pcols = my / pc->L;
    const size_t m = (size_t)mx * my;
    I.P.alloc(m);
    I.q.alloc(m);
    I.ratio.alloc(I.n);
    I.partials.alloc(kExpandBlocks); // error partials: one per expansion block
    NADIA_CUDA(cudaMemsetAsync(I.P.p, 0, I.P.bytes(), S.st));
    NADIA_CUDA(cudaMemsetAsync(I.q.p, 0, I.q.bytes(), S.st));
    const int nl = S.nlambda;
    std::vector<int> gx((size_t)nl * S.nx), gy((size_t)nl * S.ny);
    std::vector<float> w(nl);
    for (int l = 0; l < nl; ++l) {
        const double lf = S.spectrum[2 * l] / S.lambdac;
        for (int i = 0; i < S.nx; ++i) {
            const double xval = lf * ((i + S.px) - S.nx / 2.0) + S.nx / 2.0;
            gx[(size_t)l * S.nx + i] = (xval >= 0 && xval < mx) ? (int)xval * kPanel : kNoSample;
        }
        for (int j = 0; j < S.ny; ++j) {
            const double yval = lf * ((j + S.py) - S.ny / 2.0) + S.ny / 2.0;
            const int gb = (int)yval;
            gy[(size_t)l * S.ny + j] = (yval >= 0 && yval < my)
                                           ? (gb / kPanel) * kPanel * mx + gb % kPanel
                                           : kNoSample;
        }
        w[l] = (float)S.spectrum[2 * l + 1];
    }
    I.gx.alloc(gx.size());
    I.gy.alloc(gy.size());
    I.wl.alloc(nl);
    upload_now(I.gx.p, gx.data(), I.gx.bytes());
    upload_now(I.gy.p, gy.data(), I.gy.bytes());
    upload_now(I.wl.p, w.data(), I.wl.bytes());
    I.twx = twiddle_table(mx);
    I.twy = twiddle_table(my);
    Slot &h = I.h_slot;
    h.P = I.P.p;
    h.partials = I.partials.p;
    h.q = I.q.p;
    h.gx = I.gx.p;
    h.gy = I.gy.p;
    h.wl = I.wl.p;
    h.nl = nl;
    h.px = S.px;
    h.py = S.py;
    h.mx = mx;
    h.my = my;
    h.ratio = I.ratio.p;
    h.ncol = kExpandBlocks;
    h.s0 = (float)(1.0 / std::sqrt((double)mx * (double)my));
    I.p_valid = false;
    I.push_slot();
}

void Fused32::iterate_poly(int count)
{
    Impl &I = *impl;
    NADIA_REQUIRE(I.pcol && I.prow, NADIA_ERR_STATE, "PolyCDI needs set_spectrum before it can project");
    I.check_algorithm();
    I.push_slot();
    cudaStream_t st = I.S.st;
    const Slot *const *sl = I.slot_ptr.p;
    const int rtiles = I.nx / I.prow->L;
    if (!I.p_valid) I.prime(st);
    auto one = [&] {
        I.pcol->col_fwd(sl, 1, I.pcols, st, I.twx);
        I.pcol->col_inv(sl, 1, I.pcols, st, I.twx);
        I.prow->row(kRowFull, sl, 1, rtiles, st, I.twy);
    };
    const int G = Impl::kGraphIters;
    int left = count;
    if (left >= G) {
        if (!I.graph_exec) {
            cudaGraph_t g = nullptr;
            NADIA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            for (int i = 0; i < G; ++i) one();
            NADIA_CUDA(cudaStreamEndCapture(st, &g));
            NADIA_CUDA(cudaGraphInstantiate(&I.graph_exec, g, 0));
            cudaGraphDestroy(g);
        }
        while (left >= G) {
            NADIA_CUDA(cudaGraphLaunch(I.graph_exec, st));
            g_launches += 4 * G;
            left -= G;
        }
    }
    for (; left > 0; --left) {
        one();
        g_launches += 4;
    }
    NADIA_CUDA(cudaGetLastError());
    I.S.iters += count;
}

} // namespace nadia
