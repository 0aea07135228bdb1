// fused32_impl.h -- device descriptors and host state of the FP32 engine.
#pragma once

#include <vector>
#include <string>

#include <cuda.h>

#include "common.h"
#include "fused32.h"

namespace nadia {

struct Solver;

namespace f32 {

// One reconstruction as the fused kernels see it.  It lives in device
// memory, so graphs captured once keep working when the algorithm changes.
struct alignas(64) Slot {
    // tensor maps over P, x and the support for row tiles of 4, 8 and 16 rows
    // (persistent row pass); box (K, rows, <= 256 panels)
    CUtensorMap tm[3][3];
    float2 *P;              // work array (row transforms of x / column-pass output)
    float2 *x;              // estimate
    const float *sup;       // support
    const float *mI;        // sqrt(I) in transform order, -1 where unmeasured
    const float2 *W;        // Fresnel: white field in transform order (else null)
    const float2 *tx, *ty;  // Fresnel: per-axis phase factors (else null)
    double *partials;       // column-pass error partial sums, one per column block
    double *err;            // current error metric
    double *ring;           // error history
    long long *iter;        // iterations completed
    int ring_len;
    int ncol;               // column blocks per reconstruction
    float w_id, w_pf, w_ps, w_psf; // combine weights (1+PI, PF, PS, PSF)
    int er;                 // ER: x' = Ps Pf x
    int project;            // the algorithm projects (else the error is carried over)
    float s0;               // 1/sqrt(nx*ny)
    double inv_norm2;       // 1 / sum of sqrt(I)^2 over measured pixels
    int *flag;              // raised when a device-side wait gives up
};

struct Gauss {
    float w[6];
    int cut;
};

// panels per tensor box: the largest divisor of the panel count that is at
// most 256 (the TMA box limit), so the boxes tile a row tile exactly
__host__ __device__ inline int box_panels(int npan)
{
    for (int d = npan < 256 ? npan : 256; d > 1; --d)
        if (npan % d == 0) return d;
    return 1;
}

__host__ __device__ inline size_t panel_index_dev(int x, int y, int nx)
{
    return ((size_t)(y / 4) * nx + x) * 4 + (y % 4);
}

enum { kRowFull = 0, kRowPrime = 1 };

using ColLaunch = void (*)(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                           const float2 *tw, cudaStream_t st);
using RowLaunch = void (*)(int mode, const Slot *const *slots, int nslots, int nx, int ny,
                           const float2 *tw, cudaStream_t st);

// One compiled tile shape of a transform length, usable as column pass
// (length nx) and as row pass (length ny).
struct TileVariant {
    int n = 0, nt = 0, L = 0, minb = 0;
    bool persistent = false;
    bool ping = false;
    const char *radices = "";
    void (*prepare)() = nullptr;
    ColLaunch col = nullptr;
    RowLaunch row = nullptr;
};

// the variants of a transform length (empty when the length has none)
const std::vector<TileVariant> &variants(int n);
bool supported(int n);

// The column- and row-pass variants the autotuner picked for a grid, kind and
// batch class (one reconstruction, or several per launch).
struct Choice {
    const TileVariant *col = nullptr, *row = nullptr;
    float col_us = 0, row_us = 0;
};
const Choice &choose(int nx, int ny, bool fresnel, int nslots);

const float2 *twiddle_table(int n);
int sm_count();
// tensor maps of a slot's P, x and support (needs P, x, sup set)
void encode_tensor_maps(Slot &s, int nx, int ny);

} // namespace f32

struct Fused32::Impl {
    static constexpr int kGraphIters = 16;
    static constexpr int kMaxBlocks = 592;

    Solver &S;
    int nx = 0, ny = 0, ncol = 0;
    size_t n = 0;
    DevBuf<float2> P, x, W, ill, tx, ty;
    DevBuf<float> sup, mI, tmp1, tmp2, maxpart;
    DevBuf<double> partials;
    DevBuf<long long> iter;
    DevBuf<int> flag;
    DevBuf<f32::Slot> slot;
    DevBuf<f32::Slot *> slot_ptr;
    f32::Slot h_slot{};
    const float2 *twx = nullptr, *twy = nullptr;
    const f32::Choice *choice = nullptr;
    std::vector<double> h_bs;
    bool p_valid = false;
    cudaGraphExec_t graph_exec = nullptr;

    explicit Impl(Solver &s);
    ~Impl();
    void push_slot();
    void push_slot_async(cudaStream_t st);
    // the variants the next launches use (the handle's own, or a batch's);
    // sets the column-block count the row pass sums over
    void use_choice(const f32::Choice *c);
    void to_panel(const double *h, size_t stride, std::vector<float> &out) const;
    void from_panel(const std::vector<float> &in, size_t stride, double *h) const;
    void upload(void *dst, const std::vector<float> &v);
    void download(std::vector<float> &v, const void *src, size_t count);
    void upload_intensity();
    void blur(bool cplx, const void *in, double gauss_width, int cut);
    int blur_blocks() const;
    void check_algorithm() const;
    void prime(cudaStream_t st);
    void launch_iteration(cudaStream_t st);
};

} // namespace nadia
