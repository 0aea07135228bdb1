// fused32_impl.h -- device descriptors and host state of the FP32 engine.
#pragma once

#include <vector>

#include "common.h"
#include "fused32.h"

namespace nadia {

struct Solver;

namespace f32 {

// One reconstruction as the fused kernels see it.  It lives in device
// memory, so graphs captured once keep working when the algorithm changes.
struct Slot {
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
};

struct Gauss {
    float w[6];
    int cut;
};

__host__ __device__ inline size_t panel_index_dev(int x, int y, int nx)
{
    return ((size_t)(y / 4) * nx + x) * 4 + (y % 4);
}

bool supported(int n);
void prepare(int nx, int ny);
int col_tile(int n);
int row_tile(int n);
void col_launch(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                const float2 *tw, cudaStream_t st);
void row_launch(int mode, const Slot *const *slots, int nslots, int nx, int ny, const float2 *tw,
                cudaStream_t st);
const float2 *twiddle_table(int n);

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
    DevBuf<f32::Slot> slot;
    DevBuf<f32::Slot *> slot_ptr;
    f32::Slot h_slot{};
    const float2 *twx = nullptr, *twy = nullptr;
    std::vector<double> h_bs;
    bool p_valid = false;
    cudaGraphExec_t graph_exec = nullptr;

    explicit Impl(Solver &s);
    ~Impl();
    void push_slot();
    void to_panel(const double *h, size_t stride, std::vector<float> &out) const;
    void from_panel(const std::vector<float> &in, size_t stride, double *h) const;
    void upload(void *dst, const std::vector<float> &v);
    void download(std::vector<float> &v, const void *src, size_t count);
    void upload_intensity();
    void blur(bool cplx, const void *in, double gauss_width, int cut);
    void check_algorithm() const;
    void prime(cudaStream_t st);
    void launch_iteration(cudaStream_t st);
};

} // namespace nadia
