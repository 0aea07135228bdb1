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
    // tensor maps over P, x and the support for row tiles of 1, 2, 4, 8 and
    // 16 rows (persistent row passes); box (K, rows, <= 256 panels)
    CUtensorMap tm[5][3];
    // grouped column pass: P as column pairs (box (2, <= 256 rows, 1 panel))
    // and sqrt(I) as whole panels (box (4, <= 256 rows, 1 panel))
    CUtensorMap tc[2];
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
    int project;            // the algorithm projects x (else the error is carried over,
                            // or, with a PfPs term, taken from the projection of Ps x)
    // algorithms with a PfPs term: Q holds the row transforms of Ps x (the
    // second field the column pass projects), qpartials its error partials,
    // w_pfs its weight in the combine
    float2 *Q;
    double *qpartials;
    float w_pfs;
    int pfs;
    float s0;               // 1/sqrt(nx*ny)
    double inv_norm2;       // 1 / sum of sqrt(I)^2 over measured pixels
    int *flag;              // raised when a device-side wait gives up
    // polls before a persistent pass's mbarrier wait gives up (0: kWaitPolls)
    // and a hook for testing that failure path: when set, the first tile of
    // each CTA is expected on its barrier but its copy is never issued, so
    // that wait runs out (no copy is left in flight).  Both come from
    // NADIA_FAULT_WAIT=<polls> at handle creation; unset, they are 0.
    unsigned wait_polls;
    int skip_first_load;
    // TransmissionConstraint's per-pixel part (charge flipping, unit
    // magnitude) applied in each support projection of the row pass (the
    // non-persistent variants); for FresnelCDI on the transmission function,
    // with tc_ill the illumination at the sample (else null)
    int tc_on, tc_unity, tc_flip;
    float tc_sign;
    const float2 *tc_ill;
    // complex-constraint regions (TransmissionConstraint.c++:76-172), when
    // tc_R > 0: each pixel's region (0: none; panel layout), per region
    // alpha1, alpha2, fixed flag, fixed c_mean; c_mean per field and region
    // (field 0: Ps x, 1: Ps of the projection, 2: a whole array), the FP64
    // region partials, and Y, the row pass's inverse transforms, kept between
    // its two halves while the region sums are formed
    int tc_R;
    const int *tc_region;
    const float *tc_par;
    float *tc_cm;
    double *tc_part;
    float2 *Y;
    // PolyCDI: P is the padded mx x my grid (the estimate sits at rows
    // px..px+nx-1, columns py..py+ny-1); q holds |Psi|^2 of the padded
    // detector field in centred coordinates (panel layout over mx rows);
    // gx/gy[l][i] are the rows/columns sampled for wavelength l at unpadded
    // row/column i (-1: outside the grid); wl[l] the normalised weights
    float *q;
    float *ratio;           // modulus ratio per pixel of the detector window (panel layout)
    const int *gx, *gy;
    const float *wl;
    int nl, px, py, mx, my;
};

#ifdef __CUDACC__
// TransmissionConstraint::apply_constraint's per-pixel part
// (TransmissionConstraint.c++:136-160): charge flipping, then unit magnitude
// judged on the magnitude before the flip
__device__ __forceinline__ float2 tc_pixel(float2 v, const Slot &S)
{
    const float mag_old = sqrtf(v.x * v.x + v.y * v.y);
    if (S.tc_flip && S.tc_sign * v.y > 0.f) v.y = -1.f * v.y;
    if (S.tc_unity && mag_old > 1.f) {
        const float m = sqrtf(v.x * v.x + v.y * v.y);
        if (m == 0.f) {
            v = make_float2(1.f, 0.f);
        } else {
            const float q = 1.f / m;
            v = make_float2(v.x * q, v.y * q);
        }
    }
    return v;
}
#endif

struct Gauss {
    float w[6];
    int cut;
};

// rows (x) per tensor box of the grouped column pass: the largest divisor of
// nx that is at most 256
__host__ __device__ inline int box_rows(int nx)
{
    for (int d = nx < 256 ? nx : 256; d > 1; --d)
        if (nx % d == 0) return d;
    return 1;
}

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

// row-pass modes: the iteration's row pass; the forward row transform of x
// alone (prime: P = rows of x); and the same two for algorithms with a PfPs
// term, which also carry Q = rows of Ps x
enum { kRowFull = 0, kRowPrime = 1, kRowPfs = 2, kRowPrimePfs = 3 };

using ColLaunch = void (*)(bool fresnel, const Slot *const *slots, int nslots, int nx, int ny,
                           const float2 *tw, cudaStream_t st);
using RowLaunch = void (*)(int mode, const Slot *const *slots, int nslots, int nx, int ny,
                           const float2 *tw, cudaStream_t st);
using WfColLaunch = void (*)(const Slot *const *slots, int nslots, int nx, int ny,
                             const float2 *tw, cudaStream_t st);

// One compiled tile shape of a transform length, usable as column pass
// (length nx) and as row pass (length ny); a variant that serves only one of
// the two passes leaves the other launcher null.
struct TileVariant {
    int n = 0, nt = 0, L = 0, minb = 0;
    bool persistent = false;
    bool ping = false;
    bool single = false; // persistent column pass with one stage per CTA
    bool direct = false; // persistent column pass reading sqrt(I) from global memory
    int groups = 1;      // independent thread groups a CTA (grouped row pass)
    const char *radices = "";
    void (*prepare)() = nullptr;
    ColLaunch col = nullptr;
    RowLaunch row = nullptr;
    // FresnelCDI_WF passes in this tile shape (plain variants only)
    WfColLaunch wf_col = nullptr;
    RowLaunch wf_row = nullptr;
    // the row pass's two halves around complex-constraint region sums
    // (mode 1: inverse transforms into Y; 2: the constrained combine and the
    // forward transforms; plain variants only)
    RowLaunch tc_row = nullptr;
};

// PolyCDI passes of one tile shape: forward column transform of the padded
// grid (writes Psi and |Psi|^2), modulus against the wavelength-expanded
// intensity plus inverse column transform, and the row pass over the
// estimate's rows of the padded grid.
using PolyLaunch = void (*)(const Slot *const *slots, int nslots, int tiles, cudaStream_t st,
                            const float2 *tw);
using PolyRowLaunch = void (*)(int mode, const Slot *const *slots, int nslots, int tiles,
                               cudaStream_t st, const float2 *tw);
struct PolyVariant {
    int n = 0, nt = 0, L = 0;
    const char *radices = "";
    void (*prepare)() = nullptr;
    PolyLaunch col_fwd = nullptr, col_inv = nullptr;
    PolyRowLaunch row = nullptr;
};
const std::vector<PolyVariant> &poly_variants(int n);

// the variants of a transform length (empty when the length has none)
const std::vector<TileVariant> &variants(int n);
bool supported(int n);

// The column- and row-pass variants the autotuner picked for a grid, kind and
// batch class (one reconstruction, or several per launch).
struct Choice {
    const TileVariant *col = nullptr, *row = nullptr;
    float col_us = 0, row_us = 0;
};
// plain_rows: only row variants that are not persistent (the ones that
// carry the transmission constraint)
// wf: the FresnelCDI_WF passes of the plain variants (the tune file marks
// those choices with 2 in its kind column)
const Choice &choose(int nx, int ny, bool fresnel, int nslots, bool plain_rows = false,
                     bool wf = false);

// Mixed-length persistent passes (fused32_mixed.cu): one launch per pass over
// a work list of items (reconstruction index into the slot list, its column
// or row tile, length class) of Planar/Fresnel reconstructions whose column
// and row lengths both have a class.
struct alignas(16) MixItem {
    int slot, tile, cls, pad;
};
int mix_class_of(int n);   // the class of transform length n, or -1
int mix_tile(int cls);     // signals per tile of a class
int mix_len(int cls);
int mix_threads();
std::string mix_describe(int n);
int mix_ctas();            // CTAs of a mixed launch
// orders items by class and cuts them into `ctas` ranges of equal estimated work
void mix_order(std::vector<MixItem> &items, std::vector<int> &bounds, int ctas);
struct TileVariant;
const TileVariant *mix_variant(int n); // the single-length variant of n's class
void mix_prepare();        // once per device, outside graph capture
void mix_launch_col(bool fresnel, const MixItem *items, const int *bounds, int ctas,
                    const Slot *const *slots, cudaStream_t st);
void mix_launch_row(const MixItem *items, const int *bounds, int ctas, const Slot *const *slots,
                    int nslots, cudaStream_t st);

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
    // complex-constraint regions (Slot::tc_*)
    DevBuf<int> tc_region;
    DevBuf<float> tc_par, tc_cm;
    DevBuf<double> tc_part;
    DevBuf<float2> Y;
    void constrain_array(float2 *t); // the whole constraint on an array (field 2)
    DevBuf<float> sup, mI, tmp1, tmp2, maxpart;
    DevBuf<double> partials;
    DevBuf<long long> iter;
    DevBuf<int> flag;
    DevBuf<f32::Slot> slot;
    DevBuf<f32::Slot *> slot_ptr;
    f32::Slot h_slot{};
    f32::Slot slot_on_device{}; // the descriptor as last uploaded
    bool slot_uploaded = false;
    const float2 *twx = nullptr, *twy = nullptr;
    const f32::Choice *choice = nullptr;
    std::vector<double> h_bs;
    bool p_valid = false;
    // PolyCDI
    int mx = 0, my = 0, pcols = 0;
    DevBuf<float> q, wl, ratio;
    DevBuf<int> gx, gy;
    const f32::PolyVariant *pcol = nullptr, *prow = nullptr;
    // FresnelCDI_WF: the tile shapes of its column and row passes
    const f32::TileVariant *wfc = nullptr, *wfr = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    // algorithms with a PfPs term (allocated on first use): Q, its error
    // partials, the descriptor of Q's column pass, and non-persistent row
    // variants (the PfPs row pass runs in those)
    DevBuf<float2> Q;
    DevBuf<double> qpartials;
    DevBuf<f32::Slot> qslot;
    DevBuf<f32::Slot *> qslot_ptr;
    f32::Slot qslot_on_device{};
    bool qslot_uploaded = false;
    bool q_valid = false;
    const f32::Choice *pfs_choice = nullptr;
    cudaGraphExec_t graph_pfs = nullptr;

    explicit Impl(Solver &s);
    ~Impl();
    void push_slot();
    bool push_slot_async(cudaStream_t st); // false: the device copy was current
    // the variants the next launches use (the handle's own, or a batch's);
    // sets the column-block count the row pass sums over
    void use_choice(const f32::Choice *c);
    void use_ncol(int ncol) { h_slot.ncol = ncol; } // column tiles the row pass sums over
    // host arrays in the reference's order <-> device arrays in the panel
    // layout (stride 1: real, 2: complex; fold: PlanarCDI's centred detector
    // to transform order), converted on the host: plain copies on the device
    std::vector<float> stage, mstage; // host staging arrays, kept between calls
    float *staging(size_t count);
    void put_panel(const double *h, int stride, void *dst, bool fold);
    void put_panel_f(const float *h, int stride, void *dst, bool fold);
    void get_panel(const void *src, int stride, double *h);
    void get_panel_f(const void *src, int stride, float *h);
    void upload_intensity(); // marks sqrt(I) for conversion (flush_intensity)
    void flush_intensity();
    bool mI_dirty = false;
    void blur(bool cplx, const void *in, double gauss_width, int cut);
    int blur_blocks() const;
    void check_algorithm() const;
    void prime(cudaStream_t st);
    void launch_iteration(cudaStream_t st);
    bool pfs_mode() const; // the algorithm has a PfPs term (not ER)
    void prepare_pfs();
    void launch_iteration_pfs(cudaStream_t st);
    void launch_iteration_wf(cudaStream_t st);
};

} // namespace nadia
