// fft32.cuh -- single-precision tile transforms for the fused FP32 path.
//
// A CTA transforms L signals of length N held as E = N*L/NT complex values
// per thread (NT threads).  The transform is a sequence of Stockham passes
// (radix list R0..R{P-1}); in each pass a thread owns E/R butterflies, keeps
// their inputs in registers, applies the inter-pass twiddles from a table,
// runs an in-register DFT of size R and, unless it is the last pass, trades
// its outputs with the other threads through shared memory.
//
// Stockham pass p (span Ns = R0*...*R{p-1}) takes the inputs of butterfly j
// from positions j + r*N/R and sends its outputs to (j/Ns)*Ns*R + j%Ns + r*Ns.
// In the last pass (Ns = N/R) that is j + r*N/R again, so a forward transform
// that ends with radix R leaves each thread holding exactly the inputs of the
// first pass of an inverse transform that starts with radix R: the modulus
// projection (column pass) and the support update (row pass) run on
// registers between a transform and its inverse, with no extra exchange.
#pragma once

#include <cuda_runtime.h>

namespace nadia {
namespace f32 {

// ----------------------------------------------------------------- complex

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 w)
{
    return make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 w) // a * conj(w)
{
    return make_float2(a.x * w.x + a.y * w.y, a.y * w.x - a.x * w.y);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool FWD>
__device__ __forceinline__ float2 rot(float2 a)
{
    return FWD ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// ------------------------------------------------------------ small DFTs

template <int R, bool FWD>
struct Dft;

template <bool FWD>
struct Dft<2, FWD> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    }
};

template <bool FWD>
struct Dft<4, FWD> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
        float2 c = cadd(v[1], v[3]), d = rot<FWD>(csub(v[1], v[3]));
        v[0] = cadd(a, c);
        v[2] = csub(a, c);
        v[1] = cadd(b, d);
        v[3] = csub(b, d);
    }
};

template <bool FWD>
struct Dft<8, FWD> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float c8 = 0.70710678118654752f;
        float2 a[4], b[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            a[r] = cadd(v[r], v[r + 4]);
            b[r] = csub(v[r], v[r + 4]);
        }
        // b[r] *= W8^r
        b[1] = FWD ? make_float2((b[1].x + b[1].y) * c8, (b[1].y - b[1].x) * c8)
                   : make_float2((b[1].x - b[1].y) * c8, (b[1].y + b[1].x) * c8);
        b[2] = rot<FWD>(b[2]);
        b[3] = FWD ? make_float2((b[3].y - b[3].x) * c8, -(b[3].x + b[3].y) * c8)
                   : make_float2(-(b[3].x + b[3].y) * c8, (b[3].x - b[3].y) * c8);
        Dft<4, FWD>::run(a);
        Dft<4, FWD>::run(b);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            v[2 * r] = a[r];
            v[2 * r + 1] = b[r];
        }
    }
};

// 16 = 4 x 4 Cooley-Tukey: X[k1 + 4 k2] = DFT4_q( W16^(q k1) * DFT4_m(v[q + 4m])[k1] )[k2]
template <bool FWD>
struct Dft<16, FWD> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float c1 = 0.92387953251128674f; // cos(pi/8)
        const float s1 = 0.38268343236508978f; // sin(pi/8)
        const float c8 = 0.70710678118654752f;
        const float sg = FWD ? -1.f : 1.f;
        float2 a[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float2 t[4] = {v[q], v[q + 4], v[q + 8], v[q + 12]};
            Dft<4, FWD>::run(t);
#pragma unroll
            for (int k = 0; k < 4; ++k) a[q][k] = t[k];
        }
        // internal twiddles W16^(q k1), exponents q*k1 in {1,2,3,2,4,6,3,6,9}
        const float2 w1 = make_float2(c1, sg * s1);
        const float2 w2 = make_float2(c8, sg * c8);
        const float2 w3 = make_float2(s1, sg * c1);
        const float2 w6 = make_float2(-c8, sg * c8);
        const float2 w9 = make_float2(-c1, -sg * s1);
        a[1][1] = cmul(a[1][1], w1);
        a[1][2] = cmul(a[1][2], w2);
        a[1][3] = cmul(a[1][3], w3);
        a[2][1] = cmul(a[2][1], w2);
        a[2][2] = rot<FWD>(a[2][2]);
        a[2][3] = cmul(a[2][3], w6);
        a[3][1] = cmul(a[3][1], w3);
        a[3][2] = cmul(a[3][2], w6);
        a[3][3] = cmul(a[3][3], w9);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            float2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
            Dft<4, FWD>::run(t);
#pragma unroll
            for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
        }
    }
};

template <bool FWD>
struct Dft<3, FWD> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float s3 = 0.86602540378443865f; // sin(2 pi / 3)
        float2 a = v[0], b = v[1], c = v[2];
        float2 s = cadd(b, c);
        float2 d = cscale(rot<FWD>(csub(b, c)), s3);
        float2 t = make_float2(a.x - 0.5f * s.x, a.y - 0.5f * s.y);
        v[0] = cadd(a, s);
        v[1] = cadd(t, d);
        v[2] = csub(t, d);
    }
};

template <bool FWD>
struct Dft<5, FWD> {
    static __device__ __forceinline__ void run(float2 *v)
    {
        const float c1 = 0.30901699437494742f;  // cos(2 pi / 5)
        const float c2 = -0.80901699437494742f; // cos(4 pi / 5)
        const float s1 = 0.95105651629515357f;  // sin(2 pi / 5)
        const float s2 = 0.58778525229247313f;  // sin(4 pi / 5)
        float2 a = v[0];
        float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        float2 p1 = make_float2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
        float2 p2 = make_float2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
        float2 q1 = rot<FWD>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
        float2 q2 = rot<FWD>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
        v[0] = cadd(a, cadd(t1, t2));
        v[1] = cadd(p1, q1);
        v[4] = csub(p1, q1);
        v[2] = cadd(p2, q2);
        v[3] = csub(p2, q2);
    }
};

// Good-Thomas prime-factor DFT for R = A*B with gcd(A,B) = 1 (no twiddles):
// input n = (B n1 + A n2) mod R, output k with k = k1 (mod A), k = k2 (mod B),
// that is k = (k1 e1 + k2 e2) mod R with e1 = 1 (mod A), 0 (mod B) and
// e2 = 0 (mod A), 1 (mod B).  The indices are plain arithmetic on unrolled
// loop counters, so every access of v resolves to a register.
constexpr int crt_unit(int A, int B) // the multiple of B that is 1 modulo A
{
    int e = B;
    while (e % A != 1) e += B;
    return e;
}

template <int A, int B, bool FWD>
struct Pfa {
    static constexpr int E1 = crt_unit(A, B), E2 = crt_unit(B, A);
    static __device__ __forceinline__ void run(float2 *v)
    {
        constexpr int R = A * B;
        float2 t[B][A];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
            float2 u[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) u[n1] = v[(B * n1 + A * n2) % R];
            Dft<A, FWD>::run(u);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) t[n2][k1] = u[k1];
        }
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            float2 u[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) u[n2] = t[n2][k1];
            Dft<B, FWD>::run(u);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) v[(k1 * E1 + k2 * E2) % R] = u[k2];
        }
    }
};

template <bool FWD> struct Dft<6, FWD> : Pfa<2, 3, FWD> {};
template <bool FWD> struct Dft<10, FWD> : Pfa<2, 5, FWD> {};
template <bool FWD> struct Dft<12, FWD> : Pfa<4, 3, FWD> {};
template <bool FWD> struct Dft<15, FWD> : Pfa<3, 5, FWD> {};

// --------------------------------------------------------------- plans

template <int... Rs>
struct Radices {
    static constexpr bool TWD = false; // twiddles formed as products (see pass_compute)
    static constexpr int P = sizeof...(Rs);
    static constexpr int get(int p)
    {
        constexpr int a[] = {Rs...};
        return a[p];
    }
    static constexpr int prod()
    {
        int s = 1;
        for (int i = 0; i < P; ++i) s *= get(i);
        return s;
    }
    static constexpr int lcm_all()
    {
        int l = 1;
        for (int i = 0; i < P; ++i) {
            int a = l, b = get(i);
            while (b) { int t = a % b; a = b; b = t; }
            l = l / a * get(i);
        }
        return l;
    }
};

// The same radix list with every inter-pass twiddle loaded from the table
// (one load a twiddle instead of loads and products)
template <int... Rs>
struct RadicesTW : Radices<Rs...> {
    static constexpr bool TWD = true;
};

// Tile transform configuration.  MAP selects how butterflies are dealt to
// threads so that the passes touching global memory are coalesced in the
// panel layout (element (i, p) at ((p/K)*nx + i)*K + p%K):
//   kColMap: signals are K-wide groups of columns, positions run down a column;
//   kRowMap: signals are rows, positions run along the row.
enum { kColMap = 0, kRowMap = 1 };
constexpr int kPanel = 4; // panel width K

// Shared-memory address swizzle a -> a ^ ((((a >> S1) ^ (a >> S2)) & M) << SH)
// (S2 = 0: no second term), chosen per tile shape so that every exchange of
// every pass is free of bank conflicts (checked by simulating the access
// pattern of each warp).
template <int S1_, int S2_, int M_, int SH_>
struct Swizzle {
    static constexpr __host__ __device__ __forceinline__ int apply(int a)
    {
        const int t = (a >> S1_) ^ (S2_ ? (a >> S2_) : 0);
        return a ^ ((t & M_) << SH_);
    }
    // apply() is linear over GF(2) (shifts, masks and exclusive ors), so
    // where two addends have no bit in common, apply(a + b) =
    // apply(a) ^ apply(b).
    // Adding a multiple of 2^B, B above every bit the swizzle reads
    // (S1..S1+2, S2..S2+2) and writes (SH..SH+2), commutes with it:
    // apply(a + r*c) = apply(a) + r*c.
    static constexpr bool stride_commutes(int c)
    {
        const int hi = (S1_ > S2_ ? S1_ : S2_) + 3;
        return c > 0 && c % (1 << hi) == 0 && SH_ + 3 <= hi;
    }
};

// PING: exchanges alternate between two shared buffers, which saves the
// barrier between reading one pass's inputs and writing the next pass's
// outputs (a thread only overwrites a buffer after a barrier that every
// thread reaches once it has finished reading that buffer).
// GROUPS > 1: the CTA runs GROUPS independent groups of NT threads, each on
// its own tile; a group's exchanges synchronise the group alone (named
// barrier 1 + group), and its threads index butterflies by their rank in it.
template <int N_, int NT_, int L_, int MAP_, class RL, class SW, int MINB_ = 1, bool PING_ = false,
          int GROUPS_ = 1>
struct TileCfg {
    static constexpr int N = N_, NT = NT_, L = L_, MAP = MAP_, MINB = MINB_, GROUPS = GROUPS_;
    static constexpr bool PING = PING_;
    static constexpr bool TWD = RL::TWD;
    static __device__ __forceinline__ int tid() { return GROUPS > 1 ? threadIdx.x % NT : threadIdx.x; }
    static __device__ __forceinline__ void sync()
    {
        if constexpr (GROUPS > 1)
            asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)(threadIdx.x / NT)), "n"(NT) : "memory");
        else
            __syncthreads();
    }
    static constexpr int E = N * L / NT;
    static constexpr int P = RL::P;
    using Rad = RL;
    static_assert(RL::prod() == N, "radices must multiply to N");
    static_assert(N * L % NT == 0, "tile must divide over the threads");
    static_assert(E % RL::lcm_all() == 0, "every radix must divide the elements per thread");
    static_assert(MAP != kColMap || L % kPanel == 0, "a column tile covers whole panels");
    static constexpr bool rows_ok()
    {
        for (int i = 0; i < P; ++i)
            if ((N / RL::get(i)) % kPanel) return false;
        return true;
    }
    static_assert(MAP != kRowMap || rows_ok(), "row tiles need N/R divisible by the panel width");
    // radix and span of pass p in the forward (R0 first) or inverse (reversed) order
    static constexpr int radix(int p, bool fwd) { return fwd ? RL::get(p) : RL::get(P - 1 - p); }
    static constexpr int span(int p, bool fwd)
    {
        int s = 1;
        for (int i = 0; i < p; ++i) s *= radix(i, fwd);
        return s;
    }
    // shared-memory words (float2)
    static constexpr int smem_words() { return N * L * (PING ? 2 : 1); }
    static __device__ __forceinline__ int sidx(int s, int pos) { return SW::apply(pos * L + s); }
    using Swz = SW;
    // butterfly beta of a pass whose signals hold NR = N/R butterflies
    static __device__ __forceinline__ void map(int beta, int NR, int &s, int &j)
    {
        if (MAP == kColMap) {
            int lo = beta % kPanel;
            int rest = beta / kPanel;
            j = rest % NR;
            s = (rest / NR) * kPanel + lo;
        } else {
            int kk = beta % kPanel;
            s = (beta / kPanel) % L;
            j = (beta / (kPanel * L)) * kPanel + kk;
        }
    }
};

constexpr bool pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

// An exchange address (p + r*Nr)*L + s with p < Nr, s < L and r < R splits
// into addends with no common bit (p*L + s below Nr*L, r*Nr*L at and above
// it, below Nr*L*R) when Nr*L and R are powers of two; the swizzled address
// is then the swizzle of the first addend, once per butterfly, XOR the
// swizzle of the second, a constant.
template <int R, int STRIDE>
constexpr bool xor_split() { return pow2(R) && pow2(STRIDE); }

constexpr int hibit(int r)
{
    int h = 1;
    while (h * 2 <= r) h *= 2;
    return h;
}

// twiddle of pass (k, r, N/(Ns*R)): table W[t] = exp(-2 pi i t / N)
template <bool FWD>
__device__ __forceinline__ float2 twiddle(const float2 *__restrict__ tw, int t)
{
    float2 w = __ldg(&tw[t]);
    if (!FWD) w.y = -w.y;
    return w;
}

// Pass p of direction FWD on the values in v (butterfly inputs in order).
template <class C, bool FWD, int p>
__device__ __forceinline__ void pass_compute(float2 (&v)[C::E], const float2 *__restrict__ tw)
{
    constexpr int R = C::radix(p, FWD);
    constexpr int Ns = C::span(p, FWD);
    constexpr int NR = C::N / R;
    constexpr int B = C::E / R;
    constexpr int TSTEP = C::N / (Ns * R);
#pragma unroll
    for (int q = 0; q < B; ++q) {
        if (Ns > 1) {
            int s, j;
            C::map(C::tid() + q * C::NT, NR, s, j);
            const int t1 = (j % Ns) * TSTEP;
            if constexpr (C::TWD) {
                // every W^(t1*r) from the table (t1*r < N)
                float2 w[R];
#pragma unroll
                for (int r = 1; r < R; ++r) w[r] = twiddle<FWD>(tw, t1 * r);
#pragma unroll
                for (int r = 1; r < R; ++r) v[q * R + r] = cmul(v[q * R + r], w[r]);
                Dft<R, FWD>::run(&v[q * R]);
                continue;
            }
            // W^(t1*r) applied as formed: W^t1 is loaded and squared/cubed for
            // r = 1..3; W^(4a t1) is loaded for each group of four and
            // multiplied by those (at most two products per twiddle, few
            // registers live)
            const float2 w1 = twiddle<FWD>(tw, t1);
            float2 wb[4];
            wb[1] = w1;
            if (R > 2) wb[2] = cmul(w1, w1);
            if (R > 3) wb[3] = cmul(wb[2], w1);
#pragma unroll
            for (int r = 1; r < (R < 4 ? R : 4); ++r) v[q * R + r] = cmul(v[q * R + r], wb[r]);
#pragma unroll
            for (int a = 4; a < R; a += 4) {
                const float2 wa = twiddle<FWD>(tw, t1 * a);
                v[q * R + a] = cmul(v[q * R + a], wa);
#pragma unroll
                for (int b = 1; b < 4; ++b)
                    if (a + b < R) v[q * R + a + b] = cmul(v[q * R + a + b], cmul(wa, wb[b]));
            }
        }
        Dft<R, FWD>::run(&v[q * R]);
    }
}

// After pass p: write outputs to shared memory, then load the inputs of pass
// p+1.  PING tiles alternate between two buffers (sm0 after even passes, sm1
// after odd ones).
template <class C, bool FWD, int p>
__device__ __forceinline__ void pass_exchange(float2 (&v)[C::E], float2 *sm0, float2 *sm1)
{
    float2 *sm = (C::PING && (p & 1)) ? sm1 : sm0;
    constexpr int R = C::radix(p, FWD);
    constexpr int Ns = C::span(p, FWD);
    constexpr int NR = C::N / R;
    constexpr int B = C::E / R;
    constexpr int WSTRIDE = Ns * C::L;
#pragma unroll
    for (int q = 0; q < B; ++q) {
        int s, j;
        C::map(C::tid() + q * C::NT, NR, s, j);
        const int base = (j / Ns) * Ns * R + (j % Ns);
        if constexpr (C::Swz::stride_commutes(WSTRIDE)) {
            const int a0 = C::sidx(s, base);
#pragma unroll
            for (int r = 0; r < R; ++r) sm[a0 + r * WSTRIDE] = v[q * R + r];
        } else if constexpr (xor_split<R, WSTRIDE>()) {
            // base = (j/Ns)*Ns*R + j%Ns: (base*L + s) has no bit in common
            // with r*Ns*L (j%Ns*L + s < Ns*L; (j/Ns)*Ns*R*L a multiple of Ns*L*R)
            const int a0 = C::sidx(s, base);
#pragma unroll
            for (int r = 0; r < R; ++r) sm[a0 ^ C::Swz::apply(r * WSTRIDE)] = v[q * R + r];
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) sm[C::sidx(s, base + r * Ns)] = v[q * R + r];
        }
    }
    C::sync();
    constexpr int R2 = C::radix(p + 1, FWD);
    constexpr int NR2 = C::N / R2;
    constexpr int B2 = C::E / R2;
    constexpr int RSTRIDE = NR2 * C::L;
#pragma unroll
    for (int q = 0; q < B2; ++q) {
        int s, j;
        C::map(C::tid() + q * C::NT, NR2, s, j);
        if constexpr (C::Swz::stride_commutes(RSTRIDE)) {
            const int a0 = C::sidx(s, j);
#pragma unroll
            for (int r = 0; r < R2; ++r) v[q * R2 + r] = sm[a0 + r * RSTRIDE];
        } else if constexpr (xor_split<R2, RSTRIDE>()) {
            const int a0 = C::sidx(s, j); // j < NR2: j*L + s < NR2*L
#pragma unroll
            for (int r = 0; r < R2; ++r) v[q * R2 + r] = sm[a0 ^ C::Swz::apply(r * RSTRIDE)];
        } else {
#pragma unroll
            for (int r = 0; r < R2; ++r) v[q * R2 + r] = sm[C::sidx(s, j + r * NR2)];
        }
    }
    if (!C::PING) C::sync();
}

// The whole transform; before_last() runs right before the last pass's
// arithmetic (after its inputs have arrived), where a caller can start loads
// that the values leaving the transform will need.
template <class C, bool FWD, int p = 0, class H>
__device__ __forceinline__ void transform_h(float2 (&v)[C::E], float2 *sm0, float2 *sm1,
                                            const float2 *__restrict__ tw, H &&before_last)
{
    if constexpr (p + 1 == C::P) before_last();
    pass_compute<C, FWD, p>(v, tw);
    if constexpr (p + 1 < C::P) {
        pass_exchange<C, FWD, p>(v, sm0, sm1);
        transform_h<C, FWD, p + 1>(v, sm0, sm1, tw, before_last);
    }
}

template <class C, bool FWD>
__device__ __forceinline__ void transform(float2 (&v)[C::E], float2 *sm, const float2 *__restrict__ tw)
{
    transform_h<C, FWD>(v, sm, sm + C::N * C::L, tw, [] {});
}

// Visit the (signal, position) of every value a thread holds at the input of
// the first pass (FIRST=true) or at the output of the last pass of direction FWD.
template <class C, bool FWD, bool FIRST, class F>
__device__ __forceinline__ void for_each_slot(F &&f)
{
    constexpr int R = FIRST ? C::radix(0, FWD) : C::radix(C::P - 1, FWD);
    constexpr int NR = C::N / R;
    constexpr int B = C::E / R;
#pragma unroll
    for (int q = 0; q < B; ++q) {
        int s, j;
        C::map(C::tid() + q * C::NT, NR, s, j);
#pragma unroll
        for (int r = 0; r < R; ++r) f(q * R + r, s, j + r * NR);
    }
}

} // namespace f32
} // namespace nadia
