// DST-I / DCT-I row transforms through a shared-memory FFT, in float64, or
// in float32 for the float32-transform precision (one kernel template,
// fft_rows_kernel<T, Tin, Tout>: arithmetic in T, rows read as Tin and
// written as Tout).
//
// The reference realises its transforms with padded real FFTs
// (lcode.py:124-141 dst2d, 190-212 mix2d, 295-313 dct2d). Here every 1-D
// transform is one length-P complex FFT, P = 2 (N - 1), of the symmetric
// (DCT-I) or antisymmetric (DST-I) extension of a row, with TWO rows packed
// as real and imaginary parts:
//     DCT-I: Z = Y_a + i Y_b, Y real         -> X_a = Re Z[k],  X_b = Im Z[k]
//     DST-I: Z = -i X_a + X_b (Y imaginary)   -> X_a = -Im Z[k+1], X_b = Re Z[k+1]
// (unnormalised, the conventions of scipy's dct/dst type 1, so DST-I = S2 x
// and DCT-I = C x of the dense-transform form). The FFT is an
// in-place decimation-in-frequency FFT with mixed radices 8, 4, 2, 3, 5 in
// shared memory (P = 1280: 8, 8, 4, 5), read out in digit-reversed order
// through a position-sorted list. The kernel is persistent: a CTA loops over
// groups of rows and copies the next group's rows into a staging area with
// cp.async while the current group's passes run. Every launch transforms rows
// and writes its output TRANSPOSED (out[k][r]), optionally scaled on output
// by Lambda[k][r]; the 2-D solve F = L (Lambda o (L X R)) R is then four
// such passes:
//     A: rows of X by the axis-1 transform                 -> T1^T
//     B: rows of T1^T by the axis-0 transform, times Lambda -> Lambda o Z
//     C: rows of Lambda o Z by the axis-1 transform        -> T3^T
//     D: rows of T3^T by the axis-0 transform              -> F
// (Lambda on B's output rather than C's input: the multiply is the same,
// and no Lambda rows take staging space, which keeps 3 CTAs per SM.)
// One launch covers all fields of a solve; launches are programmatic
// dependent launches (the kernel waits for its predecessor on the device).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lc3d_internal.cuh"

namespace {

#ifndef LC3D_FFT_THREADS
#define LC3D_FFT_THREADS 256
#endif
#ifndef LC3D_FFT_PER_CTA
#define LC3D_FFT_PER_CTA 2
#endif
constexpr int FFT_THREADS = LC3D_FFT_THREADS;
constexpr int FFT_PER_CTA = LC3D_FFT_PER_CTA;   // complex FFTs per CTA (1 or 2; two rows each)
constexpr int ROWS_PER_CTA = 2 * FFT_PER_CTA;
static_assert(FFT_PER_CTA == 1 || FFT_PER_CTA == 2, "one or two FFTs per CTA");
static_assert(FFT_THREADS % 32 == 0 && FFT_THREADS <= 1024, "whole warps");
#ifndef LC3D_FFT_MAX_RADIX
#define LC3D_FFT_MAX_RADIX 8              // largest power-of-two butterfly in a plan (8 or 4)
#endif
#ifndef LC3D_FFT_MIN_BLOCKS
#define LC3D_FFT_MIN_BLOCKS 3             // resident CTAs per SM the registers allow (float64)
#endif
#ifndef LC3D_FFT32_SU
#define LC3D_FFT32_SU 8                   // readout entries per thread and round (float32 transforms)
#endif
#ifndef LC3D_FFT32_MIN_BLOCKS
#define LC3D_FFT32_MIN_BLOCKS 5           // ... (float32 transforms)
#endif
constexpr int MAX_RADICES = 24;
#ifndef LC3D_FFT_CLOCKS
#define LC3D_FFT_CLOCKS 0                 // instrumented builds: per-CTA phase clocks of the last launch
#endif
#if LC3D_FFT_CLOCKS
constexpr int FFT_NCLK = 8;               // wait, extension, four radix passes, readout, partial sums
__device__ long long g_fft_clocks[4096][FFT_NCLK];
#define FFT_CLK(k)                                        \
    do {                                                  \
        const long long t_ = clock64();                   \
        clk[(k) < FFT_NCLK ? (k) : FFT_NCLK - 1] += t_ - clk_last; \
        clk_last = t_;                                    \
    } while (0)
#else
#define FFT_CLK(k) \
    do {           \
    } while (0)
#endif
constexpr int FFT_PAD = 4;               // complex words between the CTA's two FFTs (bank offset)

struct FftField {
    const void* in;                      // Tin rows
    int ld_in, rows, type;               // type: 0 DCT-I (n = N), 1 DST-I (n = N - 2)
    void* out;                           // Tout
    int ld_out;
    const void* lam;                     // T: out[k][r] *= lam[k ld_lam + r], or NULL
    int ld_lam;
    double* partial;                     // per-CTA sums of the written values, or NULL
    int cta_start;
};

struct FftBatch {
    FftField f[6];
    int count, P, N;
    int nrad;
    int rad[MAX_RADICES];
    int ngroups;                         // row groups (ROWS_PER_CTA rows) over all fields
    const double2* tw;                   // tw[m] = exp(-2 pi i m / P)
    const float2* tw32;                  // the same rounded to float
    const int* rd;                       // readout lists: DCT-I (N entries), then DST-I (N - 2)
};

// Complex values of the transform arithmetic: double2 (float64 solves) or
// float2 (float32-transform solves).
template <typename V> struct ReOf;
template <> struct ReOf<double2> { using type = double; };
template <> struct ReOf<float2> { using type = float; };
template <typename T> struct CxOf;
template <> struct CxOf<double> { using type = double2; };
template <> struct CxOf<float> { using type = float2; };

template <typename V>
__device__ __forceinline__ V cmk(typename ReOf<V>::type a, typename ReOf<V>::type b) {
    V r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename V>
__device__ __forceinline__ V cmul(V a, V b) {
    return cmk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V>
__device__ __forceinline__ V cadd(V a, V b) { return cmk<V>(a.x + b.x, a.y + b.y); }
template <typename V>
__device__ __forceinline__ V csub(V a, V b) { return cmk<V>(a.x - b.x, a.y - b.y); }
// x -> -i x
template <typename V>
__device__ __forceinline__ V mul_mi(V a) { return cmk<V>(a.y, -a.x); }
template <typename V>
__device__ __forceinline__ V cscale(V a, typename ReOf<V>::type s) { return cmk<V>(a.x * s, a.y * s); }

// Where a pass's twiddles come from. Float64 passes read a per-CTA shared
// copy: the small-DFT constants dc[0..2] (exp(-2 pi i / 3), exp(-2 pi i / 5),
// its square), then one segment per pass, seg[k] = exp(-2 pi i k / (R span)),
// k < span (transforms 0.327 -> 0.319 ms per step at 641^2). Float32 passes
// read the constant global table through the read-only cache, which measured
// faster for them (0.234 against 0.238 ms per step).
template <typename V, bool SHARED> struct Twiddles;
template <typename V> struct Twiddles<V, true> {
    const V* dc;
    const V* seg;
    __device__ __forceinline__ V c(int i) const { return dc[i]; }
    __device__ __forceinline__ V w(int k) const { return seg[k]; }
};
template <typename V> struct Twiddles<V, false> {
    const V* tw;   // tw[m] = exp(-2 pi i m / P)
    int P, tstep;
    __device__ __forceinline__ V c(int i) const { return __ldg(tw + (i == 0 ? P / 3 : i * (P / 5))); }
    __device__ __forceinline__ V w(int k) const { return __ldg(tw + k * tstep); }
};

// Small DFTs in registers, forward sign, R = 2, 3, 4, 5, 8.
//  3: W = exp(-2 pi i / 3) = (c, -s) = tw.c(0) (see Twiddles).
//  5: W = (c1, -s1) = tw.c(1), W^2 = (c2, -s2) = tw.c(2);
//     X1,4 = v0 + c1 t1 + c2 t2 -+ i (s1 t3 + s2 t4),
//     X2,3 = v0 + c2 t1 + c1 t2 -+ i (s2 t3 - s1 t4),
//     t1 = v1 + v4, t2 = v2 + v3, t3 = v1 - v4, t4 = v2 - v3.
//  8: 2 x 4, a_j = v_j + v_{j+4}, b_j = (v_j - v_{j+4}) W8^j,
//     X_2k = DFT4(a)_k, X_2k+1 = DFT4(b)_k. Outputs are left in register
//     order (X_0 X_2 X_4 X_6 X_1 X_3 X_5 X_7); dft_out<8> maps register ->
//     frequency. W8 = sqrt(1/2) (1 - i), W8^2 = -i, W8^3 = -sqrt(1/2) (1 + i):
//     no table loads, two real products each for j = 1, 3.
template <int R, typename V, typename TW>
__device__ __forceinline__ void dft(V (&v)[R], const TW& tw) {
    using T = typename ReOf<V>::type;
    static_assert(R == 2 || R == 3 || R == 4 || R == 5 || R == 8, "radix 2, 3, 4, 5 or 8");
    if constexpr (R == 2) {
        const V a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 3) {
        const V w = tw.c(0);
        const V t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
        const V a = cadd(v[0], cscale(t1, w.x));
        const V bb = cscale(t2, -w.y);
        v[0] = cadd(v[0], t1);
        v[1] = cadd(a, mul_mi(bb));
        v[2] = csub(a, mul_mi(bb));
    } else if constexpr (R == 4) {
        const V a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        const V a2 = cadd(v[1], v[3]);
        const V a3 = mul_mi(csub(v[1], v[3]));   // -i (v1 - v3)
        v[0] = cadd(a0, a2);
        v[2] = csub(a0, a2);
        v[1] = cadd(a1, a3);
        v[3] = csub(a1, a3);
    } else if constexpr (R == 5) {
        const V w1 = tw.c(1), w2 = tw.c(2);
        const T c1 = w1.x, s1 = -w1.y, c2 = w2.x, s2 = -w2.y;
        const V t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const V t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const V a1 = cadd(v[0], cadd(cscale(t1, c1), cscale(t2, c2)));
        const V a2 = cadd(v[0], cadd(cscale(t1, c2), cscale(t2, c1)));
        const V b1 = cadd(cscale(t3, s1), cscale(t4, s2));
        const V b2 = csub(cscale(t3, s2), cscale(t4, s1));
        v[0] = cadd(v[0], cadd(t1, t2));
        v[1] = cadd(a1, mul_mi(b1));
        v[4] = csub(a1, mul_mi(b1));
        v[2] = cadd(a2, mul_mi(b2));
        v[3] = csub(a2, mul_mi(b2));
    } else {
        constexpr T h = (T)0.70710678118654752440;
        V a[4], b[4], d[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a[j] = cadd(v[j], v[j + 4]);
            d[j] = csub(v[j], v[j + 4]);
        }
        b[0] = d[0];
        b[1] = cmk<V>(h * (d[1].x + d[1].y), h * (d[1].y - d[1].x));
        b[2] = mul_mi(d[2]);
        b[3] = cmk<V>(h * (d[3].y - d[3].x), -h * (d[3].x + d[3].y));
        dft<4>(a, tw);
        dft<4>(b, tw);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            v[j] = a[j];
            v[j + 4] = b[j];
        }
    }
}

// Frequency held in register r after dft<R>.
template <int R>
__device__ __forceinline__ constexpr int dft_out(int r) {
    return R == 8 ? (r < 4 ? 2 * r : 2 * (r - 4) + 1) : r;
}

// One in-place decimation-in-frequency butterfly of radix R inside a
// sub-transform of length Lr = R * span: the R inputs A[base + r span] are
// transformed and output m is scaled by exp(-2 pi i m k / Lr), k the
// position inside the span, and written back in place. After all passes
// frequency k = m0 + R0 (m1 + R1 (m2 + ...)) sits at sum_s m_s P / (R0..Rs).
//
// The twiddles w^m, w = exp(-2 pi i k / Lr), are one table load (tw.w(k))
// and a product tree w^m = w^(m/2) w^(m - m/2) (at most three roundings deep
// for R <= 8), which keeps the R - 1 scattered table loads off the L1 pipe.
template <int R, typename V, typename TW>
__device__ __forceinline__ void dif_butterfly(V* A, int b, int span, float inv_span, const TW& tw) {
    // g = b / span: (b + 0.5) / span lies at least 0.5 / span from an
    // integer, far more than the float rounding for b, span < 2^16
    const int g = __float2int_rz(((float)b + 0.5f) * inv_span), k = b - g * span;
    const int base = g * span * R + k;
    V v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = A[base + r * span];
    V w[R];
    w[1] = tw.w(k);
#pragma unroll
    for (int m = 2; m < R; ++m) w[m] = cmul(w[m / 2], w[m - m / 2]);
    dft<R>(v, tw);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int m = dft_out<R>(r);   // frequency in register r
        A[base + m * span] = m ? cmul(v[r], w[m]) : v[r];
    }
}

template <int R, typename V, typename TW>
__device__ __forceinline__ void fft_pass(V* A, int span, int P, const TW& tw) {
    const int nb = P / R;
    const float inv_span = 1.0f / (float)span;
    for (int t = threadIdx.x; t < FFT_PER_CTA * nb; t += FFT_THREADS) {
        const int q = FFT_PER_CTA == 2 && t >= nb, j = t - q * nb;
        dif_butterfly<R>(A + q * (P + FFT_PAD), j, span, inv_span, tw);
    }
}

// Entries of the CTA's shared twiddle table (float64 passes): the three
// small-DFT constants, then one segment per pass of span entries.
__host__ __device__ constexpr int fft_twiddle_entries(int P, const int* rad, int nrad) {
    int n = 3, span = P;
    for (int p = 0; p < nrad; ++p) {
        span /= rad[p];
        n += span;
    }
    return n;
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src) {
    static_assert(BYTES == 4 || BYTES == 8, "4- or 8-byte copies");
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    if constexpr (BYTES == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ int field_of(const FftBatch& b, int g) {
    int fi = 0;
#pragma unroll 1
    for (int q = 1; q < b.count; ++q)
        if (g >= b.f[q].cta_start) fi = q;
    return fi;
}

// Start copying row group g (ROWS_PER_CTA rows) into the staging area, one
// cp.async per element (rows need not be 16-byte aligned); rows past the
// field are not copied (the reader uses 0).
template <typename Tin>
__device__ __forceinline__ void stage_group(const FftBatch& b, int g, Tin* stg) {
    const FftField& F = b.f[field_of(b, g)];
    const int n = F.type ? b.N - 2 : b.N;
    const int r0 = (g - F.cta_start) * ROWS_PER_CTA;
#pragma unroll
    for (int rr = 0; rr < ROWS_PER_CTA; ++rr) {
        const int row = r0 + rr;
        if (row >= F.rows) continue;
        const Tin* rp = static_cast<const Tin*>(F.in) + (size_t)row * F.ld_in;
        for (int j = threadIdx.x; j < n; j += FFT_THREADS) cp_async<sizeof(Tin)>(stg + rr * b.N + j, rp + j);
    }
    cp_async_commit();
}

// Resident CTAs per SM the register budget is sized for: float64 butterflies
// need twice the registers of float32 ones.
template <typename T>
constexpr int fft_min_blocks() { return sizeof(T) == 8 ? LC3D_FFT_MIN_BLOCKS : LC3D_FFT32_MIN_BLOCKS; }

// Persistent: CTA i transforms row groups i, i + gridDim.x, ...; the rows
// of the next group are copied into the staging area (cp.async) while the
// current group's FFT passes run, so the global-load latency of a group is
// hidden behind the previous group's work. Arithmetic in T; rows read as
// Tin and written as Tout.
template <typename T, typename Tin, typename Tout>
__global__ void __launch_bounds__(FFT_THREADS, fft_min_blocks<T>()) fft_rows_kernel(const __grid_constant__ FftBatch b) {
    using V = typename CxOf<T>::type;
    // FFT q at q (P + FFT_PAD); the twiddle table; the staging rows
    extern __shared__ __align__(16) unsigned char fft_smem[];
    const int P = b.P, L = P / 2, PS = P + FFT_PAD;
    V* A = reinterpret_cast<V*>(fft_smem);
    constexpr bool SHARED_TW = sizeof(T) == 8;
    V* tws = A + FFT_PER_CTA * PS;
    Tin* stg = reinterpret_cast<Tin*>(tws + (SHARED_TW ? fft_twiddle_entries(P, b.rad, b.nrad) : 0));   // [ROWS_PER_CTA][N]
    const V* tw = reinterpret_cast<const V*>(sizeof(T) == 8 ? static_cast<const void*>(b.tw)
                                                            : static_cast<const void*>(b.tw32));
    if (SHARED_TW) {   // the twiddles of every pass, from the constant table (written at set-up,
                       // so read before the dependency wait); first used after the next barrier
        if (threadIdx.x < 3) {
            const int m = threadIdx.x == 0 ? (P % 3 ? 0 : P / 3) : (P % 5 ? 0 : threadIdx.x * (P / 5));
            tws[threadIdx.x] = __ldg(tw + m);
        }
        int off = 3, span = P;
        for (int p = 0; p < b.nrad; ++p) {
            span /= b.rad[p];
            const int tstep = P / (span * b.rad[p]);
            for (int k = threadIdx.x; k < span; k += FFT_THREADS) tws[off + k] = __ldg(tw + k * tstep);
            off += span;
        }
    }
#if LC3D_FFT_CLOCKS
    long long clk[FFT_NCLK] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long clk_last = clock64();
#endif
    pdl_wait();
    int g = blockIdx.x;
    if (g < b.ngroups) stage_group(b, g, stg);
#pragma unroll 1
    for (; g < b.ngroups; g += gridDim.x) {
    const FftField& F = b.f[field_of(b, g)];
    const int r0 = (g - F.cta_start) * ROWS_PER_CTA;
    const int n = F.type ? b.N - 2 : b.N;     // input / output length
    cp_async_wait_all();
    __syncthreads();                     // the staging area holds group g
    FFT_CLK(0);

    // symmetric / antisymmetric extensions, rows 2q and 2q + 1 of the group
    // as the real and imaginary parts of FFT q, each staged element written
    // to its one or two positions
#pragma unroll
    for (int q = 0; q < FFT_PER_CTA; ++q) {
        V* a = A + q * PS;
        const bool ok0 = r0 + 2 * q < F.rows, ok1 = r0 + 2 * q + 1 < F.rows;
        const Tin* s0 = stg + (2 * q) * b.N;
        const Tin* s1 = s0 + b.N;
        for (int j = threadIdx.x; j < n; j += FFT_THREADS) {
            const T x0 = ok0 ? (T)s0[j] : (T)0, x1 = ok1 ? (T)s1[j] : (T)0;
            const V z = cmk<V>(x0, x1);
            if (F.type == 0) {           // m = j and P - j
                a[j] = z;
                if (j > 0 && j < L) a[P - j] = z;
            } else {                     // m = j + 1 and P - j - 1, negated
                a[j + 1] = z;
                a[P - j - 1] = cmk<V>(-z.x, -z.y);
            }
        }
    }
    if (F.type == 1 && threadIdx.x < 2 * FFT_PER_CTA)   // DST-I: zeros at m = 0 and m = L
        A[(threadIdx.x >> 1) * PS + (threadIdx.x & 1) * L] = cmk<V>((T)0, (T)0);
    __syncthreads();                     // the staging area is free: start the next group
    FFT_CLK(1);
    if (g + (int)gridDim.x < b.ngroups) stage_group(b, g + gridDim.x, stg);
    int span = P;
    const V* seg = tws + 3;
    for (int p = 0; p < b.nrad; ++p) {
        const int R = b.rad[p];
        span /= R;
        Twiddles<V, SHARED_TW> tp;
        if constexpr (SHARED_TW) {
            tp.dc = tws;
            tp.seg = seg;
        } else {
            tp.tw = tw;
            tp.P = P;
            tp.tstep = P / (span * R);
        }
        switch (R) {
#if LC3D_FFT_MAX_RADIX >= 8
            case 8: fft_pass<8>(A, span, P, tp); break;
#endif
            case 4: fft_pass<4>(A, span, P, tp); break;
            case 2: fft_pass<2>(A, span, P, tp); break;
            case 3: fft_pass<3>(A, span, P, tp); break;
            default: fft_pass<5>(A, span, P, tp); break;
        }
        seg += span;
        __syncthreads();
        FFT_CLK(2 + p);
    }
    // transposed output: out[k][row] for the CTA's rows. The readout list
    // holds (position, k) for the wanted frequencies sorted by position, so
    // a warp reads nearly consecutive shared-memory words; the threads of
    // one entry (one per FFT) write the CTA's consecutive rows of out[k]
    // (and read the same places of Lambda, when given).
    const int* rl = b.rd + (F.type ? b.N : 0);
    const T* lam = static_cast<const T*>(F.lam);
    Tout* out = static_cast<Tout*>(F.out);
    const int total = n * FFT_PER_CTA;
    // a thread's two rows of out[k] in one 16-byte store where they are
    // aligned (the padded float64 intermediates: an even pitch, rows from an
    // even row on): 0.317 -> 0.313 ms of transforms per step; the float32
    // intermediates are not padded and keep scalar stores
    using Tout2 = typename CxOf<Tout>::type;
    const bool vec_out = sizeof(Tout) == 8 && F.ld_out % 2 == 0 &&
                         (reinterpret_cast<uintptr_t>(F.out) % sizeof(Tout2)) == 0;
    double psum = 0.0;
    constexpr int SU = sizeof(T) == 8 ? 8 : LC3D_FFT32_SU;   // readout entries in flight per thread
    for (int t0 = 0; t0 < total; t0 += SU * FFT_THREADS) {
        int e[SU];
#pragma unroll
        for (int u = 0; u < SU; ++u) {
            const int t = t0 + u * FFT_THREADS + (int)threadIdx.x;
            e[u] = t < total ? __ldg(rl + t / FFT_PER_CTA) : 0;
        }
        // two halves, so that the Lambda values of only SU / 2 entries are
        // held in registers at a time
#pragma unroll
        for (int h = 0; h < SU; h += SU / 2) {
            T la[SU / 2][2];
            if (lam) {
#pragma unroll
                for (int u = 0; u < SU / 2; ++u) {
                    const int t = t0 + (h + u) * FFT_THREADS + (int)threadIdx.x;
                    const int row = r0 + 2 * (t % FFT_PER_CTA);
                    const T* lp = lam + (size_t)(e[h + u] & 0xffff) * F.ld_lam + row;
                    la[u][0] = t < total && row < F.rows ? __ldg(lp) : (T)0;
                    la[u][1] = t < total && row + 1 < F.rows ? __ldg(lp + 1) : (T)0;
                }
            }
#pragma unroll
            for (int u = 0; u < SU / 2; ++u) {
                const int t = t0 + (h + u) * FFT_THREADS + (int)threadIdx.x;
                const int q = t % FFT_PER_CTA, row = r0 + 2 * q;
                if (t >= total || row >= F.rows) continue;
                const V z = A[q * PS + (e[h + u] >> 16)];
                Tout* o = out + (size_t)(e[h + u] & 0xffff) * F.ld_out + row;
                T x0 = F.type == 0 ? z.x : -z.y, x1 = F.type == 0 ? z.y : z.x;
                if (lam) {
                    x0 *= la[u][0];
                    x1 *= la[u][1];
                }
                const Tout y0 = (Tout)x0, y1 = (Tout)x1;
                psum += (double)y0;
                if (row + 1 < F.rows) {
                    psum += (double)y1;
                    if (sizeof(Tout) == 8 && vec_out) {
                        Tout2 y;
                        y.x = y0;
                        y.y = y1;
                        *reinterpret_cast<Tout2*>(o) = y;
                    } else {
                        o[0] = y0;
                        o[1] = y1;
                    }
                } else {
                    o[0] = y0;
                }
            }
        }
    }
    FFT_CLK(6);
    if (F.partial) {   // uniform per CTA: fixed-order sum of everything this CTA wrote
        __syncthreads();   // the FFT buffer is free
        double* red = reinterpret_cast<double*>(fft_smem);
        double v = psum;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {   // the warps' sums in warp order
            double t = 0.0;
            for (int w = 0; w < FFT_THREADS / 32; ++w) t += red[w];
            F.partial[g - F.cta_start] = t;
        }
    }
    __syncthreads();                     // the FFT buffer is free for the next group
    FFT_CLK(7);
    }
    cp_async_wait_all();                 // nothing left in flight (no group was started past the end)
#if LC3D_FFT_CLOCKS
    if (threadIdx.x == 0 && blockIdx.x < 4096)
        for (int k = 0; k < FFT_NCLK; ++k) g_fft_clocks[blockIdx.x][k] = clk[k];
#endif
}

double sin_pi_frac(long long r, long long L) {
    r %= 2 * L;
    if (r < 0) r += 2 * L;
    double sign = 1;
    if (r >= L) { r -= L; sign = -1; }
    if (2 * r > L) r = L - r;
    return sign * std::sin(M_PI * (double)r / (double)L);
}

}  // namespace

// Radix plan for a length-P FFT: factors 8, 4, 2, 3, 5 (largest powers of
// two first, each a register butterfly).
// Returns the number of passes, or 0 if P has another prime factor (the
// dense transform form is used then).
int fft_plan(int P, int* rad) {
    int n = 0;
    int r = P;
    const int others[] = {8, 4, 2, 3, 5};
    for (int f : others)
        while ((f <= LC3D_FFT_MAX_RADIX || f % 2) && r % f == 0 && n < MAX_RADICES) { rad[n++] = f; r /= f; }
    return (r == 1) ? n : 0;
}

int fft_cta_rows() { return ROWS_PER_CTA; }

// Dynamic shared memory of fft_rows_kernel, the layout the kernel uses: the
// FFT buffers at a pitch of P + FFT_PAD complex words, the twiddle table
// (float64 passes), then the staging rows (ROWS_PER_CTA x N input elements).
size_t fft_cta_smem_bytes(int P, int N, int types) {
    const size_t cx = types == FFT_F64 ? sizeof(double2) : sizeof(float2);
    const size_t in = (types == FFT_F64 || types == FFT_F64_F32) ? sizeof(double) : sizeof(float);
    int rad[MAX_RADICES];
    const int nrad = fft_plan(P, rad);
    return ((size_t)FFT_PER_CTA * (P + FFT_PAD) + (types == FFT_F64 ? fft_twiddle_entries(P, rad, nrad) : 0)) * cx +
           (size_t)ROWS_PER_CTA * N * in;
}

// Layout of the twiddle buffer (in doubles): P double2 twiddles, the two
// readout lists (2 N - 2 int32), then the P float2 twiddles.
size_t fft_tw32_offset(int P, int N) { return 2 * (size_t)P + (size_t)(2 * N - 2 + 1) / 2; }

template <typename T, typename Tin, typename Tout>
constexpr int fft_types() {
    return sizeof(T) == 8 ? FFT_F64 : sizeof(Tin) == 8 ? FFT_F64_F32 : sizeof(Tout) == 8 ? FFT_F32_F64 : FFT_F32;
}

// Persistent grid of an instantiation: as many CTAs as fit on the device at
// once (queried once per context, at set-up).
template <typename T, typename Tin, typename Tout>
int fft_grid_size(int P, int N, int* grid) {
    int dev = 0, sms = 0, per_sm = 0;
    LC3D_CUDA_TRY(cudaGetDevice(&dev));
    LC3D_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    LC3D_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fft_rows_kernel<T, Tin, Tout>, FFT_THREADS,
                                                                fft_cta_smem_bytes(P, N, fft_types<T, Tin, Tout>())));
    *grid = std::max(1, sms * std::max(per_sm, 1));
    return LC3D_OK;
}

template <typename T, typename Tin, typename Tout>
int fft_launch(const FftBatch& b, int G, cudaStream_t s) {
    const size_t smem = fft_cta_smem_bytes(b.P, b.N, fft_types<T, Tin, Tout>());
    const int grid = std::max(1, std::min(b.ngroups, G));
    LC3D_CUDA_TRY(launch_pdl(fft_rows_kernel<T, Tin, Tout>, dim3(grid), dim3(FFT_THREADS), smem, s, b));
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int fft_init(lc3d_ctx* c) {
    const int N = c->N, P = 2 * (N - 1);
    int rad[MAX_RADICES];
    c->fft_ok = fft_plan(P, rad) > 0 && fft_cta_smem_bytes(P, N, FFT_F64) <= 200 * 1024;
    if (!c->fft_ok) return LC3D_OK;
    LC3D_TRY(fft_prepare(P));
    {
        int dev = 0;
        LC3D_CUDA_TRY(cudaGetDevice(&dev));
        LC3D_CUDA_TRY(cudaDeviceGetAttribute(&c->fft_sms, cudaDevAttrMultiProcessorCount, dev));
    }
    LC3D_TRY((fft_grid_size<double, double, double>(P, N, &c->fft_grid[FFT_F64])));
    LC3D_TRY((fft_grid_size<float, double, float>(P, N, &c->fft_grid[FFT_F64_F32])));
    LC3D_TRY((fft_grid_size<float, float, float>(P, N, &c->fft_grid[FFT_F32])));
    LC3D_TRY((fft_grid_size<float, float, double>(P, N, &c->fft_grid[FFT_F32_F64])));
    const int nrad = fft_plan(P, rad);
    // P twiddles exp(-2 pi i m / P), then the two readout lists. Frequency k
    // of the in-place DIF output sits at pos(k) = sum_s m_s P / (R0..Rs) for
    // the mixed-radix digits k = m0 + R0 (m1 + R1 (...)); a list holds
    // (pos << 16) | output index for the frequencies a transform keeps
    // (DCT-I: k = 0 .. N-1 -> output k; DST-I: k = 1 .. N-2 -> output k - 1),
    // sorted by position.
    auto pos = [&](int k) {
        int p = 0, rem = P;
        for (int s = 0; s < nrad; ++s) {
            const int m = k % rad[s];
            k /= rad[s];
            rem /= rad[s];
            p += m * rem;
        }
        return p;
    };
    // P <= 6400 under the shared-memory limit above: positions fit 16 bits
    std::vector<int32_t> rd;
    for (int type = 0; type < 2; ++type) {
        std::vector<int32_t> l;
        const int n = type ? N - 2 : N;
        for (int o = 0; o < n; ++o) l.push_back((pos(o + type) << 16) | o);
        std::sort(l.begin(), l.end());
        rd.insert(rd.end(), l.begin(), l.end());
    }
    const size_t o32 = fft_tw32_offset(P, N);
    std::vector<double> buf(o32 + (size_t)P);
    float* tw32 = reinterpret_cast<float*>(buf.data() + o32);
    for (int m = 0; m < P; ++m) {
        buf[2 * m] = sin_pi_frac(4LL * m + P, 2LL * P);      // cos(pi (2m) / P)
        buf[2 * m + 1] = -sin_pi_frac(2LL * m, (long long)P);
        tw32[2 * m] = (float)buf[2 * m];
        tw32[2 * m + 1] = (float)buf[2 * m + 1];
    }
    memcpy(buf.data() + 2 * (size_t)P, rd.data(), rd.size() * sizeof(int32_t));
    LC3D_CUDA_TRY(cudaMalloc(&c->fft_tw, buf.size() * sizeof(double)));
    LC3D_CUDA_TRY(cudaMemcpy(c->fft_tw, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice));
    return LC3D_OK;
}

#if LC3D_FFT_CLOCKS
// Instrumented builds only: phase clocks (summed over the CTA's row groups)
// of the last fft_rows_kernel launch, [4096][FFT_NCLK] cycles, thread 0.
extern "C" int lc3d_debug_fft_clocks(long long* host) {
    LC3D_CUDA_TRY(cudaDeviceSynchronize());
    LC3D_CUDA_TRY(cudaMemcpyFromSymbol(host, g_fft_clocks, sizeof(g_fft_clocks)));
    return LC3D_OK;
}
#endif

int fft_prepare(int P) {
    // the limit is per kernel, not per context: always the largest size any
    // context may use (contexts of different grid sizes coexist in batches)
    (void)P;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    LC3D_CUDA_TRY(cudaFuncSetAttribute(fft_rows_kernel<double, double, double>, a, 200 * 1024));
    LC3D_CUDA_TRY(cudaFuncSetAttribute(fft_rows_kernel<float, double, float>, a, 200 * 1024));
    LC3D_CUDA_TRY(cudaFuncSetAttribute(fft_rows_kernel<float, float, float>, a, 200 * 1024));
    LC3D_CUDA_TRY(cudaFuncSetAttribute(fft_rows_kernel<float, float, double>, a, 200 * 1024));
    return LC3D_OK;
}

// One transform pass over up to 6 fields: desc[f] = {in, ld_in, rows, type,
// out, ld_out, lam, ld_lam}; rows of `in` are transformed and written
// transposed into `out`. `types` (FFT_*) gives the element types of the
// rows read and written and of the arithmetic.
int fft_rows(lc3d_ctx* c, const FftRowsDesc* desc, int count, int types, cudaStream_t s) {
    FftBatch b{};
    memset(&b, 0, sizeof(b));
    b.P = 2 * (c->N - 1);
    b.N = c->N;
    b.nrad = fft_plan(b.P, b.rad);
    b.tw = reinterpret_cast<const double2*>(c->fft_tw);
    b.rd = reinterpret_cast<const int*>(c->fft_tw + 2 * (size_t)b.P);
    b.tw32 = reinterpret_cast<const float2*>(c->fft_tw + fft_tw32_offset(b.P, b.N));
    int ctas = 0;
    for (int q = 0; q < count; ++q) {
        FftField& f = b.f[b.count++];
        f.in = desc[q].in; f.ld_in = desc[q].ld_in; f.rows = desc[q].rows; f.type = desc[q].type;
        f.out = desc[q].out; f.ld_out = desc[q].ld_out; f.lam = desc[q].lam; f.ld_lam = desc[q].ld_lam;
        f.partial = desc[q].partial;
        f.cta_start = ctas;
        ctas += (f.rows + ROWS_PER_CTA - 1) / ROWS_PER_CTA;
    }
    if (!ctas) return LC3D_OK;
    b.ngroups = ctas;
    if (types < 0 || types > 3) return LC3D_ERR_PARAM;
    // resident CTAs per SM: as many as fit, or the tile setting's cap
    int G = c->fft_grid[types];
    if (c->fft_per_sm > 0) G = std::min(G, std::max(1, c->fft_per_sm * c->fft_sms));
    ProfScope ps(c, LC3D_STAGE_TRANSFORM, s);
    switch (types) {
        case FFT_F64: return fft_launch<double, double, double>(b, G, s);
        case FFT_F64_F32: return fft_launch<float, double, float>(b, G, s);
        case FFT_F32: return fft_launch<float, float, float>(b, G, s);
        default: return fft_launch<float, float, double>(b, G, s);
    }
}
