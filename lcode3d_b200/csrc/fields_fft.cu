// Float64 DST-I / DCT-I row transforms through a shared-memory FFT.
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
// in-place decimation-in-frequency FFT with mixed radices 4, 2, 3, 5 in
// shared memory, read out in digit-reversed order. Every launch transforms rows and writes its output
// TRANSPOSED (out[k][r]), optionally scaled by Lambda[k][r]; the 2-D solve
// F = L (Lambda o (L X R)) R is then four such passes:
//     A: rows of X by the axis-1 transform          -> T1^T
//     B: rows of T1^T by the axis-0 transform, x Lambda -> Z
//     C: rows of Z by the axis-1 transform          -> T3^T
//     D: rows of T3^T by the axis-0 transform       -> F
// One launch covers all fields of a solve.

#include <cmath>
#include <cstring>
#include <vector>

#include "lc3d_internal.cuh"

namespace {

constexpr int FFT_THREADS = 256;
constexpr int FFT_PER_CTA = 2;           // complex FFTs per CTA (4 rows)
constexpr int ROWS_PER_CTA = 2 * FFT_PER_CTA;
constexpr int MAX_RADICES = 24;

struct FftField {
    const double* in;
    int ld_in, rows, type;               // type: 0 DCT-I (n = N), 1 DST-I (n = N - 2)
    double* out;
    int ld_out;
    const double* lam;
    int ld_lam;
    int cta_start;
};

struct FftBatch {
    FftField f[6];
    int count, P, N;
    int nrad;
    int rad[MAX_RADICES];
    const double2* tw;                   // tw[m] = exp(-2 pi i m / P)
    const int* pos;                      // position of frequency k after the DIF passes
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }

// Small DFTs in registers, forward sign.
template <int R>
__device__ __forceinline__ void dft(double2 (&v)[R], const double2* __restrict__ tw, int P) {
    double2 o[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        double2 s = v[0];
#pragma unroll
        for (int r = 1; r < R; ++r) s = cadd(s, cmul(v[r], __ldg(tw + ((r * m) % R) * (P / R))));
        o[m] = s;
    }
#pragma unroll
    for (int m = 0; m < R; ++m) v[m] = o[m];
}

template <>
__device__ __forceinline__ void dft<2>(double2 (&v)[2], const double2*, int) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

// x -> -i x
__device__ __forceinline__ double2 mul_mi(double2 a) { return make_double2(a.y, -a.x); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// 3-point DFT: W = exp(-2 pi i / 3) = (c, -s) read from the twiddle table.
template <>
__device__ __forceinline__ void dft<3>(double2 (&v)[3], const double2* tw, int P) {
    const double2 w = __ldg(tw + P / 3);
    const double2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    const double2 a = cadd(v[0], cscale(t1, w.x));
    const double2 bb = cscale(t2, -w.y);
    v[0] = cadd(v[0], t1);
    v[1] = cadd(a, mul_mi(bb));
    v[2] = csub(a, mul_mi(bb));
}

// 5-point DFT with W = (c1, -s1), W^2 = (c2, -s2) from the twiddle table:
// X1,4 = v0 + c1 t1 + c2 t2 -+ i (s1 t3 + s2 t4),
// X2,3 = v0 + c2 t1 + c1 t2 -+ i (s2 t3 - s1 t4),
// t1 = v1 + v4, t2 = v2 + v3, t3 = v1 - v4, t4 = v2 - v3.
template <>
__device__ __forceinline__ void dft<5>(double2 (&v)[5], const double2* tw, int P) {
    const double2 w1 = __ldg(tw + P / 5), w2 = __ldg(tw + 2 * (P / 5));
    const double c1 = w1.x, s1 = -w1.y, c2 = w2.x, s2 = -w2.y;
    const double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const double2 a1 = cadd(v[0], cadd(cscale(t1, c1), cscale(t2, c2)));
    const double2 a2 = cadd(v[0], cadd(cscale(t1, c2), cscale(t2, c1)));
    const double2 b1 = cadd(cscale(t3, s1), cscale(t4, s2));
    const double2 b2 = csub(cscale(t3, s2), cscale(t4, s1));
    v[0] = cadd(v[0], cadd(t1, t2));
    v[1] = cadd(a1, mul_mi(b1));
    v[4] = csub(a1, mul_mi(b1));
    v[2] = cadd(a2, mul_mi(b2));
    v[3] = csub(a2, mul_mi(b2));
}

template <>
__device__ __forceinline__ void dft<4>(double2 (&v)[4], const double2*, int) {
    const double2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    const double2 a2 = cadd(v[1], v[3]), d = csub(v[1], v[3]);
    const double2 a3 = make_double2(d.y, -d.x);   // -i (v1 - v3)
    v[0] = cadd(a0, a2);
    v[2] = csub(a0, a2);
    v[1] = cadd(a1, a3);
    v[3] = csub(a1, a3);
}

// One in-place decimation-in-frequency butterfly of radix R inside a
// sub-transform of length Lr = R * span: the R inputs A[base + r span] are
// transformed and output m is scaled by exp(-2 pi i m k / Lr), k the
// position inside the span, and written back in place. After all passes
// frequency k = m0 + R0 (m1 + R1 (m2 + ...)) sits at sum_s m_s P / (R0..Rs).
template <int R>
__device__ __forceinline__ void dif_butterfly(double2* A, int b, int span, float inv_span, int P,
                                              const double2* __restrict__ tw) {
    // g = b / span: (b + 0.5) / span lies at least 0.5 / span from an
    // integer, far more than the float rounding for b, span < 2^16
    const int g = __float2int_rz(((float)b + 0.5f) * inv_span), k = b - g * span;
    const int base = g * span * R + k;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = A[base + r * span];
    dft<R>(v, tw, P);
    const int tstep = P / (span * R);
#pragma unroll
    for (int m = 1; m < R; ++m) v[m] = cmul(v[m], __ldg(tw + m * k * tstep));
#pragma unroll
    for (int m = 0; m < R; ++m) A[base + m * span] = v[m];
}

template <int R>
__device__ __forceinline__ void fft_pass(double2* A, int span, int P, const double2* tw) {
    static_assert(FFT_PER_CTA == 2, "the FFT index below assumes two FFTs per CTA");
    const int nb = P / R;
    const float inv_span = 1.0f / (float)span;
    for (int t = threadIdx.x; t < FFT_PER_CTA * nb; t += FFT_THREADS) {
        const int q = t >= nb, j = t - q * nb;
        dif_butterfly<R>(A + q * P, j, span, inv_span, P, tw);
    }
}

__global__ void __launch_bounds__(FFT_THREADS, 3) fft_rows_kernel(const __grid_constant__ FftBatch b) {
    extern __shared__ double2 sm[];      // [FFT_PER_CTA][P], transformed in place
    int fi = 0;
#pragma unroll 1
    for (int q = 1; q < b.count; ++q)
        if ((int)blockIdx.x >= b.f[q].cta_start) fi = q;
    const FftField& F = b.f[fi];
    const int P = b.P, L = P / 2;
    const int r0 = ((int)blockIdx.x - F.cta_start) * ROWS_PER_CTA;
    const int n = F.type ? b.N - 2 : b.N;     // input / output length
    double2* A = sm;

    // symmetric / antisymmetric extensions, two rows per complex FFT
    for (int t = threadIdx.x; t < FFT_PER_CTA * P; t += FFT_THREADS) {
        const int q = t >= P, m = t - q * P;
        double v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int row = r0 + 2 * q + h;
            double x = 0;
            if (row < F.rows) {
                const double* rp = F.in + (size_t)row * F.ld_in;
                if (F.type == 0) {
                    x = __ldg(rp + (m <= L ? m : P - m));
                } else if (m != 0 && m != L) {
                    x = m < L ? __ldg(rp + m - 1) : -__ldg(rp + P - m - 1);
                }
            }
            v[h] = x;
        }
        A[t] = make_double2(v[0], v[1]);
    }
    __syncthreads();
    int span = P;
    for (int p = 0; p < b.nrad; ++p) {
        const int R = b.rad[p];
        span /= R;
        switch (R) {
            case 4: fft_pass<4>(A, span, P, b.tw); break;
            case 2: fft_pass<2>(A, span, P, b.tw); break;
            case 3: fft_pass<3>(A, span, P, b.tw); break;
            default: fft_pass<5>(A, span, P, b.tw); break;
        }
        __syncthreads();
    }
    // transposed output, 4 consecutive rows per output index k; frequency
    // kk sits at its digit-reversed position
    const int off = F.type;   // DST-I outputs are Z[1 .. L-1]
    for (int t = threadIdx.x; t < n * ROWS_PER_CTA; t += FFT_THREADS) {
        const int k = t / ROWS_PER_CTA, rr = t - k * ROWS_PER_CTA;
        const int row = r0 + rr;
        if (row >= F.rows) continue;
        const double2 z = A[(rr >> 1) * P + __ldg(b.pos + k + off)];
        double x;
        if (F.type == 0)
            x = (rr & 1) ? z.y : z.x;
        else
            x = (rr & 1) ? z.x : -z.y;
        if (F.lam) x *= F.lam[(size_t)k * F.ld_lam + row];
        F.out[(size_t)k * F.ld_out + row] = x;
    }
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

// Radix plan for a length-P FFT: factors 4, 2, 3, 5 (powers of 4 first).
// Returns the number of passes, or 0 if P has another prime factor (the
// dense transform form is used then).
int fft_plan(int P, int* rad) {
    int n = 0;
    int r = P;
    while (r % 4 == 0 && n < MAX_RADICES) { rad[n++] = 4; r /= 4; }
    const int others[] = {2, 3, 5};
    for (int f : others)
        while (r % f == 0 && n < MAX_RADICES) { rad[n++] = f; r /= f; }
    return (r == 1) ? n : 0;
}

size_t fft_smem_bytes(int P) { return (size_t)FFT_PER_CTA * P * sizeof(double2); }

int fft_init(lc3d_ctx* c) {
    const int P = 2 * (c->N - 1);
    int rad[MAX_RADICES];
    c->fft_ok = fft_plan(P, rad) > 0 && fft_smem_bytes(P) <= 200 * 1024;
    if (!c->fft_ok) return LC3D_OK;
    LC3D_TRY(fft_prepare(P));
    const int nrad = fft_plan(P, rad);
    // P twiddles exp(-2 pi i m / P), then P int32 positions: frequency k of
    // the in-place DIF output sits at pos[k] = sum_s m_s P / (R0..Rs) for the
    // mixed-radix digits k = m0 + R0 (m1 + R1 (...))
    std::vector<double> buf(3 * (size_t)P);
    for (int m = 0; m < P; ++m) {
        buf[2 * m] = sin_pi_frac(4LL * m + P, 2LL * P);      // cos(pi (2m) / P)
        buf[2 * m + 1] = -sin_pi_frac(2LL * m, (long long)P);
    }
    int32_t* pos = reinterpret_cast<int32_t*>(buf.data() + 2 * (size_t)P);
    for (int k = 0; k < P; ++k) {
        int kk = k, p = 0, rem = P;
        for (int s = 0; s < nrad; ++s) {
            const int m = kk % rad[s];
            kk /= rad[s];
            rem /= rad[s];
            p += m * rem;
        }
        pos[k] = p;
    }
    LC3D_CUDA_TRY(cudaMalloc(&c->fft_tw, buf.size() * sizeof(double)));
    LC3D_CUDA_TRY(cudaMemcpy(c->fft_tw, buf.data(), buf.size() * sizeof(double), cudaMemcpyHostToDevice));
    return LC3D_OK;
}

int fft_prepare(int P) {
    // the limit is per kernel, not per context: always the largest size any
    // context may use (contexts of different grid sizes coexist in batches)
    (void)P;
    LC3D_CUDA_TRY(cudaFuncSetAttribute(fft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    return LC3D_OK;
}

// One transform pass over up to 6 fields: desc[f] = {in, ld_in, rows, type,
// out, ld_out, lam, ld_lam}; rows of `in` are transformed and written
// transposed into `out`.
int fft_rows(lc3d_ctx* c, const FftRowsDesc* desc, int count, cudaStream_t s) {
    FftBatch b;
    memset(&b, 0, sizeof(b));
    b.P = 2 * (c->N - 1);
    b.N = c->N;
    b.nrad = fft_plan(b.P, b.rad);
    b.tw = reinterpret_cast<const double2*>(c->fft_tw);
    b.pos = reinterpret_cast<const int*>(c->fft_tw + 2 * (size_t)b.P);
    int ctas = 0;
    for (int q = 0; q < count; ++q) {
        FftField& f = b.f[b.count++];
        f.in = desc[q].in; f.ld_in = desc[q].ld_in; f.rows = desc[q].rows; f.type = desc[q].type;
        f.out = desc[q].out; f.ld_out = desc[q].ld_out; f.lam = desc[q].lam; f.ld_lam = desc[q].ld_lam;
        f.cta_start = ctas;
        ctas += (f.rows + ROWS_PER_CTA - 1) / ROWS_PER_CTA;
    }
    if (!ctas) return LC3D_OK;
    const size_t smem = fft_smem_bytes(b.P);
    ProfScope ps(c, LC3D_STAGE_TRANSFORM, s);
    fft_rows_kernel<<<ctas, FFT_THREADS, smem, s>>>(b);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}
