// Spectral field solvers in dense-transform (GEMM) form, float64.
//
// Reference: lcode.py:124-184 (dst2d, dirichlet_matrix, calculate_Ez),
// 187-290 (mix2d, mixed_matrix, dx_dy, calculate_Ex_Ey_Bx_By), 293-364
// (dct2d, neumann_matrix, calculate_Bz).
//
// The reference builds DST-I / DCT-I out of padded real FFTs. Those
// transforms are linear maps with fixed matrices, so every solve is
//     F = L (Lambda o (L X R)) R
// with X the right-hand side, L / R the transform along axis 0 / axis 1 and
// Lambda the eigenvalue matrix (normalisation folded in):
//     S2[k][n] = 2 sin(pi (k+1)(n+1) / (N-1))            (DST-I, M = N-2)
//     C[k][n]  = c_n cos(pi k n / (N-1)), c_0 = c_{N-1} = 1, else 2   (DCT-I)
//   Ey, Bx: X = rhs[1:-1, :]      L = S2, R = C^T, Lambda = mixed_matrix
//   Ex, By: X = rhs[:, 1:-1]      L = C,  R = S2,  Lambda = mixed_matrix^T
//           (the reference solves them transposed, lcode.py:287-288)
//   Ez:     X = rhs_inner         L = S2, R = S2,  Lambda = dirichlet_matrix
//   Bz:     X = rhs               L = C,  R = C^T, Lambda = neumann_matrix
//           (dct2d is minus the DCT-I; the two signs cancel)
// All six fields of a solve run as one batched GEMM per stage (4 stages).

#include <cmath>
#include <cstring>
#include <vector>

#include "lc3d_internal.cuh"

#ifndef LC3D_FFT_STREAMS
#define LC3D_FFT_STREAMS 2   // float64 FFT passes of a solve on 1, 2 or 3 streams
#endif
#ifndef LC3D_FFT32_STREAMS
#define LC3D_FFT32_STREAMS 3   // ... float32 FFT passes
#endif
#ifndef LC3D_FIN_PER_GROUP
#define LC3D_FIN_PER_GROUP 1
#endif

namespace {

// ---------------------------------------------------------------------------
// Right-hand sides, lcode.py:166-168, 234-268, 339-343.
// ---------------------------------------------------------------------------
struct RhsArgs {
    SolveInputs in;
    double st, h, dxi;
    double inv_h2, inv_dxi;   // 1 / (2 h), 1 / dxi
    double* out[6];       // Ex Ey Ez Bx By Bz right-hand sides (N x N, may be NULL)
    int N;
};

__device__ __forceinline__ double avg_in(const double* a, const double* a_prev, size_t k) {
    return a_prev ? (a[k] + a_prev[k]) / 2 : a[k];
}

// x / d from the reciprocal: q0 = x (1/d) is within an ulp of the quotient and
// one correction with the exact residual fma(-q0, d, x) rounds it (the
// float64 divisions of the reference, without the division sequence).
__device__ __forceinline__ double div_by(double x, double d, double inv_d) {
    const double q0 = x * inv_d;
    return fma(fma(-q0, d, x), inv_d, q0);
}

// One grid row per grid line i (blockIdx.y), 128 cells of it per CTA: the
// cell's coordinates come without an integer division.
constexpr int RHS_THREADS = 128;

__global__ void __launch_bounds__(RHS_THREADS) rhs_kernel(const __grid_constant__ RhsArgs a) {
    pdl_wait();
    const int N = a.N;
    const int i = blockIdx.y, j = blockIdx.x * RHS_THREADS + threadIdx.x;
    if (j >= N) return;
    const int k = i * N + j;
    const bool interior = i >= 1 && i <= N - 2 && j >= 1 && j <= N - 2;
    const SolveInputs& in = a.in;
    const double h2 = a.h * 2;
    // every result first, then the stores: the stores could alias the
    // inputs for the compiler, so loads after a store would wait for it
    double o[6] = {};
    if (a.out[0]) {   // the four transverse fields
        double dro_dx = 0, dro_dy = 0, djz_dx = 0, djz_dy = 0;
        if (interior) {
            // (ro_in + beam_ro) and (jz_in + beam_ro) at the four neighbours
            const size_t kp = k + N, km = k - N, lp = k + 1, lm = k - 1;
            dro_dx = div_by((avg_in(in.ro, in.ro_prev, kp) + in.beam[kp]) -
                            (avg_in(in.ro, in.ro_prev, km) + in.beam[km]), h2, a.inv_h2);
            dro_dy = div_by((avg_in(in.ro, in.ro_prev, lp) + in.beam[lp]) -
                            (avg_in(in.ro, in.ro_prev, lm) + in.beam[lm]), h2, a.inv_h2);
            djz_dx = div_by((avg_in(in.jz, in.jz_prev, kp) + in.beam[kp]) -
                            (avg_in(in.jz, in.jz_prev, km) + in.beam[km]), h2, a.inv_h2);
            djz_dy = div_by((avg_in(in.jz, in.jz_prev, lp) + in.beam[lp]) -
                            (avg_in(in.jz, in.jz_prev, lm) + in.beam[lm]), h2, a.inv_h2);
        }
        const double djx_dxi = div_by(in.jx_prev[k] - in.jx[k], a.dxi, a.inv_dxi);
        const double djy_dxi = div_by(in.jy_prev[k] - in.jy[k], a.dxi, a.inv_dxi);
        const double st = a.st;
        o[0] = -((dro_dx - djx_dxi) - in.Ex_sub[k] * st);
        o[1] = -((dro_dy - djy_dxi) - in.Ey_sub[k] * st);
        o[3] = +((djz_dy - djy_dxi) + in.Bx_sub[k] * st);
        o[4] = -((djz_dx - djx_dxi) - in.By_sub[k] * st);
    }
    if (a.out[2] || a.out[5]) {
        double ez = 0, bz = 0;
        if (interior) {
            const double djx_dx = in.jx[k + N] - in.jx[k - N];
            const double djy_dy = in.jy[k + 1] - in.jy[k - 1];
            const double djx_dy = in.jx[k + 1] - in.jx[k - 1];
            const double djy_dx = in.jy[k + N] - in.jy[k - N];
            ez = -div_by(djx_dx + djy_dy, h2, a.inv_h2);
            bz = -div_by(djx_dy - djy_dx, h2, a.inv_h2);
        }
        o[2] = ez;
        o[5] = bz;
    }
#pragma unroll
    for (int f = 0; f < 6; ++f)
        if (a.out[f]) a.out[f][k] = o[f];
}

// ---------------------------------------------------------------------------
// Batched float64 GEMM, C = A B (optionally C = Lambda o (A B)), row-major,
// on the float64 tensor cores (mma.sync m8n8k4 .f64: each product and sum is
// an IEEE float64 fused multiply-add). 128 x 64 tiles per 256-thread CTA,
// eight warps in a 4 x 2 grid of 32 x 32 warp tiles (4 x 4 MMAs per k4
// step); k-steps of 16 staged by cp.async into two shared-memory buffers,
// the next k-step copied while the current one is multiplied.
// ---------------------------------------------------------------------------
constexpr int MAX_PROBS = 6;

struct GemmProb {
    const double *A, *B, *L;
    double* C;
    int M, N, K, lda, ldb, ldc, ldl;
    int tiles_n, tile_start;
};

struct GemmBatch {
    GemmProb p[MAX_PROBS];
    int count, total_tiles;
};

constexpr int GTM = 128, GTN = 64, GK = 16;
constexpr int GEMM_THREADS = 256;
// shared pitches (doubles): the fragment loads of a half-warp (rows g = 0..3
// or 4..7, columns t = 0..3) fall in distinct banks: 2 (20 g + t) and
// 2 (68 t + g) mod 32 are distinct over the 16 lanes
constexpr int AS_LD = GK + 4;    // As[m][k]
constexpr int BS_LD = GTN + 4;   // Bs[k][n]
constexpr int AS_SIZE = GTM * AS_LD, BS_SIZE = GK * BS_LD;
constexpr size_t GEMM_SMEM = 2 * (size_t)(AS_SIZE + BS_SIZE) * sizeof(double);

// 8-byte global -> shared copy; a source size of 0 writes zeros (the tile
// edges past M, N or K).
__device__ __forceinline__ void cp_async8(double* dst, const double* src, bool in) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(in ? 8 : 0) : "memory");
}

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(GEMM_THREADS, 2) dgemm_kernel(const __grid_constant__ GemmBatch b) {
    extern __shared__ __align__(16) double gsm[];   // As[2][GTM][AS_LD], Bs[2][GK][BS_LD]
    double* As = gsm;
    double* Bs = gsm + 2 * AS_SIZE;
    const int bid = blockIdx.x;
    int pi = 0;
#pragma unroll 1
    for (int q = 1; q < b.count; ++q)
        if (bid >= b.p[q].tile_start) pi = q;
    const GemmProb& P = b.p[pi];
    const int t = bid - P.tile_start;
    const int tm = t / P.tiles_n, tn = t - tm * P.tiles_n;
    const int row0 = tm * GTM, col0 = tn * GTN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tq = lane & 3;            // fragment row group, thread in group
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;

    auto load = [&](int k0, int buf) {
        double* as = As + buf * AS_SIZE;
        double* bs = Bs + buf * BS_SIZE;
#pragma unroll
        for (int i = 0; i < GTM * GK / GEMM_THREADS; ++i) {   // 8: rows idx / 16, k idx % 16
            const int idx = tid + i * GEMM_THREADS, r = idx >> 4, kk = idx & 15;
            const int row = row0 + r, k = k0 + kk;
            const bool in = row < P.M && k < P.K;
            cp_async8(as + r * AS_LD + kk, in ? P.A + (size_t)row * P.lda + k : P.A, in);
        }
#pragma unroll
        for (int i = 0; i < GK * GTN / GEMM_THREADS; ++i) {   // 4: k rows idx / 64, columns idx % 64
            const int idx = tid + i * GEMM_THREADS, kk = idx >> 6, n = idx & 63;
            const int k = k0 + kk, col = col0 + n;
            const bool in = k < P.K && col < P.N;
            cp_async8(bs + kk * BS_LD + n, in ? P.B + (size_t)k * P.ldb + col : P.B, in);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int nk = (P.K + GK - 1) / GK;
    load(0, 0);
    for (int kt = 0; kt < nk; ++kt) {
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();   // k-step kt is in; every warp is done with the other buffer
        if (kt + 1 < nk) load((kt + 1) * GK, (kt + 1) & 1);
        const double* as = As + (kt & 1) * AS_SIZE + (wm + g) * AS_LD + tq;
        const double* bs = Bs + (kt & 1) * BS_SIZE + tq * BS_LD + wn + g;
#pragma unroll
        for (int ks = 0; ks < GK; ks += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = as[i * 8 * AS_LD + ks];
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = bs[ks * BS_LD + j * 8];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j], af[i], bf[j]);
        }
    }
    // accumulator (i, j, h): row wm + 8 i + g, column wn + 8 j + 2 tq + h
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int row = row0 + wm + 8 * i + g;
        if (row >= P.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int col = col0 + wn + 8 * j + 2 * tq + h;
                if (col >= P.N) continue;
                double v = acc[i][j][h];
                if (P.L) v *= P.L[(size_t)row * P.ldl + col];
                P.C[(size_t)row * P.ldc + col] = v;
            }
        }
    }
}

int launch_gemm(lc3d_ctx* c, GemmBatch& b, cudaStream_t s) {
    int tiles = 0;
    for (int q = 0; q < b.count; ++q) {
        GemmProb& p = b.p[q];
        p.tiles_n = (p.N + GTN - 1) / GTN;
        p.tile_start = tiles;
        tiles += ((p.M + GTM - 1) / GTM) * p.tiles_n;
    }
    b.total_tiles = tiles;
    if (tiles == 0) return LC3D_OK;
    ProfScope ps(c, LC3D_STAGE_TRANSFORM, s);
    dgemm_kernel<<<tiles, GEMM_THREADS, GEMM_SMEM, s>>>(b);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

// ---------------------------------------------------------------------------
// Deterministic mean (fixed summation tree) and the step finalisation.
// ---------------------------------------------------------------------------
constexpr int RED_THREADS = 256;

__device__ __forceinline__ double block_sum_fixed(double v, double* sh) {
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int s = RED_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    return sh[0];
}

__global__ void __launch_bounds__(RED_THREADS) partial_sum_kernel(const double* __restrict__ a, int n,
                                                                  double* __restrict__ partial) {
    pdl_wait();
    __shared__ double sh[RED_THREADS];
    double v = 0;
    for (int k = blockIdx.x * RED_THREADS + threadIdx.x; k < n; k += gridDim.x * RED_THREADS) v += a[k];
    double s = block_sum_fixed(v, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__device__ double mean_from_partials(const double* partial, int nblocks, double inv_n, double* sh) {
    double v = 0;
    for (int k = threadIdx.x; k < nblocks; k += RED_THREADS) v += partial[k];
    return block_sum_fixed(v, sh) * inv_n;
}

struct FinalizeArgs {
    const double* raw[6];
    const double* prev[6];
    double* out[6];
    double* avg[6];
    const double* partial;
    int nblocks, n, variant_A, has_bz;
    int vec;                          // set by the launcher: every array 16-byte aligned, two cells per thread
    double inv_n;
};

// Field f of one cell: the mean-free Bz, Variant A's 2 F - F_prev, and the
// half-step average (lcode.py:876-881, 906-911).
__device__ __forceinline__ double2 finalize_value(const FinalizeArgs& a, int f, double raw, double prev, double mean) {
    double v = raw;
    if (f == 5) v -= mean;
    if (a.variant_A && f != 2 && f != 5) v = 2 * v - prev;
    return make_double2(v, (v + prev) / 2);
}

__global__ void __launch_bounds__(RED_THREADS) finalize_step_kernel(const __grid_constant__ FinalizeArgs a) {
    pdl_wait();
    __shared__ double sh[RED_THREADS];
    int k = blockIdx.x * RED_THREADS + threadIdx.x;
    if (a.vec) {
        // two cells per thread: all twelve 16-byte loads issued before the
        // stores, and before the Bz mean's reduction (which they overlap)
        k *= 2;
        const bool pair = k + 1 < a.n;
        double2 r[6], p[6];
        if (pair) {
#pragma unroll
            for (int f = 0; f < 6; ++f)
                if (a.raw[f]) {
                    r[f] = __ldcg(reinterpret_cast<const double2*>(a.raw[f] + k));
                    p[f] = __ldcg(reinterpret_cast<const double2*>(a.prev[f] + k));
                }
        }
        // every thread of the CTA takes part in the reduction's barriers
        const double mean = a.has_bz ? mean_from_partials(a.partial, a.nblocks, a.inv_n, sh) : 0.0;
        if (k >= a.n) return;
        if (pair) {
#pragma unroll
            for (int f = 0; f < 6; ++f) {
                if (!a.raw[f]) continue;
                const double2 v0 = finalize_value(a, f, r[f].x, p[f].x, mean);
                const double2 v1 = finalize_value(a, f, r[f].y, p[f].y, mean);
                if (a.out[f]) *reinterpret_cast<double2*>(a.out[f] + k) = make_double2(v0.x, v1.x);
                *reinterpret_cast<double2*>(a.avg[f] + k) = make_double2(v0.y, v1.y);
            }
            return;
        }
        // an odd cell count leaves the last cell to one thread
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            if (!a.raw[f]) continue;
            const double2 v = finalize_value(a, f, a.raw[f][k], a.prev[f][k], mean);
            if (a.out[f]) a.out[f][k] = v.x;
            a.avg[f][k] = v.y;
        }
        return;
    }
    const double mean = a.has_bz ? mean_from_partials(a.partial, a.nblocks, a.inv_n, sh) : 0.0;
    if (k >= a.n) return;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!a.raw[f]) continue;
        const double2 v = finalize_value(a, f, a.raw[f][k], a.prev[f][k], mean);
        if (a.out[f]) a.out[f][k] = v.x;
        a.avg[f][k] = v.y;
    }
}

__global__ void __launch_bounds__(RED_THREADS) subtract_mean_kernel(double* a, int n, const double* partial,
                                                                    int nblocks, double inv_n) {
    pdl_wait();
    __shared__ double sh[RED_THREADS];
    const double mean = mean_from_partials(partial, nblocks, inv_n, sh);
    const int k = blockIdx.x * RED_THREADS + threadIdx.x;
    if (k < n) a[k] -= mean;
}

// ---------------------------------------------------------------------------
// Host: transform and eigenvalue matrices.
// ---------------------------------------------------------------------------

// sin(pi r / L) for integer r, with the argument reduced to [0, pi/2].
double sin_pi_frac(long long r, long long L) {
    r %= 2 * L;
    if (r < 0) r += 2 * L;
    double sign = 1;
    if (r >= L) { r -= L; sign = -1; }
    if (2 * r > L) r = L - r;
    return sign * std::sin(M_PI * (double)r / (double)L);
}

// lam[k] = 4 / h**2 * sin(k pi / (2 (N - 1)))**2 as lcode.py:152-154 writes it
double lam(int k, int N, double h) {
    double s = std::sin(k * M_PI / (2.0 * (N - 1)));
    return 4 / (h * h) * (s * s);
}

int upload(double** dst, const std::vector<double>& v) {
    LC3D_CUDA_TRY(cudaMalloc(dst, v.size() * sizeof(double)));
    LC3D_CUDA_TRY(cudaMemcpy(*dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    return LC3D_OK;
}

// float copy of an eigenvalue matrix (float32-transform precision)
int upload32(float** dst, const std::vector<double>& v) {
    std::vector<float> f(v.begin(), v.end());
    LC3D_CUDA_TRY(cudaMalloc(dst, f.size() * sizeof(float)));
    LC3D_CUDA_TRY(cudaMemcpy(*dst, f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    return LC3D_OK;
}

}  // namespace

int fields_init(lc3d_ctx* c) {
    LC3D_CUDA_TRY(cudaFuncSetAttribute(dgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GEMM_SMEM));
    const int N = c->N, M = c->M;
    const long long L = N - 1;
    const double h = c->p.grid_step_size;
    std::vector<double> S2((size_t)M * M), C((size_t)N * N), CT((size_t)N * N);
    for (int k = 0; k < M; ++k)
        for (int n = 0; n < M; ++n) S2[(size_t)k * M + n] = 2 * sin_pi_frac((long long)(k + 1) * (n + 1), L);
    for (int k = 0; k < N; ++k)
        for (int n = 0; n < N; ++n) {
            // cos(pi r / L) = sin(pi (2 r + L) / (2 L)), r = k n mod 2L
            const long long r = ((long long)k * n) % (2 * L);
            const double cv = sin_pi_frac(2 * r + L, 2 * L);
            const double w = (n == 0 || n == N - 1) ? 1.0 : 2.0;
            C[(size_t)k * N + n] = w * cv;
            CT[(size_t)n * N + k] = w * cv;
        }
    const double norm = 1.0 / ((2.0 * (N - 1)) * (2.0 * (N - 1)));
    const double trick = c->p.field_solver_subtraction_trick != 0 ? 1.0 : 0.0;
    std::vector<double> ld((size_t)M * M), lm((size_t)M * N), lmT((size_t)N * M), ln((size_t)N * N);
    std::vector<double> lamk(N);
    for (int k = 0; k < N; ++k) lamk[k] = lam(k, N, h);
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < M; ++j) ld[(size_t)i * M + j] = (1 / (lamk[i + 1] + lamk[j + 1])) * norm;
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < N; ++j) {
            const double v = (1 / (lamk[i + 1] + lamk[j] + trick)) * norm;
            lm[(size_t)i * N + j] = v;
            lmT[(size_t)j * M + i] = v;
        }
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            ln[(size_t)i * N + j] = (i == 0 && j == 0) ? 0.0 : (1 / (lamk[i] + lamk[j])) * norm;
    LC3D_TRY(upload(&c->S2, S2));
    LC3D_TRY(upload(&c->C, C));
    LC3D_TRY(upload(&c->CT, CT));
    LC3D_TRY(upload(&c->lam_dir, ld));
    LC3D_TRY(upload(&c->lam_mix, lm));
    LC3D_TRY(upload(&c->lam_mixT, lmT));
    LC3D_TRY(upload(&c->lam_neu, ln));
    if (c->p.precision == LC3D_PREC_FFT32) {
        LC3D_TRY(upload32(&c->lam32_dir, ld));
        LC3D_TRY(upload32(&c->lam32_mix, lm));
        LC3D_TRY(upload32(&c->lam32_mixT, lmT));
        LC3D_TRY(upload32(&c->lam32_neu, ln));
    }
    const size_t plane = (size_t)N * N * sizeof(double);
    const size_t tplane = (size_t)N * fft_pitch(N) * sizeof(double);   // the transform intermediates
    for (int f = 0; f < 6; ++f) {
        LC3D_CUDA_TRY(cudaMalloc(&c->rhs[f], plane));
        LC3D_CUDA_TRY(cudaMalloc(&c->t1[f], tplane));
        LC3D_CUDA_TRY(cudaMalloc(&c->t2[f], tplane));
        LC3D_CUDA_TRY(cudaMalloc(&c->raw[f], plane));
        LC3D_CUDA_TRY(cudaMemset(c->rhs[f], 0, plane));
        LC3D_CUDA_TRY(cudaMemset(c->raw[f], 0, plane));
    }
    c->red_blocks = 160;
    // room for the partial-sum kernel's blocks and for the FFT pass's per-CTA sums
    LC3D_CUDA_TRY(cudaMalloc(&c->red, 4096 * sizeof(double)));
    return LC3D_OK;
}

void fields_free(lc3d_ctx* c) {
    double** ps[] = {&c->S2, &c->C, &c->CT, &c->lam_dir, &c->lam_mix, &c->lam_mixT, &c->lam_neu, &c->red};
    for (double** p : ps) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    float** ps32[] = {&c->lam32_dir, &c->lam32_mix, &c->lam32_mixT, &c->lam32_neu};
    for (float** p : ps32) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    for (int f = 0; f < 6; ++f) {
        double** q[] = {&c->rhs[f], &c->t1[f], &c->t2[f], &c->raw[f]};
        for (double** p : q) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
    }
}

namespace {

struct FieldGeom {
    int rows, cols;
    size_t off;            // offset of X / output inside an N x N plane
    const double *L, *R, *Lam;
    int ldL, ldR, ldLam;
    int type0, type1;      // axis-0 / axis-1 transform: 0 DCT-I, 1 DST-I
};

FieldGeom geom(const lc3d_ctx* c, int f) {
    const int N = c->N, M = c->M;
    FieldGeom g{};
    switch (f) {
        case 0: case 4:   // Ex, By: solved transposed
            g = {N, M, 1, c->C, c->S2, c->lam_mixT, N, M, M, 0, 1};
            break;
        case 1: case 3:   // Ey, Bx
            g = {M, N, (size_t)N, c->S2, c->CT, c->lam_mix, M, N, N, 1, 0};
            break;
        case 2:           // Ez
            g = {M, M, (size_t)N + 1, c->S2, c->S2, c->lam_dir, M, M, M, 1, 1};
            break;
        default:          // Bz
            g = {N, N, 0, c->C, c->CT, c->lam_neu, N, N, N, 0, 0};
            break;
    }
    return g;
}

// The float copy of field f's eigenvalue matrix (float32-transform precision).
const float* lam32(const lc3d_ctx* c, int f) {
    switch (f) {
        case 0: case 4: return c->lam32_mixT;
        case 1: case 3: return c->lam32_mix;
        case 2: return c->lam32_dir;
        default: return c->lam32_neu;
    }
}

}  // namespace

int solve_fields(lc3d_ctx* c, int which, const SolveInputs& in, const SolveOutputs& o, cudaStream_t s) {
    const int N = c->N;
    const int n = N * N;
    bool on[6] = {false, false, false, false, false, false};
    if (which & LC3D_F_EXEYBXBY) on[0] = on[1] = on[3] = on[4] = true;
    if (which & LC3D_F_EZ) on[2] = true;
    if (which & LC3D_F_BZ) on[5] = true;

    RhsArgs ra{};
    memset(&ra, 0, sizeof(ra));
    ra.in = in;
    ra.st = c->p.field_solver_subtraction_trick;
    ra.h = c->p.grid_step_size;
    ra.dxi = c->p.xi_step_size;
    ra.inv_h2 = 1.0 / (ra.h * 2);
    ra.inv_dxi = 1.0 / ra.dxi;
    ra.N = N;
    for (int f = 0; f < 6; ++f) ra.out[f] = on[f] ? c->rhs[f] : nullptr;
    {
        ProfScope ps(c, LC3D_STAGE_RHS, s);
        LC3D_CUDA_TRY(launch_pdl(rhs_kernel, dim3((c->N + RHS_THREADS - 1) / RHS_THREADS, c->N), dim3(RHS_THREADS), 0,
                                 s, ra));
        LC3D_CUDA_TRY(cudaGetLastError());
    }

    // destination of the raw solution
    double* dst[6];
    for (int f = 0; f < 6; ++f) {
        dst[f] = nullptr;
        if (!on[f]) continue;
        if (o.mode == 0) {
            dst[f] = o.out[f];
            if (f != 5) LC3D_CUDA_TRY(cudaMemsetAsync(dst[f], 0, (size_t)n * sizeof(double), s));
        } else {
            dst[f] = c->raw[f];
        }
    }
    int bz_partials = 0;   // > 0: the FFT pass left this many Bz partial sums in c->red
    // FFT passes on several streams whose join waits until each group's
    // finalize has run on its own stream (step finalisation only)
    int fin_groups = 0;
    int fin_group_of[6] = {0, 0, 0, 0, 0, 0};
    cudaStream_t fin_stream[3] = {s, s, s};
    if (c->p.precision == LC3D_PREC_MIXED || c->p.precision == LC3D_PREC_TF32) {
        // four split-BF16 tensor-core GEMM stages (fields_mixed.cu)
        for (int stage = 0; stage < 4; ++stage) {
            MixedStageDesc d[6]{};
            int cnt = 0;
            for (int f = 0; f < 6; ++f) {
                if (!on[f]) continue;
                const FieldGeom g = geom(c, f);
                MixedStageDesc& e = d[cnt++];
                memset(&e, 0, sizeof(e));
                e.field = f;
                e.M = g.rows;
                e.N = g.cols;
                e.ld_data = N;
                e.ldo = N;
                const int fixed_L = g.type0 ? 0 : 1, fixed_RT = g.type1 ? 0 : 1;   // 0: S2, 1: C
                switch (stage) {
                    case 0:   // T1^T = (X R)^T
                        e.data = c->rhs[f] + g.off; e.data_rows = g.rows; e.K = g.cols;
                        e.data_is_a = 1; e.fixed = fixed_RT; e.out = c->t1[f]; e.transposed = 1;
                        break;
                    case 1:   // Z = Lambda o (L T1)
                        e.data = c->t1[f]; e.data_rows = g.cols; e.K = g.rows;
                        e.data_is_a = 0; e.fixed = fixed_L; e.out = c->t2[f];
                        e.lam = g.Lam; e.ldl = g.ldLam;
                        break;
                    case 2:   // U^T = (Z R)^T
                        e.data = c->t2[f]; e.data_rows = g.rows; e.K = g.cols;
                        e.data_is_a = 1; e.fixed = fixed_RT; e.out = c->t1[f]; e.transposed = 1;
                        break;
                    default:  // F = L U
                        e.data = c->t1[f]; e.data_rows = g.cols; e.K = g.rows;
                        e.data_is_a = 0; e.fixed = fixed_L; e.out = dst[f] + g.off;
                        break;
                }
            }
            LC3D_TRY(mixed_stage(c, d, cnt, s));
        }
    } else if (c->use_fft || c->p.precision == LC3D_PREC_FFT32) {
        // four FFT row passes, each writing its output transposed; with the
        // float32-transform precision the passes compute in float32 and the
        // two intermediates (in the t1 / t2 planes) are float32
        const bool f32 = c->p.precision == LC3D_PREC_FFT32;
        const int types[4] = {f32 ? FFT_F64_F32 : FFT_F64, f32 ? FFT_F32 : FFT_F64, f32 ? FFT_F32 : FFT_F64,
                              f32 ? FFT_F32_F64 : FFT_F64};
        // The fields' passes on several streams (forked after the right-hand
        // sides, joined before the finalize): with two, the E fields on the
        // solve's stream and the B fields on a second; with three, Ex Ey /
        // Bx By / Ez Bz. The groups' passes are independent, so the tail of
        // one group's pass, when only part of the SMs still work, is filled
        // by the other groups' row groups. Measured at 641^2: float64 1802 ->
        // 1864 xi-steps/s with two streams (1835 with three); float32
        // transforms 2109 -> 2145 with two, 2176 with three. The per-launch
        // timing pass keeps one stream, and so do the steps of a batch graph
        // (its branches overlap the simulations already: a 32-simulation scan
        // measured 3772 aggregate xi-steps/s on one stream, 3600 on several).
        const int nstreams = (c->prof_on || c->one_stream) ? 1 : f32 ? LC3D_FFT32_STREAMS : LC3D_FFT_STREAMS;
        auto group_of = [&](int f) {
            if (nstreams == 3) return f == 2 || f == 5 ? 2 : (f < 2 ? 0 : 1);
            if (nstreams == 2) return f < 3 ? 0 : 1;
            return 0;
        };
        bool used[3] = {false, false, false};
        for (int f = 0; f < 6; ++f)
            if (on[f]) used[group_of(f)] = true;
        if (nstreams > 1) {
            LC3D_CUDA_TRY(cudaEventRecord(c->ev_fork, s));
            for (int q = 1; q < nstreams; ++q)
                if (used[q]) LC3D_CUDA_TRY(cudaStreamWaitEvent(c->fft_stream[q - 1], c->ev_fork, 0));
        }
        for (int stage = 0; stage < 4; ++stage) {
            FftRowsDesc d[6]{};
            int cnt = 0;
            for (int f = 0; f < 6; ++f) {
                if (!on[f]) continue;
                const FieldGeom g = geom(c, f);
                FftRowsDesc& e = d[cnt++];
                memset(&e, 0, sizeof(e));
                // the intermediates t1 / t2 at a row pitch of whole 32-byte
                // sectors, so a CTA's transposed stores fill whole sectors
                const int Np = fft_pitch(N, f32);
                e.ld_in = stage == 0 ? N : Np;
                e.ld_out = stage == 3 ? N : Np;
                switch (stage) {
                    case 0: e.in = c->rhs[f] + g.off; e.rows = g.rows; e.type = g.type1; e.out = c->t1[f]; break;
                    case 1: e.in = c->t1[f]; e.rows = g.cols; e.type = g.type0; e.out = c->t2[f];
                            e.lam = f32 ? static_cast<const void*>(lam32(c, f)) : g.Lam;
                            e.ld_lam = g.ldLam; break;   // Lambda o Z as Z is written
                    case 2: e.in = c->t2[f]; e.rows = g.rows; e.type = g.type1; e.out = c->t1[f]; break;
                    default: e.in = c->t1[f]; e.rows = g.cols; e.type = g.type0; e.out = dst[f] + g.off;
                             if (f == 5) {   // Bz: the mean's partial sums come with the last pass
                                 e.partial = c->red;
                                 bz_partials = (g.cols + fft_cta_rows() - 1) / fft_cta_rows();
                             }
                             break;
                }
            }
            if (nstreams > 1) {   // each group of fields on its stream
                for (int q = 0; q < nstreams; ++q) {
                    if (!used[q]) continue;
                    FftRowsDesc dq[6];
                    int nq = 0, k = 0;
                    for (int f = 0; f < 6; ++f) {
                        if (!on[f]) continue;
                        if (group_of(f) == q) dq[nq++] = d[k];
                        ++k;
                    }
                    LC3D_TRY(fft_rows(c, dq, nq, types[stage], q ? c->fft_stream[q - 1] : s));
                }
            } else {
                LC3D_TRY(fft_rows(c, d, cnt, types[stage], s));
            }
        }
        if (LC3D_FIN_PER_GROUP && o.mode == 1 && nstreams > 1) {   // each group finalised on its own stream, then joined
            fin_groups = nstreams;
            for (int f = 0; f < 6; ++f) fin_group_of[f] = group_of(f);
            for (int q = 1; q < nstreams; ++q) fin_stream[q] = used[q] ? c->fft_stream[q - 1] : s;
        } else {
            for (int q = 1; q < nstreams; ++q) {
                if (!used[q]) continue;
                LC3D_CUDA_TRY(cudaEventRecord(c->ev_join[q - 1], c->fft_stream[q - 1]));
                LC3D_CUDA_TRY(cudaStreamWaitEvent(s, c->ev_join[q - 1], 0));
            }
        }
    } else {
        // the four GEMM stages
        for (int stage = 0; stage < 4; ++stage) {
            GemmBatch b{};
            memset(&b, 0, sizeof(b));
            for (int f = 0; f < 6; ++f) {
                if (!on[f]) continue;
                const FieldGeom g = geom(c, f);
                GemmProb& p = b.p[b.count++];
                switch (stage) {
                    case 0:   // t1 = X R
                        p.A = c->rhs[f] + g.off; p.lda = N;
                        p.B = g.R; p.ldb = g.ldR;
                        p.C = c->t1[f]; p.ldc = N;
                        p.M = g.rows; p.N = g.cols; p.K = g.cols;
                        break;
                    case 1:   // t2 = Lambda o (L t1)
                        p.A = g.L; p.lda = g.ldL;
                        p.B = c->t1[f]; p.ldb = N;
                        p.C = c->t2[f]; p.ldc = N;
                        p.L = g.Lam; p.ldl = g.ldLam;
                        p.M = g.rows; p.N = g.cols; p.K = g.rows;
                        break;
                    case 2:   // t1 = t2 R
                        p.A = c->t2[f]; p.lda = N;
                        p.B = g.R; p.ldb = g.ldR;
                        p.C = c->t1[f]; p.ldc = N;
                        p.M = g.rows; p.N = g.cols; p.K = g.cols;
                        break;
                    default:  // out = L t1
                        p.A = g.L; p.lda = g.ldL;
                        p.B = c->t1[f]; p.ldb = N;
                        p.C = dst[f] + g.off; p.ldc = N;
                        p.M = g.rows; p.N = g.cols; p.K = g.rows;
                        break;
                }
            }
            LC3D_TRY(launch_gemm(c, b, s));
        }
    }
    const double inv_n = 1.0 / n;
    if (on[5] && !bz_partials) {
        ProfScope ps(c, LC3D_STAGE_FIELD_FIN, s);
        LC3D_CUDA_TRY(launch_pdl(partial_sum_kernel, dim3(c->red_blocks), dim3(RED_THREADS), 0, s,
                                 static_cast<const double*>(dst[5]), n, c->red));
        LC3D_CUDA_TRY(cudaGetLastError());
    }
    const int nred = bz_partials ? bz_partials : c->red_blocks;
    if (o.mode == 0) {
        if (on[5]) {
            ProfScope ps(c, LC3D_STAGE_FIELD_FIN, s);
            LC3D_CUDA_TRY(launch_pdl(subtract_mean_kernel, dim3((n + RED_THREADS - 1) / RED_THREADS),
                                     dim3(RED_THREADS), 0, s, dst[5], n, static_cast<const double*>(c->red),
                                     nred, inv_n));
            LC3D_CUDA_TRY(cudaGetLastError());
        }
        return LC3D_OK;
    }
    // one finalize over all fields, or one per group of fields on that
    // group's stream (the groups' FFT passes ran on several streams)
    for (int q = 0; q < (fin_groups ? fin_groups : 1); ++q) {
        FinalizeArgs fa{};
        memset(&fa, 0, sizeof(fa));
        for (int f = 0; f < 6; ++f) {
            if (!on[f] || (fin_groups && fin_group_of[f] != q)) continue;
            fa.raw[f] = c->raw[f];
            fa.prev[f] = o.prev[f];
            fa.out[f] = o.out[f];
            fa.avg[f] = o.avg[f];
        }
        bool any = false;
        for (int f = 0; f < 6; ++f) any = any || fa.raw[f];
        if (!any) continue;
        fa.partial = c->red;
        fa.nblocks = nred;
        fa.n = n;
        fa.variant_A = c->p.field_solver_variant_A;
        fa.has_bz = fa.raw[5] != nullptr;
        fa.inv_n = inv_n;
        uintptr_t al = 0;
        for (int f = 0; f < 6; ++f)
            al |= reinterpret_cast<uintptr_t>(fa.raw[f]) | reinterpret_cast<uintptr_t>(fa.prev[f]) |
                  reinterpret_cast<uintptr_t>(fa.out[f]) | reinterpret_cast<uintptr_t>(fa.avg[f]);
        fa.vec = (al & 15) == 0;
        const int threads = fa.vec ? (n + 1) / 2 : n;
        cudaStream_t sq = fin_groups ? fin_stream[q] : s;
        ProfScope ps(c, LC3D_STAGE_FIELD_FIN, sq);
        LC3D_CUDA_TRY(launch_pdl(finalize_step_kernel, dim3((threads + RED_THREADS - 1) / RED_THREADS),
                                 dim3(RED_THREADS), 0, sq, fa));
        LC3D_CUDA_TRY(cudaGetLastError());
    }
    for (int q = 1; q < fin_groups; ++q) {
        if (fin_stream[q] == s) continue;
        LC3D_CUDA_TRY(cudaEventRecord(c->ev_join[q - 1], fin_stream[q]));
        LC3D_CUDA_TRY(cudaStreamWaitEvent(s, c->ev_join[q - 1], 0));
    }
    return LC3D_OK;
}
