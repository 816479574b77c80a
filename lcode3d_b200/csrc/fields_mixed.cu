// Mixed-precision field solvers: the dense-transform stages of
// F = L (Lambda o (L X R)) R (see fields.cu) as split-BF16 GEMMs on the
// 5th-generation tensor cores (tcgen05, accumulators in TMEM, operands
// staged by TMA), accumulated in FP32 and combined in float64.
//
// Splitting (an Ozaki-type scheme). Every row r of an operand is scaled by a
// power of two 2^-e_r so that |x| < 1, then written as S digit slices
//     x 2^-e = sum_s d_s 2^-7(s+1),  d_s integer, |d_0| <= 128, |d_s| <= 64,
// each slice d_s 2^-7(s+1) exact in bf16. For C = A B^T (both K-major):
//     C = 2^(e_a + e_b) sum_{s+t < S} A_s B_t^T.
// All products of one digit level d = s + t share the unit 2^-7(d+2), and
// per k their integer parts sum to at most 16384, 16384, 20480, 24576 for
// d = 0, 1, 2, 3, so over K <= 682 every level sum stays below 2^24: with
// one FP32 accumulator per level (4 x 128 TMEM columns, all of TMEM) the
// tensor-core accumulation is EXACT for the first four levels (levels >= 4,
// 2^-28 smaller, join the level-3 accumulator). The only error left is the
// truncation after S slices, ~2^-7S of the row maxima; the epilogue adds the
// level sums in float64 and applies 2^(e_a + e_b).
//
// GEMM kernel: persistent, one CTA per SM looping over 128 x 64 output
// tiles; K in blocks of 32 (64-byte rows, 64-byte swizzle), all 2S operand
// slices of a K block per pipeline stage, the stages running on from one
// tile to the next. Warp 0 issues TMA loads, warp 1 owns the TMEM
// allocation and issues tcgen05.mma (128 x 64 x 16, bf16 -> f32) from one
// thread, warps 2-5 read the four accumulators with tcgen05.ld and write
// float64. TMEM holds two sets of the four accumulators (2 x 4 x 64
// columns): the MMAs of a tile run into one set while the epilogue drains
// the other's previous tile. Every mbarrier wait is bounded: on time-out the
// kernel raises an error flag and every role leaves its loop, and TMEM is
// always freed.
//
// Stages of one solve (rows x cols field, L = axis-0 and R = axis-1
// transform; S2 and C are symmetric or appear as C^T^T = C, so the two
// fixed operands are S2 and C, sliced once on the host):
//   1. T1^T = (X R)^T     A = X       B^T = R^T     output transposed
//   2. Z = Lam o (L T1)   A = L       B^T = T1^T
//   3. U^T = (Z R)^T      A = Z       B^T = R^T     output transposed
//   4. F = L U            A = L       B^T = U^T
// The data operands are sliced by a row kernel before each stage.
//
// TF32 form (LC3D_PREC_TF32). The same pipeline with tcgen05.mma kind::tf32:
// the digits are 10 bits wide, |d_0| <= 1024, |d_s| <= 512, each slice
// d_s 2^-10(s+1) exact in tf32 (11-bit significand), stored as float32 (16
// values per 64-byte row, K blocks of 16, two MMAs of K = 8 per row). A
// level's products reach 2^20 units per k, so over K of several hundred
// the FP32 accumulation is no longer exact: each stage carries the FP32
// rounding of its sums (about 2^-24 sqrt(K) of the level's size) on top of
// the truncation after S slices, ~2^-10S.

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "lc3d_internal.cuh"
#include "tc_sm100.cuh"

namespace {

constexpr int TM = 128, TN = 64;                               // output tile
constexpr int TILE_A_BYTES = TM * 64;                            // 8 KiB: 128 rows of 64 bytes
constexpr int TILE_B_BYTES = TN * 64;                            // 4 KiB
constexpr int BOX_ROWS = 64;                                     // TMA box height (an A tile is two boxes)
constexpr int KIND_BF16 = 0, KIND_TF32 = 1;
#ifndef LC3D_OZ_CLOCKS
#define LC3D_OZ_CLOCKS 0   // instrumented builds: per-CTA wait / work cycles of the MMA thread and epilogue
#endif
#if LC3D_OZ_CLOCKS
__device__ long long g_oz_clocks[1024][8];
#endif
#ifndef LC3D_OZ_MAX_STAGES
#define LC3D_OZ_MAX_STAGES 4                                     // pipeline stages at most
#endif

// Elements of one 64-byte operand row: 32 bf16 or 16 tf32 (float32).
__host__ __device__ constexpr int k_block(int kind) { return kind == KIND_TF32 ? 16 : 32; }
constexpr int MAX_SLICES = 6;
constexpr int GEMM_THREADS = 192;
constexpr int NACC = 4;                                          // f32 accumulators, one per digit level
constexpr int ACC_COLS = NACC * TN;                              // 256: one set of accumulators
constexpr int TMEM_COLS = 2 * ACC_COLS;                          // 512: two sets, all of TMEM
constexpr int EPI_BYTES = 4 * 32 * 33 * (int)sizeof(double);     // epilogue transposes, one per warp
constexpr int ROWS_PAD_ALIGN = 128;

struct OzProb {
    CUtensorMap ta, tb;            // A slices / B^T slices, stacked [S][rows_pad][k_pad]
    int a_rows_pad, b_rows_pad;
    int M, N, K;                   // output M x N, reduction K
    const int* ea;                 // per A row exponent
    const int* eb;                 // per B^T row exponent
    double* out;
    int ldo, transposed;           // out[m][n] or out[n][m]
    const double* lam;             // optional Lambda[m][n]
    int ldl;
    int tiles_n, tile_start;
};

struct OzBatch {
    OzProb p[6];
    int count, S, stages, kind, total_tiles;
    unsigned* err;
    long long wait_limit;          // bound of every pipeline wait (SM clock cycles)
    int skip_loads;                // timeout test only: the producer issues no loads
};

using namespace tc;

constexpr uint32_t IDESC = idesc_bf16(TM, TN);
// kind::tf32: A and B tf32 (format 2), f32 accumulator, both K-major.
constexpr uint32_t IDESC_TF32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) |
                                ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ double pow2(int e) {
    return __longlong_as_double((long long)(e + 1023) << 52);   // exact for -1022 <= e <= 1023
}

// ---------------------------------------------------------------------------
// The GEMM kernel
// ---------------------------------------------------------------------------
// Tile t of the batch: its problem and output corner.
__device__ __forceinline__ const OzProb& oz_tile(const OzBatch& b, int t, int& m0, int& n0) {
    int pi = 0;
#pragma unroll 1
    for (int q = 1; q < b.count; ++q)
        if (t >= b.p[q].tile_start) pi = q;
    const OzProb& P = b.p[pi];
    const int u = t - P.tile_start;
    m0 = (u / P.tiles_n) * TM;
    n0 = (u % P.tiles_n) * TN;
    return P;
}

// S (slices per operand) is a template parameter, so that the MMA issuer's
// product loop unrolls into straight-line issues with every descriptor
// offset, accumulator and accumulate flag known at compile time.
template <int KIND, int S>
__global__ void __launch_bounds__(GEMM_THREADS, 1) oz_gemm_kernel(const __grid_constant__ OzBatch b) {
    constexpr int KB = k_block(KIND);   // K elements per 64-byte row
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int NS = b.stages;
    const int STAGE_BYTES = S * (TILE_A_BYTES + TILE_B_BYTES);   // S A tiles, then S B tiles
    uint8_t* sPipe = smem;
    double* sEpi = reinterpret_cast<double*>(smem + (size_t)NS * STAGE_BYTES);
    uint64_t* full = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(sEpi) + EPI_BYTES);
    uint64_t* empty = full + NS;
    uint64_t* tfull = empty + NS;   // [2]: accumulator set complete
    uint64_t* tempty = tfull + 2;   // [2]: accumulator set drained by the epilogue
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    __shared__ volatile int s_fail;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = b.total_tiles;

    if (threadIdx.x == 0) {
        s_fail = 0;
        for (int i = 0; i < NS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&tfull[i], 1);
            mbar_init(&tempty[i], 4);   // one arrival per epilogue warp
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0 && !b.skip_loads) {   // ---- TMA producer ----
            // (skip_loads: nothing is loaded, so no copy is in flight when
            // the MMA issuer's wait for the first stage runs out)
            int it = 0;   // K blocks issued so far, over all of this CTA's tiles
            for (int t = blockIdx.x; t < total && !s_fail; t += gridDim.x) {
                int m0, n0;
                const OzProb& P = oz_tile(b, t, m0, n0);
                const int nkb = (P.K + KB - 1) / KB;
                for (int kb = 0; kb < nkb; ++kb, ++it) {
                    const int st = it % NS;
                    if (it >= NS && !mbar_wait(&empty[st], ((it / NS) - 1) & 1, b.wait_limit)) {
                        s_fail = 1;
                        break;
                    }
                    mbar_expect_tx(&full[st], (uint32_t)STAGE_BYTES);
                    uint8_t* base = sPipe + (size_t)st * STAGE_BYTES;
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        uint8_t* a = base + (size_t)s * TILE_A_BYTES;
                        tma_load_2d(a, &P.ta, &full[st], kb * KB, s * P.a_rows_pad + m0);
                        tma_load_2d(a + BOX_ROWS * 64, &P.ta, &full[st], kb * KB, s * P.a_rows_pad + m0 + BOX_ROWS);
                        tma_load_2d(base + (size_t)S * TILE_A_BYTES + (size_t)s * TILE_B_BYTES, &P.tb, &full[st],
                                    kb * KB, s * P.b_rows_pad + n0);
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {   // ---- MMA issuer ----
            // products of digit level s + u go to accumulator min(s + u, 3)
            int it = 0, j = 0;
#if LC3D_OZ_CLOCKS
            long long c_tempty = 0, c_full = 0, c_issue = 0, c_t = clock64();
#define OZ_T(var) do { const long long n_ = clock64(); var += n_ - c_t; c_t = n_; } while (0)
#else
#define OZ_T(var) do { } while (0)
#endif
            for (int t = blockIdx.x; t < total && !s_fail; t += gridDim.x, ++j) {
                const int buf = j & 1;
                OZ_T(c_issue);
                if (j >= 2 && !mbar_wait(&tempty[buf], ((j >> 1) - 1) & 1, b.wait_limit)) {
                    s_fail = 1;
                    break;
                }
                OZ_T(c_tempty);
                fence_after();
                int m0, n0;
                const OzProb& P = oz_tile(b, t, m0, n0);
                const int nkb = (P.K + KB - 1) / KB;
                const uint32_t accs = tmem + (uint32_t)(buf * ACC_COLS);
                bool ok = true;
                for (int kb = 0; kb < nkb; ++kb, ++it) {
                    const int st = it % NS;
                    OZ_T(c_issue);
                    if (!mbar_wait(&full[st], (it / NS) & 1, b.wait_limit)) {
                        ok = false;
                        break;
                    }
                    OZ_T(c_full);
                    fence_after();
                    const uint32_t a_base = smem_u32(sPipe + (size_t)st * STAGE_BYTES);
                    // descriptors of the stage's first A and B tiles; the
                    // start-address field counts 16-byte units and stays
                    // below 2^14 (shared memory < 256 KiB), so the offsets of
                    // the other tiles and of the second K half add to it
                    // without a carry into the other fields
                    const uint64_t da = umma_desc_sw64(a_base);
                    const uint64_t db = umma_desc_sw64(a_base + (uint32_t)(S * TILE_A_BYTES));
                    const uint32_t later = kb > 0 ? 1u : 0u;   // accumulators already written for this tile
#pragma unroll
                    for (int s = 0; s < S; ++s) {
                        const uint64_t das = da + (uint64_t)((s * TILE_A_BYTES) >> 4);
#pragma unroll
                        for (int u = 0; s + u < S; ++u) {
                            const int lvl = min(s + u, NACC - 1);
                            const uint32_t acc = accs + lvl * TN;
                            const uint64_t dbu = db + (uint64_t)((u * TILE_B_BYTES) >> 4);
                            // the first product of each level in this order is (0, level)
                            const uint32_t first = (s > 0 || u >= NACC) ? 1u : later;
                            // two MMAs per 64-byte row (K = 16 bf16 or 8 tf32), the second 32 bytes on
                            if constexpr (KIND == KIND_TF32) {
                                umma_tf32(acc, das, dbu, IDESC_TF32, first);
                                umma_tf32(acc, das + 2, dbu + 2, IDESC_TF32, 1u);
                            } else {
                                umma_bf16(acc, das, dbu, IDESC, first);
                                umma_bf16(acc, das + 2, dbu + 2, IDESC, 1u);
                            }
                        }
                    }
                    umma_commit(&empty[st]);   // frees the stage once these MMAs have read it
                }
                if (!ok) {
                    s_fail = 1;
                    break;
                }
                umma_commit(&tfull[buf]);      // this tile's accumulators complete
            }
#if LC3D_OZ_CLOCKS
            OZ_T(c_issue);
            if (blockIdx.x < 1024) {
                g_oz_clocks[blockIdx.x][0] = c_tempty;
                g_oz_clocks[blockIdx.x][1] = c_full;
                g_oz_clocks[blockIdx.x][2] = c_issue;
                g_oz_clocks[blockIdx.x][3] = j;
            }
#endif
        }
    } else {   // ---- epilogue: warps 2..5 cover TMEM lanes 32 (warp % 4) .. +31 ----
        const int quarter = warp & 3;
        const int row = quarter * 32 + lane;
        const uint32_t lane_base = (uint32_t)(quarter * 32) << 16;
        double* stg = sEpi + (warp - 2) * 32 * 33;
        constexpr int NA = S < NACC ? S : NACC;   // level accumulators in use
        int j = 0;
#if LC3D_OZ_CLOCKS
        long long e_wait = 0, e_work = 0, e_t = clock64();
#endif
        for (int t = blockIdx.x; t < total && !s_fail; t += gridDim.x, ++j) {
            const int buf = j & 1;
#if LC3D_OZ_CLOCKS
            { const long long n_ = clock64(); e_work += n_ - e_t; e_t = n_; }
#endif
            if (!mbar_wait(&tfull[buf], (j >> 1) & 1, b.wait_limit)) {
                s_fail = 1;
                break;
            }
#if LC3D_OZ_CLOCKS
            { const long long n_ = clock64(); e_wait += n_ - e_t; e_t = n_; }
#endif
            fence_after();
            int m0, n0;
            const OzProb& P = oz_tile(b, t, m0, n0);
            const int m = m0 + row;
            const double sa = (m < P.M) ? pow2(P.ea[m]) : 0.0;
            for (int c0 = 0; c0 < TN; c0 += 32) {
                double v[32];
#pragma unroll
                for (int jj = 0; jj < 32; ++jj) v[jj] = 0.0;
                // exact f32 level sums, added in float64 in level order; the
                // levels' TMEM loads two at a time, one wait per pair
#pragma unroll
                for (int d = 0; d < NA; d += 2) {
                    uint32_t r0[32], r1[32];
                    tmem_ld32(tmem + lane_base + (uint32_t)(buf * ACC_COLS + d * TN + c0), r0);
                    if (d + 1 < NA) tmem_ld32(tmem + lane_base + (uint32_t)(buf * ACC_COLS + (d + 1) * TN + c0), r1);
                    tmem_wait_ld();
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) v[jj] += (double)__uint_as_float(r0[jj]);
                    if (d + 1 < NA) {
#pragma unroll
                        for (int jj = 0; jj < 32; ++jj) v[jj] += (double)__uint_as_float(r1[jj]);
                    }
                }
                // lane l holds the scale of column n0 + c0 + l; rows' scales
                // are the lanes' own (sa), handed round by shuffles
                const int nl = n0 + c0 + lane;
                const double sbl = (nl < P.N) ? pow2(__ldg(P.eb + nl)) : 0.0;
                if (P.transposed) {
                    // out[n][m]: the lanes hold consecutive m, stores coalesce
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) {
                        const int n = n0 + c0 + jj;
                        const double sb = __shfl_sync(0xffffffffu, sbl, jj);
                        if (n >= P.N || m >= P.M) continue;
                        double x = v[jj] * (sa * sb);
                        if (P.lam) x *= P.lam[(size_t)m * P.ldl + n];
                        P.out[(size_t)n * P.ldo + m] = x;
                    }
                } else {
                    // out[m][n]: transpose the warp's 32 x 32 block through
                    // shared memory so the lanes write consecutive n
#pragma unroll
                    for (int jj = 0; jj < 32; ++jj) stg[lane * 33 + jj] = v[jj];
                    __syncwarp();
#pragma unroll 4
                    for (int r = 0; r < 32; ++r) {
                        const int mr = m0 + quarter * 32 + r;
                        const double sar = __shfl_sync(0xffffffffu, sa, r);
                        if (mr >= P.M || nl >= P.N) continue;
                        double x = stg[r * 33 + lane] * (sar * sbl);
                        if (P.lam) x *= P.lam[(size_t)mr * P.ldl + nl];
                        P.out[(size_t)mr * P.ldo + nl] = x;
                    }
                    __syncwarp();
                }
            }
            fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[buf]);   // this set may take the tile after next
        }
#if LC3D_OZ_CLOCKS
        { const long long n_ = clock64(); e_work += n_ - e_t; }
        if (warp == 2 && lane == 0 && blockIdx.x < 1024) {
            g_oz_clocks[blockIdx.x][4] = e_wait;
            g_oz_clocks[blockIdx.x][5] = e_work;
        }
#endif
    }
    fence_before();
    __syncthreads();
    if (s_fail && threadIdx.x == 0) atomicOr(b.err, LC3D_FLAG_TIMEOUT);
    if (warp == 1) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// ---------------------------------------------------------------------------
// Row slicing of float64 data: rows x K (ld) -> S bf16 planes
// [S][rows_pad][k_pad] and per-row exponents. One warp per row.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int exponent_bound(double amax) {
    // smallest e with amax < 2^e (0 for amax == 0)
    if (!(amax > 0)) return 0;
    const long long bits = __double_as_longlong(amax);
    int e = (int)((bits >> 52) & 0x7ff) - 1022;
    return e;
}

struct SliceArgs {
    const double* in[6];
    int ld[6], rows[6], K[6];
    void* out[6];                  // bf16 or float32 (tf32) slices
    int* e[6];
    int row_start[7];              // prefix over problems, in rows
    int count, S, rows_pad, k_pad, kind;
};

__global__ void __launch_bounds__(256) slice_rows_kernel(const __grid_constant__ SliceArgs a) {
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (gw >= a.row_start[a.count]) return;
    int q = 0;
    while (gw >= a.row_start[q + 1]) ++q;
    const int r = gw - a.row_start[q];
    const double* x = a.in[q] + (size_t)r * a.ld[q];
    const int K = a.K[q];
    double amax = 0;
    for (int k = lane; k < K; k += 32) amax = fmax(amax, fabs(x[k]));
#pragma unroll
    for (int o = 16; o; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    const int e = exponent_bound(amax);
    if (lane == 0) a.e[q][r] = e;
    const double scale = pow2(-e);
    const size_t plane = (size_t)a.rows_pad * a.k_pad;
    if (a.kind == KIND_TF32) {   // 10-bit digits, float32 storage (exact in tf32)
        float* o = static_cast<float*>(a.out[q]) + (size_t)r * a.k_pad;
        for (int k = lane; k < a.k_pad; k += 32) {
            double v = k < K ? x[k] * scale : 0.0;   // |v| < 1
            for (int s = 0; s < a.S; ++s) {
                const double d = rint(v * 1024.0);       // digit, exact
                v = v * 1024.0 - d;                      // exact remainder, |v| <= 1/2
                o[s * plane + k] = (float)(d * pow2(-10 * (s + 1)));
            }
        }
        return;
    }
    __nv_bfloat16* o = static_cast<__nv_bfloat16*>(a.out[q]) + (size_t)r * a.k_pad;
    for (int k = lane; k < a.k_pad; k += 32) {
        double v = k < K ? x[k] * scale : 0.0;   // |v| < 1
        for (int s = 0; s < a.S; ++s) {
            const double d = rint(v * 128.0);        // digit, exact
            v = v * 128.0 - d;                       // exact remainder, |v| <= 1/2
            o[s * plane + k] = __float2bfloat16_rn((float)(d * pow2(-7 * (s + 1))));
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

namespace {

// The kernel instantiation of a kind and slice count (1 .. MAX_SLICES).
using OzKernel = void (*)(OzBatch);
template <int KIND>
OzKernel oz_kernel_of(int S) {
    switch (S) {
        case 1: return oz_gemm_kernel<KIND, 1>;
        case 2: return oz_gemm_kernel<KIND, 2>;
        case 3: return oz_gemm_kernel<KIND, 3>;
        case 4: return oz_gemm_kernel<KIND, 4>;
        case 5: return oz_gemm_kernel<KIND, 5>;
        default: return oz_gemm_kernel<KIND, 6>;
    }
}
OzKernel oz_kernel(int kind, int S) { return kind == KIND_TF32 ? oz_kernel_of<KIND_TF32>(S) : oz_kernel_of<KIND_BF16>(S); }

struct MixedState {
    int S, stages, kind, sms;
    size_t smem_max;               // dynamic shared memory the GEMM kernels may use
    int rows_pad, k_pad;           // common padded shape of every operand buffer
    void* fixed[2];                // sliced S2 (M x M) and C (N x N): bf16 or float32 (tf32)
    int* efixed[2];
    void* data[6];                 // per-field data slices
    int* edata[6];
    CUtensorMap map_fixed[2];
    CUtensorMap map_data[6];
};

int make_map(CUtensorMap* m, void* base, int S, int rows_pad, int k_pad, int kind) {
    auto enc = tc_get_encode();
    if (!enc) return LC3D_ERR_CUDA;
    const int esize = kind == KIND_TF32 ? 4 : 2;
    cuuint64_t dims[2] = {(cuuint64_t)k_pad, (cuuint64_t)S * rows_pad};
    cuuint64_t strides[1] = {(cuuint64_t)k_pad * esize};
    cuuint32_t box[2] = {(cuuint32_t)k_block(kind), BOX_ROWS};   // 64-byte rows
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, kind == KIND_TF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                     base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? LC3D_OK : LC3D_ERR_CUDA;
}

uint16_t bf16_bits(float f) {   // exact values only (digits times powers of two)
    uint32_t u;
    memcpy(&u, &f, 4);
    return (uint16_t)(u >> 16);
}

// Slice a float64 matrix on the host exactly like slice_rows_kernel (bf16
// bits into out16, or float32 tf32 values into out32).
void slice_host(const std::vector<double>& A, int rows, int K, int S, int rows_pad, int k_pad, int kind,
                std::vector<uint16_t>& out16, std::vector<float>& out32, std::vector<int>& e) {
    if (kind == KIND_TF32)
        out32.assign((size_t)S * rows_pad * k_pad, 0.0f);
    else
        out16.assign((size_t)S * rows_pad * k_pad, 0);
    e.assign(rows_pad, 0);
    for (int r = 0; r < rows; ++r) {
        double amax = 0;
        for (int k = 0; k < K; ++k) amax = std::fmax(amax, std::fabs(A[(size_t)r * K + k]));
        int er = 0;
        if (amax > 0) {
            int ex;
            std::frexp(amax, &ex);   // amax = f 2^ex, f in [0.5, 1)
            er = ex;
        }
        e[r] = er;
        const int bits = kind == KIND_TF32 ? 10 : 7;
        const double base = std::ldexp(1.0, bits);
        for (int k = 0; k < K; ++k) {
            double v = std::ldexp(A[(size_t)r * K + k], -er);
            for (int s = 0; s < S; ++s) {
                const double d = std::nearbyint(v * base);
                v = v * base - d;
                const size_t o = ((size_t)s * rows_pad + r) * k_pad + k;
                if (kind == KIND_TF32)
                    out32[o] = (float)std::ldexp(d, -bits * (s + 1));
                else
                    out16[o] = bf16_bits((float)std::ldexp(d, -bits * (s + 1)));
            }
        }
    }
}

}  // namespace

int mixed_init(lc3d_ctx* c, int slices, int tf32) {
    if (slices < 1 || slices > MAX_SLICES) return LC3D_ERR_PARAM;
    const int N = c->N, M = c->M;
    if (!tf32 && N > 1000) return LC3D_ERR_SIZE;   // exactness of the leading bf16 product needs K 128^2 < 2^24
    MixedState* ms = new MixedState;
    memset(ms, 0, sizeof(*ms));
    c->mixed = ms;
    ms->S = slices;
    ms->kind = tf32 ? KIND_TF32 : KIND_BF16;
    const int esize = tf32 ? 4 : 2;
    ms->rows_pad = (N + ROWS_PAD_ALIGN - 1) / ROWS_PAD_ALIGN * ROWS_PAD_ALIGN;
    ms->k_pad = (N + 7) / 8 * 8;
    {
        // the opt-in limit of a block less the kernels' static shared memory
        int dev = 0, optin = 0;
        LC3D_CUDA_TRY(cudaGetDevice(&dev));
        LC3D_CUDA_TRY(cudaDeviceGetAttribute(&ms->sms, cudaDevAttrMultiProcessorCount, dev));
        LC3D_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        cudaFuncAttributes fa16{}, fa32{};
        LC3D_CUDA_TRY(cudaFuncGetAttributes(&fa16, oz_kernel(KIND_BF16, slices)));
        LC3D_CUDA_TRY(cudaFuncGetAttributes(&fa32, oz_kernel(KIND_TF32, slices)));
        ms->smem_max = (size_t)optin - std::max(fa16.sharedSizeBytes, fa32.sharedSizeBytes);
    }
    // pipeline stages in what the epilogue buffers, barriers and alignment leave
    ms->stages = (int)((ms->smem_max - EPI_BYTES - 1024 - 256) / ((size_t)slices * (TILE_A_BYTES + TILE_B_BYTES)));
    if (ms->stages > LC3D_OZ_MAX_STAGES) ms->stages = LC3D_OZ_MAX_STAGES;
    if (ms->stages < 2) return LC3D_ERR_PARAM;
    // fixed transform matrices, sliced on the host
    const long long L = N - 1;
    std::vector<double> S2((size_t)M * M), C((size_t)N * N);
    auto sinpi = [](long long r, long long Lq) {
        r %= 2 * Lq;
        if (r < 0) r += 2 * Lq;
        double sign = 1;
        if (r >= Lq) { r -= Lq; sign = -1; }
        if (2 * r > Lq) r = Lq - r;
        return sign * std::sin(M_PI * (double)r / (double)Lq);
    };
    for (int k = 0; k < M; ++k)
        for (int n = 0; n < M; ++n) S2[(size_t)k * M + n] = 2 * sinpi((long long)(k + 1) * (n + 1), L);
    for (int k = 0; k < N; ++k)
        for (int n = 0; n < N; ++n) {
            const long long r = ((long long)k * n) % (2 * L);
            C[(size_t)k * N + n] = ((n == 0 || n == N - 1) ? 1.0 : 2.0) * sinpi(2 * r + L, 2 * L);
        }
    const size_t plane_elems = (size_t)slices * ms->rows_pad * ms->k_pad;
    const std::vector<double>* fx[2] = {&S2, &C};
    const int fdim[2] = {M, N};
    for (int q = 0; q < 2; ++q) {
        std::vector<uint16_t> sl16;
        std::vector<float> sl32;
        std::vector<int> e;
        slice_host(*fx[q], fdim[q], fdim[q], slices, ms->rows_pad, ms->k_pad, ms->kind, sl16, sl32, e);
        const void* src = tf32 ? static_cast<const void*>(sl32.data()) : static_cast<const void*>(sl16.data());
        LC3D_CUDA_TRY(cudaMalloc(&ms->fixed[q], plane_elems * esize));
        LC3D_CUDA_TRY(cudaMemcpy(ms->fixed[q], src, plane_elems * esize, cudaMemcpyHostToDevice));
        LC3D_CUDA_TRY(cudaMalloc(&ms->efixed[q], ms->rows_pad * sizeof(int)));
        LC3D_CUDA_TRY(cudaMemcpy(ms->efixed[q], e.data(), ms->rows_pad * sizeof(int), cudaMemcpyHostToDevice));
        LC3D_TRY(make_map(&ms->map_fixed[q], ms->fixed[q], slices, ms->rows_pad, ms->k_pad, ms->kind));
    }
    for (int f = 0; f < 6; ++f) {
        LC3D_CUDA_TRY(cudaMalloc(&ms->data[f], plane_elems * esize));
        LC3D_CUDA_TRY(cudaMemset(ms->data[f], 0, plane_elems * esize));
        LC3D_CUDA_TRY(cudaMalloc(&ms->edata[f], ms->rows_pad * sizeof(int)));
        LC3D_CUDA_TRY(cudaMemset(ms->edata[f], 0, ms->rows_pad * sizeof(int)));
        LC3D_TRY(make_map(&ms->map_data[f], ms->data[f], slices, ms->rows_pad, ms->k_pad, ms->kind));
    }
    // per-kernel limit: the opt-in maximum, which every slice count's
    // pipeline fits, so contexts with different slice counts can coexist
    LC3D_CUDA_TRY(cudaFuncSetAttribute(oz_kernel(ms->kind, slices), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ms->smem_max));
    return LC3D_OK;
}

void mixed_free(lc3d_ctx* c) {
    MixedState* ms = static_cast<MixedState*>(c->mixed);
    if (!ms) return;
    for (int q = 0; q < 2; ++q) {
        if (ms->fixed[q]) cudaFree(ms->fixed[q]);
        if (ms->efixed[q]) cudaFree(ms->efixed[q]);
    }
    for (int f = 0; f < 6; ++f) {
        if (ms->data[f]) cudaFree(ms->data[f]);
        if (ms->edata[f]) cudaFree(ms->edata[f]);
    }
    delete ms;
    c->mixed = nullptr;
}

// One transform stage for the fields marked in `on`: slice the data
// operands (din[f], rows x K with ld N), then the batched GEMM.
//   data_is_a: the data slices are the A operand (stages 1, 3), else B^T.
int mixed_stage(lc3d_ctx* c, const MixedStageDesc* d, int count, cudaStream_t s) {
    MixedState* ms = static_cast<MixedState*>(c->mixed);
    if (!ms) return LC3D_ERR_STATE;
    // 1. slice the data operands
    SliceArgs sa{};
    memset(&sa, 0, sizeof(sa));
    sa.count = count;
    sa.kind = ms->kind;
    sa.S = ms->S;
    sa.rows_pad = ms->rows_pad;
    sa.k_pad = ms->k_pad;
    int rows = 0;
    for (int q = 0; q < count; ++q) {
        sa.in[q] = d[q].data;
        sa.ld[q] = d[q].ld_data;
        sa.rows[q] = d[q].data_rows;
        sa.K[q] = d[q].K;
        sa.out[q] = ms->data[d[q].field];
        sa.e[q] = ms->edata[d[q].field];
        sa.row_start[q] = rows;
        rows += d[q].data_rows;
    }
    sa.row_start[count] = rows;
    {
        ProfScope ps(c, LC3D_STAGE_SLICE, s);
        slice_rows_kernel<<<(rows * 32 + 255) / 256, 256, 0, s>>>(sa);
        LC3D_CUDA_TRY(cudaGetLastError());
    }
    // 2. the GEMMs
    OzBatch b{};
    memset(&b, 0, sizeof(b));
    b.count = count;
    b.S = ms->S;
    b.kind = ms->kind;
    b.stages = ms->stages;
    b.err = c->err;
    b.wait_limit = c->wait_limit > 0 ? c->wait_limit : WAIT_LIMIT;
    b.skip_loads = c->skip_loads;
    int tiles = 0;
    for (int q = 0; q < count; ++q) {
        OzProb& p = b.p[q];
        const int f = d[q].field, fx = d[q].fixed;   // fixed: 0 = S2, 1 = C
        if (d[q].data_is_a) {
            p.ta = ms->map_data[f];
            p.ea = ms->edata[f];
            p.tb = ms->map_fixed[fx];
            p.eb = ms->efixed[fx];
        } else {
            p.ta = ms->map_fixed[fx];
            p.ea = ms->efixed[fx];
            p.tb = ms->map_data[f];
            p.eb = ms->edata[f];
        }
        p.a_rows_pad = p.b_rows_pad = ms->rows_pad;
        p.M = d[q].M;
        p.N = d[q].N;
        p.K = d[q].K;
        p.out = d[q].out;
        p.ldo = d[q].ldo;
        p.transposed = d[q].transposed;
        p.lam = d[q].lam;
        p.ldl = d[q].ldl;
        p.tiles_n = (p.N + TN - 1) / TN;
        p.tile_start = tiles;
        tiles += ((p.M + TM - 1) / TM) * p.tiles_n;
    }
    b.total_tiles = tiles;
    if (!tiles) return LC3D_OK;
    const size_t smem =
        (size_t)ms->stages * ms->S * (TILE_A_BYTES + TILE_B_BYTES) + EPI_BYTES + 1024 + 256;
    const int grid = std::min(tiles, std::max(ms->sms, 1));   // persistent: one CTA per SM
    ProfScope ps(c, LC3D_STAGE_TRANSFORM, s);
    oz_kernel(ms->kind, ms->S)<<<grid, GEMM_THREADS, smem, s>>>(b);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

#if LC3D_OZ_CLOCKS
extern "C" int lc3d_debug_oz_clocks(long long* host) {
    LC3D_CUDA_TRY(cudaDeviceSynchronize());
    LC3D_CUDA_TRY(cudaMemcpyFromSymbol(host, g_oz_clocks, sizeof(g_oz_clocks)));
    return LC3D_OK;
}
#endif

PFN_cuTensorMapEncodeTiled_v12000 tc_get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}
