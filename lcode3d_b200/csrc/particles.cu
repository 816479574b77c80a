// Plasma particle kernels: field-free estimate, pusher with TSC field gather,
// coarse->fine interpolation with deterministic 9-point TSC deposition.
//
// Reference: lcode.py:369-391 (move_estimate_wo_fields), 396-449 (weights,
// interp9, deposit9), 576-689 (mix, coarse_to_fine, deposit_kernel,
// deposit), 704-823 (move_smart_kernel, move_smart).
//
// Deposition is deterministic. The reference adds every fine particle's 36
// contributions with float64 atomics in an unspecified order. Here every
// contribution c is split exactly into two integers,
//     c = hi * 2^-24 + lo * 2^-76 + (rounding below 2^-77),
// which are summed with 64-bit integer adds; integer addition is associative,
// so the sums do not depend on the order in which threads add them, and the
// final conversion rounds once. Each CTA owns a tile of 8 (or 4, 16) fine
// lattice rows x 32 columns and accumulates into a shared-memory window
// placed on the bounding box of its particles' cells (float64 sums in a
// fixed order); particles whose stencil falls outside the window (strongly
// displaced plasma) add straight to the global accumulators. The window is
// then flushed with 64-bit integer reductions into global memory, and a
// finalize pass converts to float64, adds the ion background and clears the
// accumulators for the next call.

#include <mutex>

#include "lc3d_internal.cuh"

namespace {

constexpr int DEP_WORDS_PER_CELL = 8;   // accumulator planes: 4 fields x (hi, lo)

// ---------------------------------------------------------------------------
// TSC weights, lcode.py:396-418. Order MP 0P PP M0 00 P0 MM 0M PM.
// ---------------------------------------------------------------------------
struct Tsc {
    int i, j;
    double wxM, wx0, wxP, wyM, wy0, wyP;
};

// Centre cell (i, j) and offset from the cell centre, lcode.py:404-406.
// x / h correctly rounded from the reciprocal: q0 = x (1/h) is within an ulp,
// one Newton correction with the exact residual fma(-q0, h, x) rounds it.
__device__ __forceinline__ double div_h(double x, double h, double inv_h) {
    const double q0 = x * inv_h;
    return fma(fma(-q0, h, x), inv_h, q0);
}

__device__ __forceinline__ void tsc_cell(double x, double y, int N, double h, double inv_h, int& i, int& j,
                                         double& xl, double& yl) {
    double x_h = div_h(x, h, inv_h) + .5, y_h = div_h(y, h, inv_h) + .5;
    double fx = floor(x_h), fy = floor(y_h);
    xl = x_h - fx - .5;
    yl = y_h - fy - .5;
    // out-of-range positions map to an invalid index without UB in the cast
    fx = fmin(fmax(fx, -1.0e6), 1.0e6);
    fy = fmin(fmax(fy, -1.0e6), 1.0e6);
    i = (int)fx + N / 2;
    j = (int)fy + N / 2;
}

// Quadratic-spline weights along one axis, lcode.py:410-412.
__device__ __forceinline__ void tsc_axis(double l, double& wM, double& w0, double& wP) {
    w0 = .75 - l * l;
    wP = (.5 + l) * (.5 + l) / 2;
    wM = (.5 - l) * (.5 - l) / 2;
}

__device__ __forceinline__ Tsc tsc_weights(double x, double y, int N, double h, double inv_h) {
    Tsc t;
    double xl, yl;
    tsc_cell(x, y, N, h, inv_h, t.i, t.j, xl, yl);
    tsc_axis(xl, t.wxM, t.wx0, t.wxP);
    tsc_axis(yl, t.wyM, t.wy0, t.wyP);
    return t;
}

__device__ __forceinline__ bool tsc_in_grid(const Tsc& t, int N) {
    return t.i >= 1 && t.i <= N - 2 && t.j >= 1 && t.j <= N - 2;
}

// interp9, lcode.py:421-430 (same summation order), in two halves: the
// nine values a field is read at, then their weighted sum. The pusher issues
// all six fields' gathers before any sum, so the 54 loads of a particle are
// in flight together (one round of memory latency instead of several:
// 0.0416 -> 0.0342 ms per xi step at 641^2).
__device__ __forceinline__ void gather9(const double* __restrict__ a, const Tsc& t, int N, double (&v)[9]) {
    const double* r0 = a + (size_t)(t.i - 1) * N + t.j;   // row i-1
    const double* r1 = r0 + N;
    const double* r2 = r1 + N;
    v[0] = r0[+1]; v[1] = r1[+1]; v[2] = r2[+1];
    v[3] = r0[0];  v[4] = r1[0];  v[5] = r2[0];
    v[6] = r0[-1]; v[7] = r1[-1]; v[8] = r2[-1];
}
__device__ __forceinline__ double sum9(const double (&v)[9], const Tsc& t) {
    return v[0] * (t.wxM * t.wyP) + v[1] * (t.wx0 * t.wyP) + v[2] * (t.wxP * t.wyP) +
           v[3] * (t.wxM * t.wy0) + v[4] * (t.wx0 * t.wy0) + v[5] * (t.wxP * t.wy0) +
           v[6] * (t.wxM * t.wyM) + v[7] * (t.wx0 * t.wyM) + v[8] * (t.wxP * t.wyM);
}

// ---------------------------------------------------------------------------
// Field-free estimate, lcode.py:369-391 (reflection with >= and <=).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void estimate_one(double m, double xi0, double yi0, double xo, double yo,
                                             double px, double py, double pz, double dxi, double rb,
                                             double& ex, double& ey) {
    double x = xi0 + xo, y = yi0 + yo;
    double gamma_m = sqrt(m * m + pz * pz + px * px + py * py);
    x += px / (gamma_m - pz) * dxi;
    y += py / (gamma_m - pz) * dxi;
    if (x >= +rb) x = +2 * rb - x;
    if (x <= -rb) x = -2 * rb - x;
    if (y >= +rb) y = +2 * rb - y;
    if (y <= -rb) y = -2 * rb - y;
    ex = x - xi0;
    ey = y - yi0;
}

__global__ void __launch_bounds__(256) move_estimate_kernel(EstimateArgs a) {
    pdl_wait();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    double ex, ey;
    estimate_one(a.m[k], a.x_init[k], a.y_init[k], a.x_prev[k], a.y_prev[k], a.px[k], a.py[k],
                 a.pz[k], a.dxi, a.rb, ex, ey);
    a.out_x[k] = ex;
    a.out_y[k] = ey;
}

// One coarse particle's seven deposit inputs as 64 contiguous bytes, so that
// the deposition gathers a coarse neighbour with four 16-byte loads instead
// of seven scattered 8-byte ones.
__device__ __forceinline__ void store_packed(double* p, double x, double y, double m, double q, double px,
                                             double py, double pz) {
    double2* p2 = reinterpret_cast<double2*>(p);
    p2[0] = make_double2(x, y);
    p2[1] = make_double2(m, q);
    p2[2] = make_double2(px, py);
    p2[3] = make_double2(pz, 0.0);
}

// ---------------------------------------------------------------------------
// Pusher, lcode.py:704-793. One thread per coarse particle. With est_x ==
// NULL the field-free estimate of lcode.py:369-391 is computed inline (the
// predictor pass of step()).
// ---------------------------------------------------------------------------
#ifndef LC3D_MOVE_THREADS
#define LC3D_MOVE_THREADS 64    // the gathers in flight take ~150 registers a thread: small CTAs keep
#endif                          // 42,025 particles (641^2) in one wave (64 measured a little ahead of 128)
__global__ void __launch_bounds__(LC3D_MOVE_THREADS, 1) move_smart_kernel(MoveArgs a) {
    pdl_wait();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const double m = a.m[k], q = a.q[k];
    const double xi0 = a.x_init[k], yi0 = a.y_init[k];
    const double opx = a.px_prev[k], opy = a.py_prev[k], opz = a.pz_prev[k];
    double x_offt = a.x_prev[k], y_offt = a.y_prev[k];
    double ex, ey;
    if (a.est_x) {
        ex = a.est_x[k];
        ey = a.est_y[k];
    } else {
        estimate_one(m, xi0, yi0, x_offt, y_offt, opx, opy, opz, a.dxi, a.rb, ex, ey);
    }
    double x_half = xi0 + (x_offt + ex) / 2;
    double y_half = yi0 + (y_offt + ey) / 2;
    Tsc t = tsc_weights(x_half, y_half, a.N, a.h, a.inv_h);
    if (!tsc_in_grid(t, a.N)) {
        // the reference would read out of bounds here; flag and keep prev
        atomicOr(a.err, LC3D_FLAG_WINDOW);
        a.out_x[k] = x_offt;
        a.out_y[k] = y_offt;
        a.out_px[k] = opx;
        a.out_py[k] = opy;
        a.out_pz[k] = opz;
        if (a.out_packed) store_packed(a.out_packed + 8 * (size_t)k, x_offt, y_offt, m, q, opx, opy, opz);
        return;
    }
    double g[6][9];
#pragma unroll
    for (int f = 0; f < 6; ++f) gather9(a.F[f], t, a.N, g[f]);
    const double Ex = sum9(g[0], t), Ey = sum9(g[1], t);
    const double Ez = sum9(g[2], t), Bx = sum9(g[3], t);
    const double By = sum9(g[4], t), Bz = sum9(g[5], t);

    double px = opx, py = opy, pz = opz;
    double dpx, dpy, dpz;
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        double gamma_m = sqrt(m * m + pz * pz + px * px + py * py);
        double vx = px / gamma_m, vy = py / gamma_m, vz = pz / gamma_m;
        double factor_1 = q * a.dxi / (1 - pz / gamma_m);
        dpx = factor_1 * (Ex + vy * Bz - vz * By);
        dpy = factor_1 * (Ey - vx * Bz + vz * Bx);
        dpz = factor_1 * (Ez + vx * By - vy * Bx);
        px = opx + dpx / 2;
        py = opy + dpy / 2;
        pz = opz + dpz / 2;
    }
    double gamma_m = sqrt(m * m + pz * pz + px * px + py * py);
    x_offt += px / (gamma_m - pz) * a.dxi;
    y_offt += py / (gamma_m - pz) * a.dxi;
    px = opx + dpx;
    py = opy + dpy;
    pz = opz + dpz;

    const double rb = a.rb;
    double x = xi0 + x_offt, y = yi0 + y_offt;
    if (x > +rb) { x = +2 * rb - x; x_offt = x - xi0; px = -px; }
    if (x < -rb) { x = -2 * rb - x; x_offt = x - xi0; px = -px; }
    if (y > +rb) { y = +2 * rb - y; y_offt = y - yi0; py = -py; }
    if (y < -rb) { y = -2 * rb - y; y_offt = y - yi0; py = -py; }
    a.out_x[k] = x_offt;
    a.out_y[k] = y_offt;
    a.out_px[k] = px;
    a.out_py[k] = py;
    a.out_pz[k] = pz;
    if (a.out_packed) store_packed(a.out_packed + 8 * (size_t)k, x_offt, y_offt, m, q, px, py, pz);
}

// ---------------------------------------------------------------------------
// Exact fixed-point split of a contribution.
// hi = round(c * 2^24) through the 1.5*2^28 magic constant (valid for
// |c| < 2^27); r = c - hi*2^-24 is exact and |r| <= 2^-25, so
// lo = round(r * 2^76) through 1.5*2^-24. The bit-pattern difference of two
// doubles in the same (or the adjacent upper) binade counts ulps exactly.
// ---------------------------------------------------------------------------
constexpr double FX_MAX = 0x1p+27;

__device__ __forceinline__ void fx_split(double c, long long& hi, long long& lo) {
    const double MH = 0x1.8p+28;                      // 1.5 * 2^28
    const double ML = 0x1.8p-24;                      // 1.5 * 2^-24
    double t = c + MH;
    hi = __double_as_longlong(t) - __double_as_longlong(MH);
    double r = c - (t - MH);
    double t2 = r + ML;
    lo = __double_as_longlong(t2) - __double_as_longlong(ML);
}

__device__ __forceinline__ double fx_value(long long hi, long long lo) {
    return (double)hi * 0x1p-24 +
           (double)lo * 0x1p-76;
}

// One fine particle: coarse->fine mix (lcode.py:591-621) and the deposit
// quantities (lcode.py:651-655).
struct FineParticle {
    double x, y, dro, djx, djy, djz;
};

// Deposit quantities from the mixed coarse values (lcode.py:651-655).
__device__ __forceinline__ void particle_values(FineParticle& p, double m, double q, double px, double py,
                                                double pz) {
    const double gamma_m = sqrt(m * m + px * px + py * py + pz * pz);
    // the two quotients by gamma_m from one reciprocal, each corrected by
    // its exact residual (div_h): the reference's divisions, one division
    // sequence fewer per particle (the algebraically equal single division
    // q / (gamma_m - pz) measured only 0.5 % faster and departs from the
    // reference's rounding)
    const double inv_g = 1.0 / gamma_m;
    p.dro = q / (1 - div_h(pz, gamma_m, inv_g));
    const double dro_g = div_h(p.dro, gamma_m, inv_g);
    p.djx = px * dro_g;
    p.djy = py * dro_g;
    p.djz = pz * dro_g;
}

__device__ __forceinline__ FineParticle fine_particle(const DepositArgs& a, int fi, int fj) {
    const double ipi = a.inf_prev[fi], ini = a.inf_next[fi];
    const double ipj = a.inf_prev[fj], inj = a.inf_next[fj];
    const double A = ipi * ipj, B = ipi * inj, C = ini * ipj, D = ini * inj;
    const int pi = a.idx_prev[fi], ni = a.idx_next[fi];
    const int pj = a.idx_prev[fj], nj = a.idx_next[fj];
    const int kA = pi * a.Nc + pj, kB = pi * a.Nc + nj, kC = ni * a.Nc + pj, kD = ni * a.Nc + nj;
    FineParticle p;
    if (a.packed) {   // the same values and arithmetic, four 16-byte loads per neighbour
        const double2* P2 = reinterpret_cast<const double2*>(a.packed);
        double2 w[4][4];
        const int ks[4] = {kA, kB, kC, kD};
#pragma unroll
        for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int h = 0; h < 4; ++h) w[c][h] = __ldg(P2 + 4 * (size_t)ks[c] + h);
#define LC3D_MIX4(h, comp) (A * w[0][h].comp + B * w[1][h].comp + C * w[2][h].comp + D * w[3][h].comp)
        p.x = a.fine_grid[fi] + LC3D_MIX4(0, x);
        p.y = a.fine_grid[fj] + LC3D_MIX4(0, y);
        particle_values(p, a.sf * LC3D_MIX4(1, x), a.sf * LC3D_MIX4(1, y), a.sf * LC3D_MIX4(2, x),
                        a.sf * LC3D_MIX4(2, y), a.sf * LC3D_MIX4(3, x));
#undef LC3D_MIX4
        return p;
    }
#define LC3D_MIX(arr) (A * __ldg(arr + kA) + B * __ldg(arr + kB) + C * __ldg(arr + kC) + D * __ldg(arr + kD))
    p.x = a.fine_grid[fi] + LC3D_MIX(a.x_offt);
    p.y = a.fine_grid[fj] + LC3D_MIX(a.y_offt);
    particle_values(p, a.sf * LC3D_MIX(a.m), a.sf * LC3D_MIX(a.q), a.sf * LC3D_MIX(a.px), a.sf * LC3D_MIX(a.py),
                    a.sf * LC3D_MIX(a.pz));
#undef LC3D_MIX
    return p;
}

__device__ __forceinline__ void fx_add(unsigned long long* hi_plane, unsigned long long* lo_plane, size_t cell,
                                       double c) {
    long long hi, lo;
    fx_split(c, hi, lo);
    atomicAdd(hi_plane + cell, (unsigned long long)hi);
    atomicAdd(lo_plane + cell, (unsigned long long)lo);
}

// ---------------------------------------------------------------------------
// Deposition kernel. A CTA of TI warps deposits TI fine-lattice rows x 32
// columns; one thread per fine particle, then one per (2 x 2 block, field).
//  1. Coarse->fine mix in two separable passes (the equivalent formula noted
//     beside the reference's make_plasma, lcode.py:554-556). Each warp holds
//     one fine row fi of the tile; it first mixes the two coarse rows of fi,
//         R[c] = inf_prev[fi] Q[prev_i][c] + inf_next[fi] Q[next_i][c],
//     for every coarse column c its 32 fine columns use (7 quantities, a
//     warp-private shared-memory table), and each lane then mixes two
//     entries, Q = inf_prev[fj] R[prev_j] + inf_next[fj] R[next_j]: 14
//     float64 operations and 8 shared loads per particle, no CTA barrier. A
//     tile whose columns span more than DEP2_CMAX coarse columns (other
//     coarseness / fineness settings, or arbitrary virt_params) mixes per
//     particle from global memory (fine_particle). Then the deposit values
//     (lcode.py:651-655) and the TSC cell, staged in shared memory; the CTA's
//     bounding box of cells places the window.
//  2. One thread per (2 x 2 block of fine particles, field). If the block's
//     centre cells span at most 2 x 2 cells -- neighbouring fine particles
//     are interpolated from the same coarse particles and move together --
//     its four TSC stencils are summed in a fixed order into a register
//     patch: 3 x 3 when all four lie in one cell, else 4 x 4. Tiles start
//     `a.fine_off` fine particles before the lattice origin: with an even
//     fineness the lattice has two particles per cell and axis and the fine
//     index pairs (odd, even) share a cell, so with an offset of 1 every
//     block of an undisturbed lattice lies in one cell (9 window entries and
//     36 products per field instead of 16 and 64). Blocks claim their patch's
//     corner cell (atomicMax of the block index: the winner does not depend
//     on timing); winners add their patches to the window in 9 or 16
//     barrier-separated steps, one patch entry per step, so in each step
//     every window cell has at most one writer and its summation order is
//     fixed. Losing blocks (two on one corner) and blocks that span more
//     cells or leave the window add their contributions straight to the
//     global accumulators through the exact split.
//  3. Each touched window cell is split once into fixed point and added to
//     the global accumulators.
// ---------------------------------------------------------------------------
#ifndef LC3D_DEP2_CLOCKS
#define LC3D_DEP2_CLOCKS 0
#endif
constexpr int DEP2_CMAX = 16;               // coarse columns one row table holds
constexpr int DEP2_WC = 32;                 // window columns (cells); rows: 2 per fine row of the tile

// Dynamic shared memory of a tile of `ti` fine rows x 32 columns.
constexpr size_t dep2_smem(int ti) {
    return (size_t)ti * DEP2_CMAX * 8 * sizeof(double)              // row tables
           + (size_t)ti * 32 * (6 * sizeof(double) + sizeof(int))   // staging
           + (size_t)4 * (2 * ti * DEP2_WC) * sizeof(double)        // window, 4 fields
           + (size_t)(2 * ti * DEP2_WC) * sizeof(int);               // anchor claims
}

#if LC3D_DEP2_CLOCKS
constexpr int DEP2_NCLK = 6;
__device__ long long g_dep2_clocks[16384][DEP2_NCLK];
#define DEP2_CLK(k)                                                                      \
    do {                                                                                 \
        if (threadIdx.x == 0) {                                                          \
            const int cta = blockIdx.y * gridDim.x + blockIdx.x;                         \
            if (cta < 16384) g_dep2_clocks[cta][k] = clock64() - clk0;                   \
        }                                                                                \
    } while (0)
#else
#define DEP2_CLK(k) do { } while (0)
#endif

// TSC weights of staged particle k from its staged cell offsets (xl at
// s_pos[k], yl at s_pos[threads + k]). Staging the six weights instead
// measured slower (shared-memory traffic against 12 float64 operations).
__device__ __forceinline__ void staged_weights(const double* s_pos, int threads, int k, double& wxM, double& wx0,
                                               double& wxP, double& wyM, double& wy0, double& wyP) {
    tsc_axis(s_pos[k], wxM, wx0, wxP);
    tsc_axis(s_pos[threads + k], wyM, wy0, wyP);
}

// Two of the seven coarse quantities of coarse particle k as a pair: h = 0
// (x_offt, y_offt), 1 (m, q), 2 (px, py), 3 (pz, 0).
__device__ __forceinline__ double2 coarse_pair(const DepositArgs& a, int k, int h) {
    if (a.packed) return __ldg(reinterpret_cast<const double2*>(a.packed) + 4 * (size_t)k + h);
    switch (h) {
        case 0: return make_double2(__ldg(a.x_offt + k), __ldg(a.y_offt + k));
        case 1: return make_double2(__ldg(a.m + k), __ldg(a.q + k));
        case 2: return make_double2(__ldg(a.px + k), __ldg(a.py + k));
        default: return make_double2(__ldg(a.pz + k), 0.0);
    }
}

// TI fine rows x 32 fine columns per CTA, one warp per row (TI = 4, 8, 16:
// 8, 4 or 2 resident CTAs per SM at 64 registers).
template <int TI>
__device__ __forceinline__ void deposit_tile(const DepositArgs& a, int tile_x, int tile_y) {
    constexpr int DEP2_TI = TI;
    constexpr int DEP2_THREADS = DEP2_TI * 32;
    constexpr int DEP2_BLOCKS = DEP2_THREADS / 4;
    constexpr int DEP2_WR = 2 * DEP2_TI;   // window rows (cells)
    constexpr int DEP2_WIN = DEP2_WR * DEP2_WC;
    static_assert(DEP2_TI % 2 == 0 && DEP2_TI <= 32, "2 x 2 blocks, at most 32 warps");
#if LC3D_DEP2_CLOCKS
    const long long clk0 = clock64();
#endif
    extern __shared__ double smem_f64[];
    double2* s_R = reinterpret_cast<double2*>(smem_f64);                 // [DEP2_TI][DEP2_CMAX][4]
    double* s_pos = smem_f64 + DEP2_TI * DEP2_CMAX * 8;                  // cell offsets xl, yl: [2][DEP2_THREADS]
    double* s_xl = s_pos;
    double* s_yl = s_xl + DEP2_THREADS;
    double* s_v = s_yl + DEP2_THREADS;                                   // [4][DEP2_THREADS]
    double* s_win = s_v + 4 * DEP2_THREADS;                              // [4][DEP2_WIN]
    int* s_claim = reinterpret_cast<int*>(s_win + 4 * DEP2_WIN);         // [DEP2_WIN]
    int* s_cell = s_claim + DEP2_WIN;                                    // [DEP2_THREADS]: i << 16 | j, or -1
    __shared__ int s_bb[4];                                              // imin imax jmin jmax
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) {
        s_bb[0] = s_bb[2] = 1 << 30;
        s_bb[1] = s_bb[3] = -(1 << 30);
    }
    for (int w = t; w < 4 * DEP2_WIN; w += DEP2_THREADS) s_win[w] = 0.0;
    for (int w = t; w < DEP2_WIN; w += DEP2_THREADS) s_claim[w] = -1;
    const int N = a.N;
    const size_t NN = a.plane;
    pdl_wait();   // global memory from here on
    DEP2_CLK(0);

    // ---- phase 1: one fine particle per thread; warp = fine row ----
    {
        const int fi = tile_y * DEP2_TI + warp - a.fine_off;
        const int fj = tile_x * 32 + lane - a.fine_off;
        const bool row_ok = fi >= 0 && fi < a.Nf, col_ok = fj >= 0 && fj < a.Nf;
        // every input of the particle first (independent loads), then the
        // coarse rows of the row table
        int pi = 0, ni = 0, pj = 0, nj = 0;
        double ipi = 0, ini = 0, fgi = 0, ipj = 0, inj = 0, fgj = 0;
        if (row_ok) {
            pi = a.idx_prev[fi];
            ni = a.idx_next[fi];
            ipi = a.inf_prev[fi];
            ini = a.inf_next[fi];
            fgi = a.fine_grid[fi];
        }
        if (col_ok) {
            pj = a.idx_prev[fj];
            nj = a.idx_next[fj];
            ipj = a.inf_prev[fj];
            inj = a.inf_next[fj];
            fgj = a.fine_grid[fj];
        }
        const bool row_idx = pi >= 0 && pi < a.Nc && ni >= 0 && ni < a.Nc;
        const bool col_idx = pj >= 0 && pj < a.Nc && nj >= 0 && nj < a.Nc;
        // the coarse columns of the tile (the same in every warp)
        const int c0 = __reduce_min_sync(0xffffffffu, col_ok ? (col_idx ? min(pj, nj) : -(1 << 30)) : 1 << 30);
        const int c1 = __reduce_max_sync(0xffffffffu, col_ok ? (col_idx ? max(pj, nj) : 1 << 30) : -(1 << 30));
        const int nc = c1 - c0 + 1;
        const bool staged = c0 >= 0 && nc >= 1 && nc <= DEP2_CMAX;
        double2* R = s_R + warp * DEP2_CMAX * 4;
        if (staged && row_ok && row_idx) {
            for (int it = lane; it < nc * 4; it += 32) {
                const int jc = it >> 2, h = it & 3;
                const double2 qp = coarse_pair(a, pi * a.Nc + c0 + jc, h);
                const double2 qn = coarse_pair(a, ni * a.Nc + c0 + jc, h);
                R[it] = make_double2(ipi * qp.x + ini * qn.x, ipi * qp.y + ini * qn.y);
            }
        }
        __syncwarp();
        int cell = -1, i = 1 << 30, j = 1 << 30;
        if (row_ok && col_ok) {
            if (!(row_idx && col_idx)) {
                atomicOr(a.err, LC3D_FLAG_WINDOW);
            } else {
                FineParticle f;
                if (staged) {
                    const double2* Rp = R + (pj - c0) * 4;
                    const double2* Rn = R + (nj - c0) * 4;
                    double2 q[4];
#pragma unroll
                    for (int h = 0; h < 4; ++h) {
                        const double2 rp = Rp[h], rn = Rn[h];
                        q[h] = make_double2(ipj * rp.x + inj * rn.x, ipj * rp.y + inj * rn.y);
                    }
                    f.x = fgi + q[0].x;
                    f.y = fgj + q[0].y;
                    particle_values(f, a.sf * q[1].x, a.sf * q[1].y, a.sf * q[2].x, a.sf * q[2].y,
                                    a.sf * q[3].x);
                } else {
                    f = fine_particle(a, fi, fj);
                }
                double xl, yl;
                tsc_cell(f.x, f.y, N, a.h, a.inv_h, i, j, xl, yl);
                const double vmax = fmax(fmax(fabs(f.dro), fabs(f.djx)), fmax(fabs(f.djy), fabs(f.djz)));
                if (!(i >= 1 && i <= N - 2 && j >= 1 && j <= N - 2)) {
                    atomicOr(a.err, LC3D_FLAG_WINDOW);
                } else if (!(vmax < FX_MAX)) {   // also catches NaN
                    atomicOr(a.err, LC3D_FLAG_NONFINITE);
                } else {
                    cell = (i << 16) | j;
                }
                s_xl[t] = xl;
                s_yl[t] = yl;
                s_v[t] = f.dro;
                s_v[DEP2_THREADS + t] = f.djx;
                s_v[2 * DEP2_THREADS + t] = f.djy;
                s_v[3 * DEP2_THREADS + t] = f.djz;
            }
        }
        s_cell[t] = cell;
        // warp bounding box of the cells (one redux instruction each)
        const int imin = __reduce_min_sync(0xffffffffu, cell >= 0 ? i : 1 << 30);
        const int imax = __reduce_max_sync(0xffffffffu, cell >= 0 ? i : -(1 << 30));
        const int jmin = __reduce_min_sync(0xffffffffu, cell >= 0 ? j : 1 << 30);
        const int jmax = __reduce_max_sync(0xffffffffu, cell >= 0 ? j : -(1 << 30));
        __syncthreads();   // s_bb initialised, window and claims cleared
        if (lane == 0 && imin <= imax) {
            atomicMin(&s_bb[0], imin);
            atomicMax(&s_bb[1], imax);
            atomicMin(&s_bb[2], jmin);
            atomicMax(&s_bb[3], jmax);
        }
    }
    __syncthreads();
    DEP2_CLK(1);

    // ---- phase 2: one (2 x 2 block, field) per thread ----
    const int f = t / DEP2_BLOCKS, blk = t % DEP2_BLOCKS;
    const int p0 = (blk >> 4) * 64 + (blk & 15) * 2;   // top-left particle of the block
    const int pidx[4] = {p0, p0 + 1, p0 + 32, p0 + 33};
    int ci[4], cj[4];
    bool ok[4];
    int i0 = 1 << 30, i1 = -(1 << 30), j0 = 1 << 30, j1 = -(1 << 30);
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int c = s_cell[pidx[p]];
        ok[p] = c >= 0;
        ci[p] = c >> 16;
        cj[p] = c & 0xffff;
        if (ok[p]) {
            i0 = min(i0, ci[p]);
            i1 = max(i1, ci[p]);
            j0 = min(j0, cj[p]);
            j1 = max(j1, cj[p]);
        }
    }
    const int oi = s_bb[0] - 1, oj = s_bb[2] - 1;   // window origin (cells)
    const bool patch = i0 <= i1 && i1 - i0 <= 1 && j1 - j0 <= 1 && i0 + 2 - oi < DEP2_WR && j0 + 2 - oj < DEP2_WC;
    const bool one = patch && i1 == i0 && j1 == j0;   // all four in one cell: a 3 x 3 patch
    const int ar = i0 - 1, ac = j0 - 1;             // the patch's corner cell
    const int r0 = ar - oi, c0w = ac - oj;          // ... in window coordinates
    if (patch && f == 0) atomicMax(&s_claim[r0 * DEP2_WC + c0w], blk);
    __syncthreads();
    const bool winner = patch && s_claim[r0 * DEP2_WC + c0w] == blk;
    unsigned long long* ghi = a.acc + (2 * f) * NN;
    unsigned long long* glo = ghi + NN;
    const double* vf = s_v + f * DEP2_THREADS;
    double acc[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) acc[k] = 0.0;
    if (one) {
        // the four stencils on the same 3 x 3 cells: entry (r, c) of the
        // patch is acc[r * 4 + c], r, c < 3
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            if (!ok[p]) continue;
            double wx[3], wy[3];
            staged_weights(s_pos, DEP2_THREADS, pidx[p], wx[0], wx[1], wx[2], wy[0], wy[1], wy[2]);
            const double v = vf[pidx[p]];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const double vx = v * wx[r];
#pragma unroll
                for (int c = 0; c < 3; ++c) acc[r * 4 + c] = fma(vx, wy[c], acc[r * 4 + c]);
            }
        }
    } else if (patch) {
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            if (!ok[p]) continue;
            double wxM, wx0, wxP, wyM, wy0, wyP;
            staged_weights(s_pos, DEP2_THREADS, pidx[p], wxM, wx0, wxP, wyM, wy0, wyP);
            const bool si = ci[p] != i0, sj = cj[p] != j0;
            const double wx4[4] = {si ? 0.0 : wxM, si ? wxM : wx0, si ? wx0 : wxP, si ? wxP : 0.0};
            const double wy4[4] = {sj ? 0.0 : wyM, sj ? wyM : wy0, sj ? wy0 : wyP, sj ? wyP : 0.0};
            const double v = vf[pidx[p]];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const double vx = v * wx4[r];
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r * 4 + c] = fma(vx, wy4[c], acc[r * 4 + c]);
            }
        }
    } else {
#pragma unroll 1
        for (int p = 0; p < 4; ++p) {
            const int c = s_cell[pidx[p]];
            if (c < 0) continue;
            const int pi = c >> 16, pj = c & 0xffff;
            double wx[3], wy[3];
            staged_weights(s_pos, DEP2_THREADS, pidx[p], wx[0], wx[1], wx[2], wy[0], wy[1], wy[2]);
            const double v = vf[pidx[p]];
#pragma unroll
            for (int di = 0; di < 3; ++di)
#pragma unroll
                for (int dj = 0; dj < 3; ++dj)
                    fx_add(ghi, glo, (size_t)(pi + di - 1) * N + (pj + dj - 1), v * (wx[di] * wy[dj]));
        }
    }
    if (patch && !winner) {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (acc[r * 4 + c] != 0.0) fx_add(ghi, glo, (size_t)(ar + r) * N + (ac + c), acc[r * 4 + c]);
    }
    DEP2_CLK(2);
    // winners add their patches, one entry per barrier-separated step; a
    // CTA whose blocks all lie in single cells needs only the 9 entries of
    // a 3 x 3 patch
    double* fw = s_win + f * DEP2_WIN + (winner ? r0 * DEP2_WC + c0w : 0);
    if (__syncthreads_or(patch && !one)) {   // uniform over the CTA
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            if (winner && acc[k] != 0.0) fw[(k >> 2) * DEP2_WC + (k & 3)] += acc[k];
            __syncthreads();
        }
    } else {
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            const int k = (e / 3) * 4 + e % 3;
            if (winner && acc[k] != 0.0) fw[(k >> 2) * DEP2_WC + (k & 3)] += acc[k];
            __syncthreads();
        }
    }
    DEP2_CLK(3);

    // ---- phase 3: split each touched window cell once, add to global ----
    if (s_bb[0] <= s_bb[1]) {
        // lane = window column (the window is 32 cells wide), warps step over
        // the rows of each field: consecutive lanes add to consecutive cells
        const int ni = min(s_bb[1] + 2 - oi, DEP2_WR), nj = min(s_bb[3] + 2 - oj, DEP2_WC);
        static_assert(DEP2_WC == 32, "one lane per window column");
        if (lane < nj) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                unsigned long long* hi = a.acc + (2 * q) * NN;
                for (int r = warp; r < ni; r += DEP2_TI) {
                    const double v = s_win[q * DEP2_WIN + r * DEP2_WC + lane];
                    if (v != 0.0) fx_add(hi, hi + NN, (size_t)(oi + r) * N + (oj + lane), v);
                }
            }
        }
    }
    DEP2_CLK(4);
}

// One tile per CTA: blockIdx.x / .y = tile column / row.
template <int TI>
__global__ void __launch_bounds__(TI * 32, 1024 / (TI * 32)) deposit_kernel(DepositArgs a) {
    deposit_tile<TI>(a, blockIdx.x, blockIdx.y);
}

// Depositions of several simulations in one launch: CTA b takes the tile
// b - cta_start[s] of simulation s (cta_start: prefix sums of the tile
// counts, n + 1 entries), whose arguments are args[s].
template <int TI>
__global__ void __launch_bounds__(TI * 32, 1024 / (TI * 32))
    deposit_multi_kernel(const DepositArgs* __restrict__ args, const int* __restrict__ cta_start, int n) {
    __shared__ DepositArgs sa;
    __shared__ int s_sim;
    if (threadIdx.x == 0) {
        int lo = 0, hi = n - 1;   // the last s with cta_start[s] <= blockIdx.x
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (cta_start[mid] <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
        }
        s_sim = lo;
    }
    __syncthreads();
    {
        static_assert(sizeof(DepositArgs) % 4 == 0, "copied as words");
        const int* src = reinterpret_cast<const int*>(args + s_sim);
        int* dst = reinterpret_cast<int*>(&sa);
        for (int w = threadIdx.x; w < (int)(sizeof(DepositArgs) / 4); w += blockDim.x) dst[w] = src[w];
    }
    __syncthreads();
    const int t = (int)blockIdx.x - cta_start[s_sim];
    const int ntx = (sa.Nf + sa.fine_off + 31) / 32;
    deposit_tile<TI>(sa, t % ntx, t / ntx);
}

// Accumulators -> float64 (+ ion background), two cells per thread; the
// accumulators are cleared for the next deposition. All eight 16-byte
// accumulator loads of a thread are issued before any store (the clears
// could alias later loads for the compiler otherwise, serialising them);
// the float64 side uses 16-byte accesses when every array allows it.
__global__ void __launch_bounds__(256) deposit_finalize_kernel(DepositFinalizeArgs f) {
    pdl_wait();
    const int k = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= f.n) return;
    const size_t P = f.plane;
    unsigned long long* acc = f.acc;
    if (k + 1 < f.n) {
        ulonglong2 w[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) w[q] = __ldcg(reinterpret_cast<const ulonglong2*>(acc + q * P + k));
        double2 ri = make_double2(0.0, 0.0);
        if (f.ro_initial) {
            if (f.vec) {
                ri = __ldg(reinterpret_cast<const double2*>(f.ro_initial + k));
            } else {
                ri.x = __ldg(f.ro_initial + k);
                ri.y = __ldg(f.ro_initial + k + 1);
            }
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) __stcg(reinterpret_cast<ulonglong2*>(acc + q * P + k), make_ulonglong2(0ull, 0ull));
        double2 o[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            o[q] = make_double2(fx_value((long long)w[2 * q].x, (long long)w[2 * q + 1].x),
                                fx_value((long long)w[2 * q].y, (long long)w[2 * q + 1].y));
        if (f.ro_initial) {
            o[0].x += ri.x;
            o[0].y += ri.y;
        }
        double* dst[4] = {f.ro, f.jx, f.jy, f.jz};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (f.vec) {
                *reinterpret_cast<double2*>(dst[q] + k) = o[q];
            } else {
                dst[q][k] = o[q].x;
                dst[q][k + 1] = o[q].y;
            }
        }
    } else {
        double out[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            unsigned long long* hp = acc + (2 * q) * P + k;
            unsigned long long* lp = acc + (2 * q + 1) * P + k;
            out[q] = fx_value((long long)*hp, (long long)*lp);
            *hp = 0ull;
            *lp = 0ull;
        }
        double ro = out[0];
        if (f.ro_initial) ro += f.ro_initial[k];
        f.ro[k] = ro;
        f.jx[k] = out[1];
        f.jy[k] = out[2];
        f.jz[k] = out[3];
    }
}

}  // namespace

int launch_move_estimate(const EstimateArgs& a, cudaStream_t s) {
    if (a.n <= 0) return LC3D_OK;
    LC3D_CUDA_TRY(launch_pdl(move_estimate_kernel, dim3((a.n + 255) / 256), dim3(256), 0, s, a));
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int launch_move_smart(const MoveArgs& a, cudaStream_t s) {
    if (a.n <= 0) return LC3D_OK;
    LC3D_CUDA_TRY(launch_pdl(move_smart_kernel, dim3((a.n + LC3D_MOVE_THREADS - 1) / LC3D_MOVE_THREADS),
                             dim3(LC3D_MOVE_THREADS), 0, s, a));
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int particles_prepare() {
    LC3D_CUDA_TRY(cudaFuncSetAttribute(deposit_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dep2_smem(4)));
    LC3D_CUDA_TRY(cudaFuncSetAttribute(deposit_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dep2_smem(8)));
    LC3D_CUDA_TRY(cudaFuncSetAttribute(deposit_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dep2_smem(16)));
    LC3D_CUDA_TRY(cudaFuncSetAttribute(deposit_multi_kernel<DEP_MULTI_ROWS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)dep2_smem(DEP_MULTI_ROWS)));
    return LC3D_OK;
}

// Tile origin of the deposition: with an even fineness the fine lattice
// (lcode.py:468-487) puts two particles per cell and axis, and the pairs of
// fine indices (odd, even) share a cell, so tiles start one particle early.
int deposit_fine_offset(int fineness) {
#ifdef LC3D_DEP2_FORCE_OFF
    (void)fineness;
    return LC3D_DEP2_FORCE_OFF;
#else
    return fineness % 2 == 0 ? 1 : 0;
#endif
}

int launch_deposit_main(const DepositArgs& a, cudaStream_t s) {
    if (a.Nf <= 0) return LC3D_OK;
    const int ti = a.tile_rows ? a.tile_rows : LC3D_DEP2_ROWS;
    const dim3 grid2((a.Nf + a.fine_off + 31) / 32, (a.Nf + a.fine_off + ti - 1) / ti);
    switch (ti) {
        case 4: LC3D_CUDA_TRY(launch_pdl(deposit_kernel<4>, grid2, dim3(4 * 32), dep2_smem(4), s, a)); break;
        case 8: LC3D_CUDA_TRY(launch_pdl(deposit_kernel<8>, grid2, dim3(8 * 32), dep2_smem(8), s, a)); break;
        case 16: LC3D_CUDA_TRY(launch_pdl(deposit_kernel<16>, grid2, dim3(16 * 32), dep2_smem(16), s, a)); break;
        default: return LC3D_ERR_PARAM;
    }
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

#if LC3D_DEP2_CLOCKS
// Instrumented builds only: phase clocks of the last deposit_kernel launch,
// [16384][DEP2_NCLK] cycles since each CTA's start.
extern "C" int lc3d_debug_dep_clocks(long long* host) {
    LC3D_CUDA_TRY(cudaDeviceSynchronize());
    LC3D_CUDA_TRY(cudaMemcpyFromSymbol(host, g_dep2_clocks, sizeof(g_dep2_clocks)));
    return LC3D_OK;
}
#endif

// Tiles of one simulation's deposition at the multi-simulation tile height.
int deposit_multi_tiles(const DepositArgs& a) {
    return ((a.Nf + a.fine_off + 31) / 32) * ((a.Nf + a.fine_off + DEP_MULTI_ROWS - 1) / DEP_MULTI_ROWS);
}

int launch_deposit_multi(const DepositArgs* args_dev, const int* cta_start_dev, int n, int ctas, cudaStream_t s) {
    if (n <= 0 || ctas <= 0) return LC3D_OK;
    deposit_multi_kernel<DEP_MULTI_ROWS><<<ctas, DEP_MULTI_ROWS * 32, dep2_smem(DEP_MULTI_ROWS), s>>>(
        args_dev, cta_start_dev, n);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int launch_deposit_finalize(const DepositFinalizeArgs& f_in, cudaStream_t s) {
    DepositFinalizeArgs f = f_in;
    const uintptr_t al = reinterpret_cast<uintptr_t>(f.ro) | reinterpret_cast<uintptr_t>(f.jx) |
                         reinterpret_cast<uintptr_t>(f.jy) | reinterpret_cast<uintptr_t>(f.jz) |
                         reinterpret_cast<uintptr_t>(f.ro_initial);
    f.vec = (al & 15) == 0;
    LC3D_CUDA_TRY(launch_pdl(deposit_finalize_kernel, dim3(((f.n + 1) / 2 + 255) / 256), dim3(256), 0, s, f));
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

// ---------------------------------------------------------------------------
// Deposition without any device allocation.
//
// Some callers cannot allocate device memory when they deposit: a host
// program that reserved the GPU's memory up front for its own pool and
// forbids further cudaMalloc calls, or code that must not call cudaMalloc
// because it synchronises the device (a latency-critical loop) or is not
// allowed at all (while a CUDA graph is being captured). Creating a
// context (lc3d_create) allocates, so lc3d_deposit_noalloc takes every
// input from the caller and keeps its scratch -- the fixed-point
// accumulators and the error word -- in the file-scope device array below:
// 8 planes of LC3D_NOALLOC_MAX_GRID^2 64-bit words (6.6 MB for 321 x 321),
// which every GPU that loads this library holds until the process exits.
//
// Host code cannot use the array's name as a device address; the address
// is looked up once per device with cudaGetSymbolAddress (with that device
// current) on the first call made on that device, which also sets the
// kernel's shared-memory limit. That first call must therefore come before
// any stream capture. All calls share the array: each call clears the part
// it uses before depositing, and calls that overlap on the GPU (different
// streams, no ordering between them) race on it.
// ---------------------------------------------------------------------------

namespace {

constexpr size_t NOALLOC_PLANE =
    ((size_t)LC3D_NOALLOC_MAX_GRID * LC3D_NOALLOC_MAX_GRID + 31) / 32 * 32;
constexpr size_t NOALLOC_WORDS = DEP_WORDS_PER_CELL * NOALLOC_PLANE + 32;   // + error word (padded)

}  // namespace

static __device__ __align__(256) unsigned long long g_noalloc_scratch[NOALLOC_WORDS];

namespace {

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
unsigned long long* g_noalloc_ptr[NOALLOC_MAX_DEVICES];

// Device address of g_noalloc_scratch on the current device (looked up once).
int noalloc_scratch(unsigned long long** out) {
    int dev = 0;
    LC3D_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return LC3D_ERR_PARAM;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        LC3D_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        LC3D_TRY(particles_prepare());
        g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return LC3D_OK;
}

}  // namespace

extern "C" int lc3d_deposit_noalloc(const lc3d_params* p, const double* ro_initial, const double* x_offt,
                                    const double* y_offt, const double* m, const double* q, const double* px,
                                    const double* py, const double* pz, const double* influence_prev,
                                    const double* influence_next, const int32_t* indices_prev,
                                    const int32_t* indices_next, const double* fine_grid, double* out_ro,
                                    double* out_jx, double* out_jy, double* out_jz, void* stream) {
    int Nc = 0, Nf = 0;
    double rb = 0;
    LC3D_TRY(lc3d_sizes(p, &Nc, &Nf, &rb));
    if (p->grid_steps > LC3D_NOALLOC_MAX_GRID) return LC3D_ERR_SIZE;
    const void* req[] = {x_offt, y_offt, m, q, px, py, pz, influence_prev, influence_next,
                         indices_prev, indices_next, fine_grid, out_ro, out_jx, out_jy, out_jz};
    for (const void* r : req)
        if (!r) return LC3D_ERR_PARAM;
    unsigned long long* scratch = nullptr;
    LC3D_TRY(noalloc_scratch(&scratch));
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int N = p->grid_steps;
    const size_t plane = ((size_t)N * N + 31) / 32 * 32;
    unsigned long long* err_word = scratch + DEP_WORDS_PER_CELL * NOALLOC_PLANE;
    // clear the accumulators this grid uses and the error word
    LC3D_CUDA_TRY(cudaMemsetAsync(scratch, 0, DEP_WORDS_PER_CELL * plane * sizeof(unsigned long long), s));
    LC3D_CUDA_TRY(cudaMemsetAsync(err_word, 0, sizeof(unsigned long long), s));
    const int c = p->plasma_coarseness, f = p->plasma_fineness;
    DepositArgs a{};
    a.x_offt = x_offt; a.y_offt = y_offt; a.m = m; a.q = q; a.px = px; a.py = py; a.pz = pz;
    a.inf_prev = influence_prev; a.inf_next = influence_next; a.fine_grid = fine_grid;
    a.idx_prev = indices_prev; a.idx_next = indices_next;
    a.acc = scratch;
    a.plane = plane;
    a.Nc = Nc; a.Nf = Nf; a.N = N;
    a.fine_off = deposit_fine_offset(p->plasma_fineness);
    a.h = p->grid_step_size;
    a.inv_h = 1.0 / p->grid_step_size;
    a.sf = 1.0 / ((double)(c * f) * (c * f));
    a.err = reinterpret_cast<unsigned*>(err_word);
    DepositFinalizeArgs fa{};
    fa.acc = scratch;
    fa.plane = plane;
    fa.ro_initial = ro_initial;
    fa.ro = out_ro; fa.jx = out_jx; fa.jy = out_jy; fa.jz = out_jz;
    fa.n = N * N;
    LC3D_TRY(launch_deposit_main(a, s));
    return launch_deposit_finalize(fa, s);
}
