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
// final conversion rounds once. Each CTA owns a 16x16 patch of the fine
// lattice and accumulates into a shared-memory window placed on the bounding
// box of its particles' cells; particles whose stencil falls outside the
// window (strongly displaced plasma) add straight to the global accumulators.
// The window is then flushed with 64-bit integer reductions into global
// memory, and a finalize pass converts to float64, adds the ion background
// and clears the accumulators for the next call.

#include "lc3d_internal.cuh"

namespace {

// ---------------------------------------------------------------------------
// TSC weights, lcode.py:396-418. Order MP 0P PP M0 00 P0 MM 0M PM.
// ---------------------------------------------------------------------------
struct Tsc {
    int i, j;
    double wxM, wx0, wxP, wyM, wy0, wyP;
};

__device__ __forceinline__ Tsc tsc_weights(double x, double y, int N, double h) {
    Tsc t;
    double x_h = x / h + .5, y_h = y / h + .5;
    double fx = floor(x_h), fy = floor(y_h);
    // out-of-range positions map to an invalid index without UB in the cast
    fx = fmin(fmax(fx, -1.0e6), 1.0e6);
    fy = fmin(fmax(fy, -1.0e6), 1.0e6);
    t.i = (int)fx + N / 2;
    t.j = (int)fy + N / 2;
    double xl = x_h - fx - .5, yl = y_h - fy - .5;
    t.wx0 = .75 - xl * xl;
    t.wy0 = .75 - yl * yl;
    t.wxP = (.5 + xl) * (.5 + xl) / 2;
    t.wyP = (.5 + yl) * (.5 + yl) / 2;
    t.wxM = (.5 - xl) * (.5 - xl) / 2;
    t.wyM = (.5 - yl) * (.5 - yl) / 2;
    return t;
}

__device__ __forceinline__ bool tsc_in_grid(const Tsc& t, int N) {
    return t.i >= 1 && t.i <= N - 2 && t.j >= 1 && t.j <= N - 2;
}

// interp9, lcode.py:421-430 (same summation order).
__device__ __forceinline__ double interp9(const double* __restrict__ a, const Tsc& t, int N) {
    const double* r0 = a + (size_t)(t.i - 1) * N + t.j;   // row i-1
    const double* r1 = r0 + N;
    const double* r2 = r1 + N;
    return r0[+1] * (t.wxM * t.wyP) + r1[+1] * (t.wx0 * t.wyP) + r2[+1] * (t.wxP * t.wyP) +
           r0[0] * (t.wxM * t.wy0) + r1[0] * (t.wx0 * t.wy0) + r2[0] * (t.wxP * t.wy0) +
           r0[-1] * (t.wxM * t.wyM) + r1[-1] * (t.wx0 * t.wyM) + r2[-1] * (t.wxP * t.wyM);
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
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    double ex, ey;
    estimate_one(a.m[k], a.x_init[k], a.y_init[k], a.x_prev[k], a.y_prev[k], a.px[k], a.py[k],
                 a.pz[k], a.dxi, a.rb, ex, ey);
    a.out_x[k] = ex;
    a.out_y[k] = ey;
}

// ---------------------------------------------------------------------------
// Pusher, lcode.py:704-793. One thread per coarse particle. With est_x ==
// NULL the field-free estimate of lcode.py:369-391 is computed inline (the
// predictor pass of step()).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) move_smart_kernel(MoveArgs a) {
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
    Tsc t = tsc_weights(x_half, y_half, a.N, a.h);
    if (!tsc_in_grid(t, a.N)) {
        // the reference would read out of bounds here; flag and keep prev
        atomicOr(a.err, LC3D_FLAG_WINDOW);
        a.out_x[k] = x_offt;
        a.out_y[k] = y_offt;
        a.out_px[k] = opx;
        a.out_py[k] = opy;
        a.out_pz[k] = opz;
        return;
    }
    const double Ex = interp9(a.F[0], t, a.N), Ey = interp9(a.F[1], t, a.N);
    const double Ez = interp9(a.F[2], t, a.N), Bx = interp9(a.F[3], t, a.N);
    const double By = interp9(a.F[4], t, a.N), Bz = interp9(a.F[5], t, a.N);

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

constexpr int DEP_T = 16;      // fine particles per CTA side
constexpr int DEP_W = 24;      // shared window side (cells)
constexpr int DEP_WORDS = 8;   // 4 fields x (hi, lo)

// One fine particle: coarse->fine mix (lcode.py:591-621) and the deposit
// quantities (lcode.py:651-655).
struct FineParticle {
    double x, y, dro, djx, djy, djz;
};

__device__ __forceinline__ FineParticle fine_particle(const DepositArgs& a, int fi, int fj) {
    const double ipi = a.inf_prev[fi], ini = a.inf_next[fi];
    const double ipj = a.inf_prev[fj], inj = a.inf_next[fj];
    const double A = ipi * ipj, B = ipi * inj, C = ini * ipj, D = ini * inj;
    const int pi = a.idx_prev[fi], ni = a.idx_next[fi];
    const int pj = a.idx_prev[fj], nj = a.idx_next[fj];
    const int kA = pi * a.Nc + pj, kB = pi * a.Nc + nj, kC = ni * a.Nc + pj, kD = ni * a.Nc + nj;
#define LC3D_MIX(arr) (A * __ldg(arr + kA) + B * __ldg(arr + kB) + C * __ldg(arr + kC) + D * __ldg(arr + kD))
    FineParticle p;
    p.x = a.fine_grid[fi] + LC3D_MIX(a.x_offt);
    p.y = a.fine_grid[fj] + LC3D_MIX(a.y_offt);
    const double m = a.sf * LC3D_MIX(a.m);
    const double q = a.sf * LC3D_MIX(a.q);
    const double px = a.sf * LC3D_MIX(a.px);
    const double py = a.sf * LC3D_MIX(a.py);
    const double pz = a.sf * LC3D_MIX(a.pz);
#undef LC3D_MIX
    const double gamma_m = sqrt(m * m + px * px + py * py + pz * pz);
    p.dro = q / (1 - pz / gamma_m);
    p.djx = px * (p.dro / gamma_m);
    p.djy = py * (p.dro / gamma_m);
    p.djz = pz * (p.dro / gamma_m);
    return p;
}

__global__ void __launch_bounds__(256) deposit_kernel(DepositArgs a) {
    __shared__ unsigned long long win[DEP_W * DEP_W * DEP_WORDS];
    __shared__ int s_imin, s_imax, s_jmin, s_jmax;

    const int tid = threadIdx.y * DEP_T + threadIdx.x;
    const int fi = blockIdx.y * DEP_T + threadIdx.y;
    const int fj = blockIdx.x * DEP_T + threadIdx.x;
    const bool in_lattice = fi < a.Nf && fj < a.Nf;
    const int N = a.N;

    if (tid == 0) {
        s_imin = s_jmin = 1 << 30;
        s_imax = s_jmax = -(1 << 30);
    }
    for (int w = tid; w < DEP_W * DEP_W * DEP_WORDS; w += 256) win[w] = 0ull;

    FineParticle p;
    Tsc t;
    bool valid = false;
    if (in_lattice) {
        p = fine_particle(a, fi, fj);
        t = tsc_weights(p.x, p.y, N, a.h);
        valid = tsc_in_grid(t, N);
        if (!valid) atomicOr(a.err, LC3D_FLAG_WINDOW);
        const double vmax = fmax(fmax(fabs(p.dro), fabs(p.djx)), fmax(fabs(p.djy), fabs(p.djz)));
        if (valid && !(vmax < FX_MAX)) {   // also catches NaN
            atomicOr(a.err, LC3D_FLAG_NONFINITE);
            valid = false;
        }
    }
    __syncthreads();
    if (valid) {
        atomicMin(&s_imin, t.i);
        atomicMax(&s_imax, t.i);
        atomicMin(&s_jmin, t.j);
        atomicMax(&s_jmax, t.j);
    }
    __syncthreads();
    const int oi = s_imin - 1, oj = s_jmin - 1;   // window origin (cells)
    if (valid) {
        const double wx[3] = {t.wxM, t.wx0, t.wxP};
        const double wy[3] = {t.wyM, t.wy0, t.wyP};
        const double val[4] = {p.dro, p.djx, p.djy, p.djz};
        const int li = t.i - oi, lj = t.j - oj;   // stencil centre in the window
        const bool inside = li + 1 < DEP_W && lj + 1 < DEP_W;
#pragma unroll
        for (int di = 0; di < 3; ++di) {
#pragma unroll
            for (int dj = 0; dj < 3; ++dj) {
                const double w = wx[di] * wy[dj];
#pragma unroll
                for (int f = 0; f < 4; ++f) {
                    long long hi, lo;
                    fx_split(val[f] * w, hi, lo);
                    if (inside) {
                        unsigned long long* c =
                            &win[((li + di - 1) * DEP_W + (lj + dj - 1)) * DEP_WORDS + 2 * f];
                        atomicAdd(c, (unsigned long long)hi);
                        atomicAdd(c + 1, (unsigned long long)lo);
                    } else {
                        unsigned long long* c =
                            a.acc + ((size_t)(t.i + di - 1) * N + (t.j + dj - 1)) * DEP_WORDS + 2 * f;
                        atomicAdd(c, (unsigned long long)hi);
                        atomicAdd(c + 1, (unsigned long long)lo);
                    }
                }
            }
        }
    }
    __syncthreads();
    // flush the touched part of the window
    const int ni = min(s_imax + 2 - oi, DEP_W), nj = min(s_jmax + 2 - oj, DEP_W);
    if (s_imin <= s_imax) {
        const int rowlen = nj * DEP_WORDS;
        for (int w = tid; w < ni * rowlen; w += 256) {
            const int r = w / rowlen, c = w - r * rowlen;
            const unsigned long long v = win[r * DEP_W * DEP_WORDS + c];
            if (v) atomicAdd(a.acc + ((size_t)(oi + r) * N + oj) * DEP_WORDS + c, v);
        }
    }
}

__global__ void __launch_bounds__(256) deposit_finalize_kernel(DepositFinalizeArgs f) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= f.n) return;
    ulonglong2* w = reinterpret_cast<ulonglong2*>(f.acc + (size_t)k * DEP_WORDS);
    ulonglong2 a0 = w[0], a1 = w[1], a2 = w[2], a3 = w[3];
    const ulonglong2 z = make_ulonglong2(0ull, 0ull);
    w[0] = z; w[1] = z; w[2] = z; w[3] = z;
    double ro = fx_value((long long)a0.x, (long long)a0.y);
    if (f.ro_initial) ro += f.ro_initial[k];
    f.ro[k] = ro;
    f.jx[k] = fx_value((long long)a1.x, (long long)a1.y);
    f.jy[k] = fx_value((long long)a2.x, (long long)a2.y);
    f.jz[k] = fx_value((long long)a3.x, (long long)a3.y);
}

}  // namespace

int launch_move_estimate(const EstimateArgs& a, cudaStream_t s) {
    if (a.n <= 0) return LC3D_OK;
    move_estimate_kernel<<<(a.n + 255) / 256, 256, 0, s>>>(a);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int launch_move_smart(const MoveArgs& a, cudaStream_t s) {
    if (a.n <= 0) return LC3D_OK;
    move_smart_kernel<<<(a.n + 255) / 256, 256, 0, s>>>(a);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int launch_deposit_main(const DepositArgs& a, cudaStream_t s) {
    if (a.Nf <= 0) return LC3D_OK;
    dim3 grid((a.Nf + DEP_T - 1) / DEP_T, (a.Nf + DEP_T - 1) / DEP_T);
    deposit_kernel<<<grid, dim3(DEP_T, DEP_T), 0, s>>>(a);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int launch_deposit_finalize(const DepositFinalizeArgs& f, cudaStream_t s) {
    deposit_finalize_kernel<<<(f.n + 255) / 256, 256, 0, s>>>(f);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}
