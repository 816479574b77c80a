// C ABI of liblc3d: context management, the xi-step schedule and the
// per-stage entry points. Reference: lcode.py:828-931 (step), 936-975
// (init), and the stage functions cited in include/lc3d.h.

#include <cstdlib>
#include <cstring>
#include <new>

#include "lc3d_internal.cuh"

static thread_local char g_last_cuda[512];

void lc3d_set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
    snprintf(g_last_cuda, sizeof(g_last_cuda), "%s (%s) at %s:%d: %s", cudaGetErrorName(e), what, file, line,
             cudaGetErrorString(e));
}

ProfScope::ProfScope(lc3d_ctx* c_, int cat_, cudaStream_t s_) : c(c_), cat(cat_), slot(-1), s(s_) {
    c->launches[cat]++;
    if (c->prof_on && !c->capturing) {
        if (c->prof_used < c->prof_cap) {
            slot = c->prof_used++;
            c->prof_cat[slot] = cat;
            cudaEventRecord(c->prof_ev[2 * slot], s);
        } else {
            c->prof_overflow = 1;
        }
    }
}

ProfScope::~ProfScope() {
    if (slot >= 0) cudaEventRecord(c->prof_ev[2 * slot + 1], s);
}

namespace {

constexpr int PROF_CAP = 8192;

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    bool ok = false;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) return;
        ok = (prev == dev) || (cudaSetDevice(dev) == cudaSuccess);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int check_params(const lc3d_params* p, int* Nc, int* Nf, double* rb) {
    if (!p) return LC3D_ERR_PARAM;
    const int N = p->grid_steps, c = p->plasma_coarseness, f = p->plasma_fineness;
    if (N < 5 || N % 2 != 1) return LC3D_ERR_PARAM;                       // lcode.py:941
    if (!(p->grid_step_size > 0) || !(p->xi_step_size > 0)) return LC3D_ERR_PARAM;
    if (c < 1 || f < 1) return LC3D_ERR_PARAM;
    if (!(p->reflect_padding_steps > c + 1)) return LC3D_ERR_PARAM;       // lcode.py:944
    if (p->precision != LC3D_PREC_FP64 && p->precision != LC3D_PREC_MIXED && p->precision != LC3D_PREC_FFT32 &&
        p->precision != LC3D_PREC_TF32)
        return LC3D_ERR_PARAM;
    if (p->fp64_transform < LC3D_FP64_AUTO || p->fp64_transform > LC3D_FP64_DENSE) return LC3D_ERR_PARAM;
    if (p->mixed_slices < 0 || p->mixed_slices > 6) return LC3D_ERR_PARAM;
    if (p->precision == LC3D_PREC_MIXED && N > 1000) return LC3D_ERR_SIZE;
    const int steps = N - 2 * p->plasma_padding_steps;                   // lcode.py:956
    if (steps < 2) return LC3D_ERR_PARAM;
    const int R = steps / (2 * c);                                        // lcode.py:461
    if (R < 1) return LC3D_ERR_PARAM;
    const int Rf = steps / 2 * f;                                         // lcode.py:480, 483
    if (Rf < 1) return LC3D_ERR_PARAM;
    if (Nc) *Nc = 2 * R - 1;
    if (Nf) *Nf = (f % 2) ? 2 * Rf - 1 : 2 * Rf;
    if (rb) *rb = p->grid_step_size * (N / 2.0 - p->reflect_padding_steps);   // lcode.py:947-949
    return LC3D_OK;
}

template <class T>
int dalloc(T** p, size_t count) {
    LC3D_CUDA_TRY(cudaMalloc(p, count * sizeof(T) + 16));
    LC3D_CUDA_TRY(cudaMemset(*p, 0, count * sizeof(T) + 16));
    return LC3D_OK;
}

int alloc_state(lc3d_state_ptrs& s, size_t np, size_t ng) {
    double** parts[] = {&s.x_offt, &s.y_offt, &s.px, &s.py, &s.pz};
    for (double** q : parts) LC3D_TRY(dalloc(q, np));
    double** grids[] = {&s.Ex, &s.Ey, &s.Ez, &s.Bx, &s.By, &s.Bz, &s.ro, &s.jx, &s.jy, &s.jz};
    for (double** q : grids) LC3D_TRY(dalloc(q, ng));
    return LC3D_OK;
}

void free_state(lc3d_state_ptrs& s) {
    double* all[] = {s.x_offt, s.y_offt, s.px, s.py, s.pz, s.Ex, s.Ey, s.Ez, s.Bx, s.By, s.Bz, s.ro, s.jx, s.jy, s.jz};
    for (double* q : all)
        if (q) cudaFree(q);
    memset(&s, 0, sizeof(s));
}

int copy_state(const lc3d_state_ptrs& dst, const lc3d_state_ptrs& src, size_t np, size_t ng, cudaStream_t s) {
    double* const d[] = {dst.x_offt, dst.y_offt, dst.px, dst.py, dst.pz, dst.Ex, dst.Ey, dst.Ez,
                         dst.Bx, dst.By, dst.Bz, dst.ro, dst.jx, dst.jy, dst.jz};
    const double* const r[] = {src.x_offt, src.y_offt, src.px, src.py, src.pz, src.Ex, src.Ey, src.Ez,
                               src.Bx, src.By, src.Bz, src.ro, src.jx, src.jy, src.jz};
    for (int k = 0; k < 15; ++k) {
        if (!d[k] || !r[k]) return LC3D_ERR_PARAM;
        LC3D_CUDA_TRY(cudaMemcpyAsync(d[k], r[k], (k < 5 ? np : ng) * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s));
    }
    return LC3D_OK;
}

bool state_complete(const lc3d_state_ptrs* s) {
    if (!s) return false;
    const void* all[] = {s->x_offt, s->y_offt, s->px, s->py, s->pz, s->Ex, s->Ey, s->Ez,
                         s->Bx, s->By, s->Bz, s->ro, s->jx, s->jy, s->jz};
    for (const void* q : all)
        if (!q) return false;
    return true;
}

MoveArgs move_base(lc3d_ctx* c) {
    MoveArgs a{};
    memset(&a, 0, sizeof(a));
    a.n = c->Nc * c->Nc;
    a.N = c->N;
    a.h = c->p.grid_step_size;
    a.inv_h = 1.0 / c->p.grid_step_size;
    a.dxi = c->p.xi_step_size;
    a.rb = c->rb;
    a.err = c->err;
    return a;
}

DepositArgs deposit_args(lc3d_ctx* c, const double* x, const double* y, const double* m, const double* q,
                         const double* px, const double* py, const double* pz, const double* packed) {
    DepositArgs a{};
    a.x_offt = x; a.y_offt = y; a.m = m; a.q = q; a.px = px; a.py = py; a.pz = pz;
    a.packed = packed;   // the same values, packed by the move just before
    a.inf_prev = c->inf_prev; a.inf_next = c->inf_next; a.fine_grid = c->fine_grid;
    a.idx_prev = c->idx_prev; a.idx_next = c->idx_next;
    a.acc = c->acc;
    a.plane = c->acc_plane;
    a.Nc = c->Nc; a.Nf = c->Nf; a.N = c->N;
    a.fine_off = deposit_fine_offset(c->p.plasma_fineness);
    a.tile_rows = c->dep_rows;
    a.h = c->p.grid_step_size; a.inv_h = 1.0 / c->p.grid_step_size; a.sf = c->sf;
    a.err = c->err;
    return a;
}

DepositFinalizeArgs finalize_args(lc3d_ctx* c, const double* ro_initial, double* ro, double* jx, double* jy,
                                  double* jz) {
    DepositFinalizeArgs f{};
    f.acc = c->acc;
    f.plane = c->acc_plane;
    f.ro_initial = ro_initial;
    f.ro = ro; f.jx = jx; f.jy = jy; f.jz = jz;
    f.n = c->N * c->N;
    return f;
}

int deposit_into(lc3d_ctx* c, const double* ro_initial, const double* x, const double* y, const double* m,
                 const double* q, const double* px, const double* py, const double* pz, double* ro, double* jx,
                 double* jy, double* jz, cudaStream_t s, const double* packed = nullptr) {
    const DepositArgs a = deposit_args(c, x, y, m, q, px, py, pz, packed);
    const DepositFinalizeArgs f = finalize_args(c, ro_initial, ro, jx, jy, jz);
    {
        ProfScope ps(c, LC3D_STAGE_DEPOSIT, s);
        LC3D_TRY(launch_deposit_main(a, s));
    }
    ProfScope ps(c, LC3D_STAGE_DEPOSIT_FIN, s);
    return launch_deposit_finalize(f, s);
}

// Optional extras of a step: first-pass fields out, or a prediction that
// replaces the first pass, with the residual of the corrector against it.
struct StepExtras {
    double* const* first;                 // 6 fields, or NULL
    const double* const* pred;            // 6 fields, or NULL
    double* residual;                     // device double, or NULL
    const double* beam_host;              // host beam to copy during the first pass, or NULL
};

struct AvgArgs {
    const double* a[6];
    const double* b[6];
    double* out[6];
    int n;
};

// out = (a + b) / 2 for 6 fields
__global__ void pred_avg_kernel(const __grid_constant__ AvgArgs g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.n) return;
#pragma unroll
    for (int f = 0; f < 6; ++f) g.out[f][i] = (g.a[f][i] + g.b[f][i]) / 2;
}

struct ResidArgs {
    const double* f[5];                   // corrector fields Ex Ey Bx By Bz
    const double* pred[5];
    unsigned long long* acc;              // [max |f - pred|, max |f|] as double bits
    int n;
};

// Maxima over the 5 fields; non-negative doubles order like their bits.
__global__ void resid_kernel(const __grid_constant__ ResidArgs a) {
    double d = 0, m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x)
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const double x = a.f[f][i];
            d = fmax(d, fabs(x - a.pred[f][i]));
            m = fmax(m, fabs(x));
        }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(a.acc, (unsigned long long)__double_as_longlong(d));
        atomicMax(a.acc + 1, (unsigned long long)__double_as_longlong(m));
    }
}

__global__ void resid_final_kernel(const unsigned long long* acc, double* out) {
    const double d = __longlong_as_double((long long)acc[0]), m = __longlong_as_double((long long)acc[1]);
    *out = m > 0 ? d / m : d;
}

// The xi step of lcode.py:828-931.
int run_step(lc3d_ctx* c, const lc3d_state_ptrs& prev, const lc3d_state_ptrs& out, const double* beam,
             cudaStream_t s, const StepExtras* x = nullptr) {
    const double* prevF[6] = {prev.Ex, prev.Ey, prev.Ez, prev.Bx, prev.By, prev.Bz};
    const bool A = c->p.field_solver_variant_A != 0;
    const bool predicted = x && x->pred;
    MoveArgs mv = move_base(c);
    mv.m = c->m; mv.q = c->q; mv.x_init = c->x_init; mv.y_init = c->y_init;
    mv.x_prev = prev.x_offt; mv.y_prev = prev.y_offt;
    mv.px_prev = prev.px; mv.py_prev = prev.py; mv.pz_prev = prev.pz;
    mv.out_packed = c->packed;            // each deposition below follows a move

    SolveInputs in{};
    memset(&in, 0, sizeof(in));
    in.ro = c->dens[0]; in.jx = c->dens[1]; in.jy = c->dens[2]; in.jz = c->dens[3];
    in.ro_prev = A ? prev.ro : nullptr;
    in.jz_prev = A ? prev.jz : nullptr;
    in.jx_prev = prev.jx; in.jy_prev = prev.jy;
    in.beam = beam;

    SolveOutputs so{};
    memset(&so, 0, sizeof(so));
    so.mode = 1;
    for (int f = 0; f < 6; ++f) {
        so.prev[f] = prevF[f];
        so.avg[f] = c->avg[f];
    }

    for (int pass = 0; pass < 2; ++pass) {
        // move_smart with the estimate (pass 0: field-free, inline) and the
        // previous (pass 0) or half-step averaged (pass 1) fields
        double* const* pw = c->pw[pass];
        mv.est_x = pass ? c->pw[0][0] : nullptr;
        mv.est_y = pass ? c->pw[0][1] : nullptr;
        for (int f = 0; f < 6; ++f) mv.F[f] = pass ? c->avg[f] : prevF[f];
        mv.out_x = pw[0]; mv.out_y = pw[1]; mv.out_px = pw[2]; mv.out_py = pw[3]; mv.out_pz = pw[4];
        if (pass == 0 && x && x->beam_host) {
            // the host beam crosses on the copy stream while the first push
            // and deposition run (it waits only for the work queued before
            // this step, the previous step's reads of the buffer); the first
            // field solve waits for it
            LC3D_CUDA_TRY(cudaEventRecord(c->ev_main, s));
            LC3D_CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, c->ev_main, 0));
            LC3D_CUDA_TRY(cudaMemcpyAsync(c->beam_dev, x->beam_host, (size_t)c->N * c->N * sizeof(double),
                                          cudaMemcpyHostToDevice, c->copy_stream));
            LC3D_CUDA_TRY(cudaEventRecord(c->ev_copy, c->copy_stream));
            in.beam = c->beam_dev;
        }
        {
            ProfScope ps(c, LC3D_STAGE_MOVE, s);
            LC3D_TRY(launch_move_smart(mv, s));
        }
        if (pass == 0 && predicted) {
            // the prediction stands in for the first-pass fields: only the
            // particle positions of this pass are used (as the estimate)
            AvgArgs g{};
            for (int f = 0; f < 6; ++f) {
                g.a[f] = x->pred[f];
                g.b[f] = prevF[f];
                g.out[f] = c->avg[f];
            }
            g.n = c->N * c->N;
            ProfScope ps(c, LC3D_STAGE_FIELD_FIN, s);
            pred_avg_kernel<<<(g.n + 255) / 256, 256, 0, s>>>(g);
            LC3D_CUDA_TRY(cudaGetLastError());
            continue;
        }
        LC3D_TRY(deposit_into(c, c->ro_initial, pw[0], pw[1], c->m, c->q, pw[2], pw[3], pw[4], c->dens[0],
                              c->dens[1], c->dens[2], c->dens[3], s, c->packed));
        if (pass == 0) {
            in.Ex_sub = prev.Ex; in.Ey_sub = prev.Ey; in.Bx_sub = prev.Bx; in.By_sub = prev.By;
            for (int f = 0; f < 6; ++f) so.out[f] = (x && x->first) ? x->first[f] : nullptr;
        } else {
            in.Ex_sub = c->avg[0]; in.Ey_sub = c->avg[1]; in.Bx_sub = c->avg[3]; in.By_sub = c->avg[4];
            so.out[0] = out.Ex; so.out[1] = out.Ey; so.out[2] = out.Ez;
            so.out[3] = out.Bx; so.out[4] = out.By; so.out[5] = out.Bz;
        }
        if (x && x->beam_host) LC3D_CUDA_TRY(cudaStreamWaitEvent(s, c->ev_copy, 0));
        LC3D_TRY(solve_fields(c, LC3D_F_ALL, in, so, s));
    }
    if (predicted && x->residual) {
        ResidArgs ra{};
        const double* F2[5] = {out.Ex, out.Ey, out.Bx, out.By, out.Bz};
        const int pi[5] = {0, 1, 3, 4, 5};
        for (int f = 0; f < 5; ++f) {
            ra.f[f] = F2[f];
            ra.pred[f] = x->pred[pi[f]];
        }
        ra.acc = c->resid;
        ra.n = c->N * c->N;
        ProfScope ps(c, LC3D_STAGE_OTHER, s);
        LC3D_CUDA_TRY(cudaMemsetAsync(c->resid, 0, 2 * sizeof(unsigned long long), s));
        resid_kernel<<<296, 256, 0, s>>>(ra);
        resid_final_kernel<<<1, 1, 0, s>>>(c->resid, x->residual);
        LC3D_CUDA_TRY(cudaGetLastError());
    }
    // final move with the corrector's averaged fields, then deposit
    mv.est_x = c->pw[1][0];
    mv.est_y = c->pw[1][1];
    for (int f = 0; f < 6; ++f) mv.F[f] = c->avg[f];
    mv.out_x = out.x_offt; mv.out_y = out.y_offt; mv.out_px = out.px; mv.out_py = out.py; mv.out_pz = out.pz;
    {
        ProfScope ps(c, LC3D_STAGE_MOVE, s);
        LC3D_TRY(launch_move_smart(mv, s));
    }
    LC3D_TRY(deposit_into(c, c->ro_initial, out.x_offt, out.y_offt, c->m, c->q, out.px, out.py, out.pz, out.ro,
                          out.jx, out.jy, out.jz, s, c->packed));
    return LC3D_OK;
}

void destroy(lc3d_ctx* c) {
    if (!c) return;
    double* singles[] = {c->m, c->q, c->x_init, c->y_init, c->ro_initial, c->inf_prev, c->inf_next, c->fine_grid};
    for (double* p : singles)
        if (p) cudaFree(p);
    if (c->idx_prev) cudaFree(c->idx_prev);
    if (c->idx_next) cudaFree(c->idx_next);
    free_state(c->st[0]);
    free_state(c->st[1]);
    for (int a = 0; a < 2; ++a)
        for (int k = 0; k < 5; ++k)
            if (c->pw[a][k]) cudaFree(c->pw[a][k]);
    for (int k = 0; k < 4; ++k)
        if (c->dens[k]) cudaFree(c->dens[k]);
    for (int k = 0; k < 6; ++k)
        if (c->avg[k]) cudaFree(c->avg[k]);
    if (c->acc) cudaFree(c->acc);
    if (c->err) cudaFree(c->err);
    if (c->err_host) cudaFreeHost(c->err_host);
    if (c->zeros) cudaFree(c->zeros);
    if (c->resid) cudaFree(c->resid);
    if (c->beam_dev) cudaFree(c->beam_dev);
    if (c->packed) cudaFree(c->packed);
    if (c->ev_main) cudaEventDestroy(c->ev_main);
    if (c->ev_copy) cudaEventDestroy(c->ev_copy);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    for (int q = 0; q < 2; ++q) {
        if (c->ev_join[q]) cudaEventDestroy(c->ev_join[q]);
        if (c->fft_stream[q]) cudaStreamDestroy(c->fft_stream[q]);
    }
    diag_free(c);
    if (c->fft_tw) cudaFree(c->fft_tw);
    mixed_free(c);
    run_free(c);
    if (c->prof_ev) {
        for (int k = 0; k < 2 * c->prof_cap; ++k) cudaEventDestroy(c->prof_ev[k]);
        free(c->prof_ev);
        free(c->prof_cat);
    }
    fields_free(c);
    delete c;
}

inline cudaStream_t S(void* p) { return reinterpret_cast<cudaStream_t>(p); }

// ---------------------------------------------------------------------------
// Plasma layout on the device (lcode.py:454-573, make_coarse_plasma_grid,
// make_fine_plasma_grid, make_plasma): the same float64 expressions as the
// host layout, element by element, so the arrays are bit-identical.
// ---------------------------------------------------------------------------
struct PlasmaArgs {
    double *m, *q, *x_init, *y_init;      // Nc x Nc
    double *inf_prev, *inf_next, *fine;   // Nf
    int32_t *idx_prev, *idx_next;         // Nf
    int Nc, Nf, R, Rf, f;                 // R = Nc half-width + 1, Rf fine half count
    double hc, d, m0, q0;                 // h * coarseness, h / fineness, particle mass and charge
};

// coarse lattice: -(R-1) .. R-1 times h c, the negative half as negated
// products. __dmul_rn: a rounded product that the compiler may not contract
// into an FMA with the subtraction that uses it (numpy rounds it first).
__device__ __forceinline__ double coarse_at(const PlasmaArgs& a, int i) {
    const int j = i - (a.R - 1);
    return j < 0 ? -__dmul_rn((double)(-j), a.hc) : __dmul_rn((double)j, a.hc);
}

__device__ __forceinline__ double fine_at(const PlasmaArgs& a, int i) {
    if (a.f % 2) {
        const int j = i - (a.Rf - 1);
        return j < 0 ? -__dmul_rn((double)(-j), a.d) : __dmul_rn((double)j, a.d);
    }
    return i < a.Rf ? -__dmul_rn(.5 + (double)(a.Rf - 1 - i), a.d) : __dmul_rn(.5 + (double)(i - a.Rf), a.d);
}

__global__ void plasma_coarse_kernel(const __grid_constant__ PlasmaArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.Nc * a.Nc) return;
    const int i = k / a.Nc, j = k - i * a.Nc;
    a.x_init[k] = coarse_at(a, i);
    a.y_init[k] = coarse_at(a, j);
    a.m[k] = a.m0;
    a.q[k] = a.q0;
}

__global__ void plasma_fine_kernel(const __grid_constant__ PlasmaArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.Nf) return;
    const double x = fine_at(a, i);
    // searchsorted(coarse, x), side left: the first index with coarse >= x
    int lo = 0, hi = a.Nc;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (coarse_at(a, mid) < x) lo = mid + 1;
        else hi = mid;
    }
    const int nxt = min(max(lo, 0), a.Nc - 1), prv = min(max(lo - 1, 0), a.Nc - 1);
    double ip = (coarse_at(a, nxt) - x) / a.hc, in = (x - coarse_at(a, prv)) / a.hc;
    if (nxt == 0) { ip = 0; in = 1; }
    if (prv == a.Nc - 1) { in = 0; ip = 1; }
    a.fine[i] = x;
    a.idx_prev[i] = prv;
    a.idx_next[i] = nxt;
    a.inf_prev[i] = ip;
    a.inf_next[i] = in;
}

__global__ void negate_kernel(const double* __restrict__ a, double* __restrict__ out, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = -a[k];
}

}  // namespace

int step_schedule(lc3d_ctx* c, const lc3d_state_ptrs& prev, const lc3d_state_ptrs& out, const double* beam,
                  cudaStream_t s) {
    return run_step(c, prev, out, beam, s);
}

// The plain xi step of run_step cut at its three depositions, for batches
// whose depositions run as one launch over all simulations. Segment `seg`
// enqueues the launches between deposition seg - 1 and deposition seg and
// returns the kernel arguments of deposition seg in *dep (segments 0-2);
// the finalize of deposition seg - 1 opens segment seg (1-3). The launches
// and their order are those of run_step without extras.
int step_schedule_segment(lc3d_ctx* c, const lc3d_state_ptrs& prev, const lc3d_state_ptrs& out,
                          const double* beam, cudaStream_t s, int seg, DepositArgs* dep) {
    const double* prevF[6] = {prev.Ex, prev.Ey, prev.Ez, prev.Bx, prev.By, prev.Bz};
    const bool A = c->p.field_solver_variant_A != 0;
    MoveArgs mv = move_base(c);
    mv.m = c->m; mv.q = c->q; mv.x_init = c->x_init; mv.y_init = c->y_init;
    mv.x_prev = prev.x_offt; mv.y_prev = prev.y_offt;
    mv.px_prev = prev.px; mv.py_prev = prev.py; mv.pz_prev = prev.pz;
    mv.out_packed = c->packed;
    auto move = [&](int pass) -> int {   // pass 0, 1: predictor / corrector; 2: final
        if (pass == 0) {
            mv.est_x = mv.est_y = nullptr;
        } else {
            mv.est_x = c->pw[pass - 1][0];
            mv.est_y = c->pw[pass - 1][1];
        }
        for (int f = 0; f < 6; ++f) mv.F[f] = pass ? c->avg[f] : prevF[f];
        double* const* o = pass < 2 ? c->pw[pass] : nullptr;
        mv.out_x = o ? o[0] : out.x_offt; mv.out_y = o ? o[1] : out.y_offt;
        mv.out_px = o ? o[2] : out.px; mv.out_py = o ? o[3] : out.py; mv.out_pz = o ? o[4] : out.pz;
        ProfScope ps(c, LC3D_STAGE_MOVE, s);
        LC3D_TRY(launch_move_smart(mv, s));
        *dep = deposit_args(c, mv.out_x, mv.out_y, c->m, c->q, mv.out_px, mv.out_py, mv.out_pz, c->packed);
        return LC3D_OK;
    };
    auto finalize = [&](double* ro, double* jx, double* jy, double* jz) -> int {
        ProfScope ps(c, LC3D_STAGE_DEPOSIT_FIN, s);
        return launch_deposit_finalize(finalize_args(c, c->ro_initial, ro, jx, jy, jz), s);
    };
    if (seg == 0) return move(0);
    if (seg == 3) return finalize(out.ro, out.jx, out.jy, out.jz);
    if (seg != 1 && seg != 2) return LC3D_ERR_PARAM;
    const int pass = seg - 1;
    LC3D_TRY(finalize(c->dens[0], c->dens[1], c->dens[2], c->dens[3]));
    SolveInputs in{};
    in.ro = c->dens[0]; in.jx = c->dens[1]; in.jy = c->dens[2]; in.jz = c->dens[3];
    in.ro_prev = A ? prev.ro : nullptr;
    in.jz_prev = A ? prev.jz : nullptr;
    in.jx_prev = prev.jx; in.jy_prev = prev.jy;
    in.beam = beam;
    SolveOutputs so{};
    so.mode = 1;
    for (int f = 0; f < 6; ++f) {
        so.prev[f] = prevF[f];
        so.avg[f] = c->avg[f];
    }
    if (pass == 0) {
        in.Ex_sub = prev.Ex; in.Ey_sub = prev.Ey; in.Bx_sub = prev.Bx; in.By_sub = prev.By;
    } else {
        in.Ex_sub = c->avg[0]; in.Ey_sub = c->avg[1]; in.Bx_sub = c->avg[3]; in.By_sub = c->avg[4];
        so.out[0] = out.Ex; so.out[1] = out.Ey; so.out[2] = out.Ez;
        so.out[3] = out.Bx; so.out[4] = out.By; so.out[5] = out.Bz;
    }
    LC3D_TRY(solve_fields(c, LC3D_F_ALL, in, so, s));
    return move(pass + 1);
}

extern "C" {

const char* lc3d_strerror(int code) {
    switch (code) {
        case LC3D_OK: return "ok";
        case LC3D_ERR_PARAM: return "invalid parameter";
        case LC3D_ERR_CUDA: return g_last_cuda[0] ? g_last_cuda : "CUDA error";
        case LC3D_ERR_WINDOW: return "a plasma particle stencil left the grid (reflect_padding_steps too small or the plasma escaped)";
        case LC3D_ERR_NONFINITE: return "non-finite or out-of-range density/current contribution";
        case LC3D_ERR_STATE: return "const / virt_params or state not set on the context";
        case LC3D_ERR_SIZE: return "size beyond the documented maximum";
        case LC3D_ERR_TIMEOUT: return "a bounded wait inside a kernel ran out (tensor-core pipeline stalled)";
        default: return "unknown error";
    }
}

int lc3d_sizes(const lc3d_params* p, int* Nc, int* Nf, double* reflect_boundary) {
    return check_params(p, Nc, Nf, reflect_boundary);
}

int lc3d_create(const lc3d_params* p, int device, lc3d_ctx** out) {
    if (!out) return LC3D_ERR_PARAM;
    *out = nullptr;
    int Nc, Nf;
    double rb;
    LC3D_TRY(check_params(p, &Nc, &Nf, &rb));
    DeviceGuard g(device);
    if (!g.ok) {
        lc3d_set_last_cuda_error(cudaErrorInvalidDevice, "cudaSetDevice", __FILE__, __LINE__);
        return LC3D_ERR_CUDA;
    }
    lc3d_ctx* c = new (std::nothrow) lc3d_ctx;
    if (!c) return LC3D_ERR_PARAM;
    memset(c, 0, sizeof(*c));
    c->p = *p;
    c->device = device;
    c->N = p->grid_steps;
    c->M = c->N - 2;
    c->Nc = Nc;
    c->Nf = Nf;
    c->rb = rb;
    c->sf = 1.0 / ((double)(p->plasma_coarseness * p->plasma_fineness) * (p->plasma_coarseness * p->plasma_fineness));
    const size_t np = (size_t)Nc * Nc, ng = (size_t)c->N * c->N;
    int rc = LC3D_OK;
#define LC3D_STEP(expr) \
    if (rc == LC3D_OK) rc = (expr)
    LC3D_STEP(dalloc(&c->m, np));
    LC3D_STEP(dalloc(&c->q, np));
    LC3D_STEP(dalloc(&c->x_init, np));
    LC3D_STEP(dalloc(&c->y_init, np));
    LC3D_STEP(dalloc(&c->ro_initial, ng));
    LC3D_STEP(dalloc(&c->inf_prev, (size_t)Nf));
    LC3D_STEP(dalloc(&c->inf_next, (size_t)Nf));
    LC3D_STEP(dalloc(&c->fine_grid, (size_t)Nf));
    LC3D_STEP(dalloc(&c->idx_prev, (size_t)Nf));
    LC3D_STEP(dalloc(&c->idx_next, (size_t)Nf));
    LC3D_STEP(alloc_state(c->st[0], np, ng));
    LC3D_STEP(alloc_state(c->st[1], np, ng));
    for (int a = 0; a < 2; ++a)
        for (int k = 0; k < 5; ++k) LC3D_STEP(dalloc(&c->pw[a][k], np));
    for (int k = 0; k < 4; ++k) LC3D_STEP(dalloc(&c->dens[k], ng));
    for (int k = 0; k < 6; ++k) LC3D_STEP(dalloc(&c->avg[k], ng));
    c->acc_plane = (ng + 31) / 32 * 32;
    LC3D_STEP(dalloc(&c->acc, c->acc_plane * 8));
    LC3D_STEP(dalloc(&c->err, (size_t)1));
    // pinned host word the flag is read into (a direct copy, no staging)
    if (rc == LC3D_OK && cudaHostAlloc(&c->err_host, sizeof(unsigned), cudaHostAllocDefault) != cudaSuccess)
        rc = LC3D_ERR_CUDA;
    LC3D_STEP(dalloc(&c->zeros, ng));
    LC3D_STEP(dalloc(&c->resid, (size_t)2));
    LC3D_STEP(dalloc(&c->beam_dev, ng));
    LC3D_STEP(dalloc(&c->packed, 8 * np));
    if (rc == LC3D_OK && cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess) rc = LC3D_ERR_CUDA;
    if (rc == LC3D_OK && cudaEventCreateWithFlags(&c->ev_main, cudaEventDisableTiming) != cudaSuccess) rc = LC3D_ERR_CUDA;
    if (rc == LC3D_OK && cudaEventCreateWithFlags(&c->ev_copy, cudaEventDisableTiming) != cudaSuccess) rc = LC3D_ERR_CUDA;
    for (int q = 0; q < 2; ++q) {
        if (rc == LC3D_OK && cudaStreamCreateWithFlags(&c->fft_stream[q], cudaStreamNonBlocking) != cudaSuccess)
            rc = LC3D_ERR_CUDA;
        if (rc == LC3D_OK && cudaEventCreateWithFlags(&c->ev_join[q], cudaEventDisableTiming) != cudaSuccess)
            rc = LC3D_ERR_CUDA;
    }
    if (rc == LC3D_OK && cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess) rc = LC3D_ERR_CUDA;
    LC3D_STEP(particles_prepare());
    LC3D_STEP(fields_init(c));
    LC3D_STEP(fft_init(c));
    LC3D_STEP(run_init(c));
    LC3D_STEP(diag_init(c));
    if (rc == LC3D_OK) {
        if (p->fp64_transform == LC3D_FP64_FFT && !c->fft_ok) rc = LC3D_ERR_PARAM;
        if (p->precision == LC3D_PREC_FFT32 && !c->fft_ok) rc = LC3D_ERR_PARAM;   // no dense float32 form
        c->use_fft = c->fft_ok && p->fp64_transform != LC3D_FP64_DENSE;
    }
    if (rc == LC3D_OK && p->precision == LC3D_PREC_MIXED)
        rc = mixed_init(c, p->mixed_slices ? p->mixed_slices : 4, 0);
    if (rc == LC3D_OK && p->precision == LC3D_PREC_TF32)
        rc = mixed_init(c, p->mixed_slices ? p->mixed_slices : 3, 1);
#undef LC3D_STEP
    if (rc == LC3D_OK && cudaDeviceSynchronize() != cudaSuccess) rc = LC3D_ERR_CUDA;
    if (rc != LC3D_OK) {
        destroy(c);
        return rc;
    }
    *out = c;
    return LC3D_OK;
}

int lc3d_destroy(lc3d_ctx* ctx) {
    if (!ctx) return LC3D_OK;
    DeviceGuard g(ctx->device);
    cudaDeviceSynchronize();
    destroy(ctx);
    return LC3D_OK;
}

int lc3d_set_const(lc3d_ctx* c, const lc3d_const_ptrs* k, const lc3d_virt_ptrs* v, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    const cudaStream_t s = S(stream);
    const size_t np = (size_t)c->Nc * c->Nc * sizeof(double), ng = (size_t)c->N * c->N * sizeof(double);
    const size_t nf = (size_t)c->Nf * sizeof(double), ni = (size_t)c->Nf * sizeof(int32_t);
    if (k) {
        if (!k->m || !k->q || !k->x_init || !k->y_init) return LC3D_ERR_PARAM;
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->m, k->m, np, cudaMemcpyDeviceToDevice, s));
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->q, k->q, np, cudaMemcpyDeviceToDevice, s));
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->x_init, k->x_init, np, cudaMemcpyDeviceToDevice, s));
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->y_init, k->y_init, np, cudaMemcpyDeviceToDevice, s));
        if (k->ro_initial)
            LC3D_CUDA_TRY(cudaMemcpyAsync(c->ro_initial, k->ro_initial, ng, cudaMemcpyDeviceToDevice, s));
        else
            LC3D_CUDA_TRY(cudaMemsetAsync(c->ro_initial, 0, ng, s));
        c->const_set |= 1;
    }
    if (v) {
        if (!v->influence_prev || !v->influence_next || !v->indices_prev || !v->indices_next || !v->fine_grid)
            return LC3D_ERR_PARAM;
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->inf_prev, v->influence_prev, nf, cudaMemcpyDeviceToDevice, s));
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->inf_next, v->influence_next, nf, cudaMemcpyDeviceToDevice, s));
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->fine_grid, v->fine_grid, nf, cudaMemcpyDeviceToDevice, s));
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->idx_prev, v->indices_prev, ni, cudaMemcpyDeviceToDevice, s));
        LC3D_CUDA_TRY(cudaMemcpyAsync(c->idx_next, v->indices_next, ni, cudaMemcpyDeviceToDevice, s));
        c->const_set |= 2;
    }
    return LC3D_OK;
}

int lc3d_init_plasma(lc3d_ctx* c, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    const cudaStream_t s = S(stream);
    const int N = c->N, co = c->p.plasma_coarseness, fi = c->p.plasma_fineness;
    const int steps = N - 2 * c->p.plasma_padding_steps;
    PlasmaArgs a{};
    a.m = c->m; a.q = c->q; a.x_init = c->x_init; a.y_init = c->y_init;
    a.inf_prev = c->inf_prev; a.inf_next = c->inf_next; a.fine = c->fine_grid;
    a.idx_prev = c->idx_prev; a.idx_next = c->idx_next;
    a.Nc = c->Nc; a.Nf = c->Nf;
    a.R = steps / (2 * co);
    a.Rf = steps / 2 * fi;
    a.f = fi;
    a.hc = c->p.grid_step_size * co;
    a.d = c->p.grid_step_size / fi;
    a.m0 = (double)(1 * co * co);      // electron mass 1, charge -1 (lcode.py:494-495)
    a.q0 = (double)(-1 * co * co);
    const size_t np = (size_t)c->Nc * c->Nc, ng = (size_t)N * N;
    plasma_coarse_kernel<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(a);
    plasma_fine_kernel<<<(c->Nf + 255) / 256, 256, 0, s>>>(a);
    LC3D_CUDA_TRY(cudaGetLastError());
    c->const_set = 3;
    // state at the start: zero offsets, momenta, fields, densities and currents
    lc3d_state_ptrs& st = c->st[c->cur];
    double* parts[] = {st.x_offt, st.y_offt, st.px, st.py, st.pz};
    double* grids[] = {st.Ex, st.Ey, st.Ez, st.Bx, st.By, st.Bz, st.ro, st.jx, st.jy, st.jz};
    for (double* p : parts) LC3D_CUDA_TRY(cudaMemsetAsync(p, 0, np * sizeof(double), s));
    for (double* p : grids) LC3D_CUDA_TRY(cudaMemsetAsync(p, 0, ng * sizeof(double), s));
    // ion background = minus the initial electron deposition (lcode.py:692-699)
    LC3D_TRY(deposit_into(c, nullptr, st.x_offt, st.y_offt, c->m, c->q, st.px, st.py, st.pz, c->dens[0],
                          c->dens[1], c->dens[2], c->dens[3], s));
    negate_kernel<<<(unsigned)((ng + 255) / 256), 256, 0, s>>>(c->dens[0], c->ro_initial, (int)ng);
    LC3D_CUDA_TRY(cudaGetLastError());
    c->state_set = 1;
    return LC3D_OK;
}

int lc3d_get_const(lc3d_ctx* c, double* m, double* q, double* x_init, double* y_init, double* ro_initial,
                   double* influence_prev, double* influence_next, int32_t* indices_prev, int32_t* indices_next,
                   double* fine_grid, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    if (c->const_set != 3) return LC3D_ERR_STATE;
    DeviceGuard g(c->device);
    const cudaStream_t s = S(stream);
    const size_t np = (size_t)c->Nc * c->Nc * sizeof(double), ng = (size_t)c->N * c->N * sizeof(double);
    const size_t nf = (size_t)c->Nf * sizeof(double), ni = (size_t)c->Nf * sizeof(int32_t);
    struct { void* dst; const void* src; size_t n; } cp[] = {
        {m, c->m, np}, {q, c->q, np}, {x_init, c->x_init, np}, {y_init, c->y_init, np},
        {ro_initial, c->ro_initial, ng}, {influence_prev, c->inf_prev, nf}, {influence_next, c->inf_next, nf},
        {indices_prev, c->idx_prev, ni}, {indices_next, c->idx_next, ni}, {fine_grid, c->fine_grid, nf}};
    for (auto& e : cp)
        if (e.dst) LC3D_CUDA_TRY(cudaMemcpyAsync(e.dst, e.src, e.n, cudaMemcpyDeviceToDevice, s));
    return LC3D_OK;
}

int lc3d_set_state(lc3d_ctx* c, const lc3d_state_ptrs* s, void* stream) {
    if (!c || !state_complete(s)) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    LC3D_TRY(copy_state(c->st[c->cur], *s, (size_t)c->Nc * c->Nc, (size_t)c->N * c->N, S(stream)));
    c->state_set = 1;
    return LC3D_OK;
}

int lc3d_get_state(lc3d_ctx* c, lc3d_state_ptrs* s, void* stream) {
    if (!c || !state_complete(s)) return LC3D_ERR_PARAM;
    if (!c->state_set) return LC3D_ERR_STATE;
    DeviceGuard g(c->device);
    return copy_state(*s, c->st[c->cur], (size_t)c->Nc * c->Nc, (size_t)c->N * c->N, S(stream));
}

int lc3d_step(lc3d_ctx* c, const double* beam_ro, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    if (c->const_set != 3 || !c->state_set) return LC3D_ERR_STATE;
    DeviceGuard g(c->device);
    const int cur = c->cur;
    LC3D_TRY(run_step(c, c->st[cur], c->st[cur ^ 1], beam_ro ? beam_ro : c->zeros, S(stream)));
    c->cur = cur ^ 1;
    return LC3D_OK;
}

int lc3d_step_arrays(lc3d_ctx* c, const lc3d_state_ptrs* prev, const lc3d_state_ptrs* out,
                     const double* beam_ro, void* stream) {
    if (!c || !state_complete(prev) || !state_complete(out)) return LC3D_ERR_PARAM;
    if (c->const_set != 3) return LC3D_ERR_STATE;
    DeviceGuard g(c->device);
    return run_step(c, *prev, *out, beam_ro ? beam_ro : c->zeros, S(stream));
}

int lc3d_step_arrays_host_beam(lc3d_ctx* c, const lc3d_state_ptrs* prev, const lc3d_state_ptrs* out,
                               const double* beam_host, void* stream) {
    if (!c || !state_complete(prev) || !state_complete(out)) return LC3D_ERR_PARAM;
    if (c->const_set != 3) return LC3D_ERR_STATE;
    DeviceGuard g(c->device);
    if (!beam_host) return run_step(c, *prev, *out, c->zeros, S(stream));
    // the previous call's copy has finished reading its host buffer
    LC3D_CUDA_TRY(cudaEventSynchronize(c->ev_copy));
    StepExtras x{nullptr, nullptr, nullptr, beam_host};
    return run_step(c, *prev, *out, c->zeros, S(stream), &x);
}

int lc3d_step_arrays_first_pass(lc3d_ctx* c, const lc3d_state_ptrs* prev, const lc3d_state_ptrs* out,
                                const double* beam_ro, double* const* first, void* stream) {
    if (!c || !state_complete(prev) || !state_complete(out) || !first) return LC3D_ERR_PARAM;
    for (int f = 0; f < 6; ++f)
        if (!first[f]) return LC3D_ERR_PARAM;
    if (c->const_set != 3) return LC3D_ERR_STATE;
    DeviceGuard g(c->device);
    StepExtras x{first, nullptr, nullptr, nullptr};
    return run_step(c, *prev, *out, beam_ro ? beam_ro : c->zeros, S(stream), &x);
}

int lc3d_step_arrays_predicted(lc3d_ctx* c, const lc3d_state_ptrs* prev, const lc3d_state_ptrs* out,
                               const double* beam_ro, const double* const* pred, double* residual, void* stream) {
    if (!c || !state_complete(prev) || !state_complete(out) || !pred) return LC3D_ERR_PARAM;
    for (int f = 0; f < 6; ++f)
        if (!pred[f]) return LC3D_ERR_PARAM;
    if (c->const_set != 3) return LC3D_ERR_STATE;
    DeviceGuard g(c->device);
    StepExtras x{nullptr, pred, residual, nullptr};
    return run_step(c, *prev, *out, beam_ro ? beam_ro : c->zeros, S(stream), &x);
}

int lc3d_fields_rel_diff(lc3d_ctx* c, const double* const* a, const double* const* b, double* out, void* stream) {
    if (!c || !a || !b || !out) return LC3D_ERR_PARAM;
    ResidArgs ra{};
    const int pi[5] = {0, 1, 3, 4, 5};   // Ex, Ey, Bx, By, Bz
    for (int f = 0; f < 5; ++f) {
        if (!a[pi[f]] || !b[pi[f]]) return LC3D_ERR_PARAM;
        ra.pred[f] = a[pi[f]];
        ra.f[f] = b[pi[f]];
    }
    ra.acc = c->resid;
    ra.n = c->N * c->N;
    DeviceGuard g(c->device);
    const cudaStream_t s = S(stream);
    LC3D_CUDA_TRY(cudaMemsetAsync(c->resid, 0, 2 * sizeof(unsigned long long), s));
    resid_kernel<<<296, 256, 0, s>>>(ra);
    resid_final_kernel<<<1, 1, 0, s>>>(c->resid, out);
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

int lc3d_move_estimate_wo_fields(lc3d_ctx* c, const double* m, const double* x_init, const double* y_init,
                                 const double* prev_x_offt, const double* prev_y_offt, const double* px,
                                 const double* py, const double* pz, double* out_x_offt, double* out_y_offt,
                                 void* stream) {
    if (!c || !m || !x_init || !y_init || !prev_x_offt || !prev_y_offt || !px || !py || !pz || !out_x_offt ||
        !out_y_offt)
        return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    EstimateArgs a{};
    a.m = m; a.x_init = x_init; a.y_init = y_init; a.x_prev = prev_x_offt; a.y_prev = prev_y_offt;
    a.px = px; a.py = py; a.pz = pz; a.out_x = out_x_offt; a.out_y = out_y_offt;
    a.n = c->Nc * c->Nc;
    a.dxi = c->p.xi_step_size;
    a.rb = c->rb;
    ProfScope ps(c, LC3D_STAGE_MOVE, S(stream));
    return launch_move_estimate(a, S(stream));
}

int lc3d_move_smart(lc3d_ctx* c, const double* m, const double* q, const double* x_init, const double* y_init,
                    const double* x_prev_offt, const double* y_prev_offt, const double* estimated_x_offt,
                    const double* estimated_y_offt, const double* px_prev, const double* py_prev,
                    const double* pz_prev, const double* Ex_avg, const double* Ey_avg, const double* Ez_avg,
                    const double* Bx_avg, const double* By_avg, const double* Bz_avg, double* new_x_offt,
                    double* new_y_offt, double* new_px, double* new_py, double* new_pz, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    const void* req[] = {m, q, x_init, y_init, x_prev_offt, y_prev_offt, estimated_x_offt, estimated_y_offt,
                         px_prev, py_prev, pz_prev, Ex_avg, Ey_avg, Ez_avg, Bx_avg, By_avg, Bz_avg,
                         new_x_offt, new_y_offt, new_px, new_py, new_pz};
    for (const void* r : req)
        if (!r) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    MoveArgs a = move_base(c);
    a.m = m; a.q = q; a.x_init = x_init; a.y_init = y_init;
    a.x_prev = x_prev_offt; a.y_prev = y_prev_offt;
    a.est_x = estimated_x_offt; a.est_y = estimated_y_offt;
    a.px_prev = px_prev; a.py_prev = py_prev; a.pz_prev = pz_prev;
    a.F[0] = Ex_avg; a.F[1] = Ey_avg; a.F[2] = Ez_avg; a.F[3] = Bx_avg; a.F[4] = By_avg; a.F[5] = Bz_avg;
    a.out_x = new_x_offt; a.out_y = new_y_offt; a.out_px = new_px; a.out_py = new_py; a.out_pz = new_pz;
    ProfScope ps(c, LC3D_STAGE_MOVE, S(stream));
    return launch_move_smart(a, S(stream));
}

int lc3d_deposit(lc3d_ctx* c, const double* ro_initial, const double* x_offt, const double* y_offt,
                 const double* m, const double* q, const double* px, const double* py, const double* pz,
                 double* out_ro, double* out_jx, double* out_jy, double* out_jz, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    if (!(c->const_set & 2)) return LC3D_ERR_STATE;
    const void* req[] = {x_offt, y_offt, m, q, px, py, pz, out_ro, out_jx, out_jy, out_jz};
    for (const void* r : req)
        if (!r) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    return deposit_into(c, ro_initial, x_offt, y_offt, m, q, px, py, pz, out_ro, out_jx, out_jy, out_jz,
                        S(stream));
}

int lc3d_calculate_Ex_Ey_Bx_By(lc3d_ctx* c, const double* Ex_avg, const double* Ey_avg, const double* Bx_avg,
                               const double* By_avg, const double* beam_ro, const double* ro, const double* jx,
                               const double* jy, const double* jz, const double* jx_prev, const double* jy_prev,
                               double* Ex, double* Ey, double* Bx, double* By, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    const void* req[] = {Ex_avg, Ey_avg, Bx_avg, By_avg, ro, jx, jy, jz, jx_prev, jy_prev, Ex, Ey, Bx, By};
    for (const void* r : req)
        if (!r) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    SolveInputs in{};
    memset(&in, 0, sizeof(in));
    in.ro = ro; in.jz = jz; in.jx = jx; in.jy = jy; in.jx_prev = jx_prev; in.jy_prev = jy_prev;
    in.beam = beam_ro ? beam_ro : c->zeros;
    in.Ex_sub = Ex_avg; in.Ey_sub = Ey_avg; in.Bx_sub = Bx_avg; in.By_sub = By_avg;
    SolveOutputs o{};
    memset(&o, 0, sizeof(o));
    o.out[0] = Ex; o.out[1] = Ey; o.out[3] = Bx; o.out[4] = By;
    return solve_fields(c, LC3D_F_EXEYBXBY, in, o, S(stream));
}

int lc3d_calculate_Ez(lc3d_ctx* c, const double* jx, const double* jy, double* Ez, void* stream) {
    if (!c || !jx || !jy || !Ez) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    SolveInputs in{};
    memset(&in, 0, sizeof(in));
    in.jx = jx; in.jy = jy;
    SolveOutputs o{};
    memset(&o, 0, sizeof(o));
    o.out[2] = Ez;
    return solve_fields(c, LC3D_F_EZ, in, o, S(stream));
}

int lc3d_calculate_Bz(lc3d_ctx* c, const double* jx, const double* jy, double* Bz, void* stream) {
    if (!c || !jx || !jy || !Bz) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    SolveInputs in{};
    memset(&in, 0, sizeof(in));
    in.jx = jx; in.jy = jy;
    SolveOutputs o{};
    memset(&o, 0, sizeof(o));
    o.out[5] = Bz;
    return solve_fields(c, LC3D_F_BZ, in, o, S(stream));
}

int lc3d_profile(lc3d_ctx* c, int enable) {
    if (!c) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    if (enable && !c->prof_ev) {
        c->prof_ev = (cudaEvent_t*)calloc(2 * PROF_CAP, sizeof(cudaEvent_t));
        c->prof_cat = (int*)calloc(PROF_CAP, sizeof(int));
        if (!c->prof_ev || !c->prof_cat) return LC3D_ERR_PARAM;
        for (int k = 0; k < 2 * PROF_CAP; ++k) LC3D_CUDA_TRY(cudaEventCreate(&c->prof_ev[k]));
        c->prof_cap = PROF_CAP;
    }
    c->prof_on = enable ? 1 : 0;
    c->prof_used = 0;
    c->prof_overflow = 0;
    for (int k = 0; k < LC3D_NSTAGES; ++k) {
        c->launches[k] = 0;
        c->prof_ms[k] = 0;
        c->prof_count[k] = 0;
    }
    return LC3D_OK;
}

int lc3d_profile_read(lc3d_ctx* c, long long* launches, double* ms, long long* timed) {
    if (!c) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    LC3D_CUDA_TRY(cudaDeviceSynchronize());
    for (int k = 0; k < c->prof_used; ++k) {
        float t = 0;
        LC3D_CUDA_TRY(cudaEventElapsedTime(&t, c->prof_ev[2 * k], c->prof_ev[2 * k + 1]));
        c->prof_ms[c->prof_cat[k]] += t;
        c->prof_count[c->prof_cat[k]]++;
    }
    for (int k = 0; k < LC3D_NSTAGES; ++k) {
        if (launches) launches[k] = c->launches[k];
        if (ms) ms[k] = c->prof_ms[k];
        if (timed) timed[k] = c->prof_count[k];
        c->launches[k] = 0;
        c->prof_ms[k] = 0;
        c->prof_count[k] = 0;
    }
    c->prof_used = 0;
    return c->prof_overflow ? LC3D_ERR_SIZE : LC3D_OK;
}

int lc3d_test_wait_limit(lc3d_ctx* c, long long cycles, int skip_loads) {
    if (!c) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    LC3D_CUDA_TRY(cudaDeviceSynchronize());   // no replay of a graph holding the old bound is in flight
    c->wait_limit = cycles > 0 ? cycles : 0;
    c->skip_loads = skip_loads ? 1 : 0;
    run_drop_graphs(c);                       // the bound is a kernel parameter inside them
    return LC3D_OK;
}

int lc3d_set_tiles(lc3d_ctx* c, int deposit_rows, int fft_ctas_per_sm) {
    if (!c) return LC3D_ERR_PARAM;
    if (!(deposit_rows == 0 || deposit_rows == 4 || deposit_rows == 8 || deposit_rows == 16)) return LC3D_ERR_PARAM;
    if (fft_ctas_per_sm < 0 || fft_ctas_per_sm > 64) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    LC3D_CUDA_TRY(cudaDeviceSynchronize());   // no replay of the old graphs is in flight
    c->dep_rows = deposit_rows;
    c->fft_per_sm = fft_ctas_per_sm;
    run_drop_graphs(c);                       // the shapes are launch parameters inside them
    return LC3D_OK;
}

int lc3d_check_error(lc3d_ctx* c, void* stream) {
    if (!c) return LC3D_ERR_PARAM;
    DeviceGuard g(c->device);
    LC3D_CUDA_TRY(cudaMemcpyAsync(c->err_host, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost, S(stream)));
    LC3D_CUDA_TRY(cudaStreamSynchronize(S(stream)));
    const unsigned flag = *c->err_host;
    if (flag) LC3D_CUDA_TRY(cudaMemsetAsync(c->err, 0, sizeof(unsigned), S(stream)));
    if (flag & LC3D_FLAG_WINDOW) return LC3D_ERR_WINDOW;
    if (flag & LC3D_FLAG_NONFINITE) return LC3D_ERR_NONFINITE;
    if (flag & LC3D_FLAG_TIMEOUT) return LC3D_ERR_TIMEOUT;
    return LC3D_OK;
}

}  // extern "C"
