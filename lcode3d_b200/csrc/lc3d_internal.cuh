// Internal declarations shared by the liblc3d translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/lc3d.h"

// Device error flag bits (the host maps them to LC3D_ERR_*).
#define LC3D_FLAG_WINDOW 1u
#define LC3D_FLAG_NONFINITE 2u
#define LC3D_FLAG_TIMEOUT 4u

#define LC3D_CUDA_TRY(expr)                                                  \
    do {                                                                     \
        cudaError_t _e = (expr);                                             \
        if (_e != cudaSuccess) {                                             \
            lc3d_set_last_cuda_error(_e, #expr, __FILE__, __LINE__);         \
            return LC3D_ERR_CUDA;                                            \
        }                                                                    \
    } while (0)

#define LC3D_TRY(expr)                                                       \
    do {                                                                     \
        int _rc = (expr);                                                    \
        if (_rc != LC3D_OK) return _rc;                                      \
    } while (0)

void lc3d_set_last_cuda_error(cudaError_t e, const char* what, const char* file, int line);

// ---------------------------------------------------------------------------
// Programmatic dependent launch of the xi-step kernels. They are launched
// with programmatic stream serialization: the launch of a kernel is
// processed while its predecessor in the stream is still running, and its
// CTAs start as soon as the predecessor has exited. Every such kernel calls
// pdl_wait() before its first global-memory access, read or write (reads
// of tables written once at set-up, which no kernel of the chain writes,
// may come before it): the wait returns once the preceding grid has
// completed and its writes are visible, so stream order holds for all data,
// and transitively, since every kernel in the chain waits. No kernel triggers its successor early
// (griddepcontrol.launch_dependents): resident, waiting successor CTAs
// measured slower, also when an FFT pass signalled only from each CTA's
// last row group (1770 -> 1756 xi-steps/s in float64, 2083 -> 1966 with
// float32 transforms). pdl_wait() is a no-op for a kernel launched without the
// attribute. Step loops launched from the host gain 4-7 % from this; CUDA
// graph replays are unchanged.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}

// ---------------------------------------------------------------------------
// Particle kernels (particles.cu)
// ---------------------------------------------------------------------------

struct MoveArgs {
    const double *m, *q, *x_init, *y_init;
    const double *x_prev, *y_prev;        // prev offsets
    const double *est_x, *est_y;          // estimated offsets (NULL: estimate inline)
    const double *px_prev, *py_prev, *pz_prev;
    const double *F[6];                   // Ex Ey Ez Bx By Bz (averaged)
    double *out_x, *out_y, *out_px, *out_py, *out_pz;
    double* out_packed;                   // optional: [n][8] = x_offt y_offt m q px py pz, pad
    int n;                                // coarse particles
    int N;                                // grid_steps
    double h, inv_h, dxi, rb;
    unsigned* err;
};

struct EstimateArgs {
    const double *m, *x_init, *y_init, *x_prev, *y_prev, *px, *py, *pz;
    double *out_x, *out_y;
    int n;
    double dxi, rb;
};

struct DepositArgs {
    const double *x_offt, *y_offt, *m, *q, *px, *py, *pz;   // coarse, Nc x Nc
    const double *inf_prev, *inf_next, *fine_grid;            // Nf
    const int32_t *idx_prev, *idx_next;                       // Nf
    const double* packed;                                     // optional: the 7 coarse arrays as [Nc*Nc][8]
    unsigned long long* acc;                                  // 8 planes of fixed-point words
    size_t plane;                                             // plane stride (>= N*N, 256-byte multiple)
    int Nc, Nf, N;
    int fine_off;                                             // tile origin: fine_off particles before 0
    int tile_rows;                                            // fine rows per CTA (4, 8, 16; 0: default)
    double h, inv_h, sf;
    unsigned* err;
};

struct DepositFinalizeArgs {
    unsigned long long* acc;
    size_t plane;
    const double* ro_initial;             // may be NULL
    double *ro, *jx, *jy, *jz;
    int n;                                // N*N
    int vec;                              // set by the launcher: 16-byte aligned float64 arrays
};

int launch_move_estimate(const EstimateArgs& a, cudaStream_t s);
int launch_move_smart(const MoveArgs& a, cudaStream_t s);
int launch_deposit_main(const DepositArgs& a, cudaStream_t s);
int deposit_fine_offset(int fineness);
// Default fine rows per deposition CTA (4, 8 or 16; 4 measured fastest at
// 641^2).
#ifndef LC3D_DEP2_ROWS
#define LC3D_DEP2_ROWS 4
#endif
// Depositions of several simulations in one launch (batches): tiles of
// DEP_MULTI_ROWS fine rows, CTA b of the launch takes tile b - cta_start[s]
// of simulation s. The same height as the default: the window's float64 sums
// follow the tile, so only the same tiles give results bit-identical to each
// simulation run alone.
constexpr int DEP_MULTI_ROWS = LC3D_DEP2_ROWS;
int deposit_multi_tiles(const DepositArgs& a);
int launch_deposit_multi(const DepositArgs* args_dev, const int* cta_start_dev, int n, int ctas, cudaStream_t s);
int launch_deposit_finalize(const DepositFinalizeArgs& f, cudaStream_t s);

// ---------------------------------------------------------------------------
// Launch accounting and optional per-launch CUDA-event timing (lc3d_api.cu).
// Categories are the LC3D_STAGE_* values of include/lc3d.h.
// ---------------------------------------------------------------------------
struct lc3d_ctx;
struct ProfScope {
    lc3d_ctx* c;
    int cat, slot;
    cudaStream_t s;
    ProfScope(lc3d_ctx* c, int cat, cudaStream_t s);
    ~ProfScope();
};

// ---------------------------------------------------------------------------
// Field solvers (fields.cu)
// ---------------------------------------------------------------------------

// Which fields a solve computes.
#define LC3D_F_EXEYBXBY 1
#define LC3D_F_EZ 2
#define LC3D_F_BZ 4
#define LC3D_F_ALL 7

struct SolveInputs {
    const double *ro, *ro_prev;           // ro_prev != NULL: ro_in = (ro + ro_prev) / 2
    const double *jz, *jz_prev;           // likewise for jz
    const double *jx, *jy, *jx_prev, *jy_prev, *beam;
    const double *Ex_sub, *Ey_sub, *Bx_sub, *By_sub;   // subtraction-trick terms
};

// mode 0: raw fields into out[] (zero border, Bz mean removed), as the
//         reference's calculate_* functions return them;
// mode 1: step finalisation: Variant A (if set) against prev[], Bz mean
//         removed, fields into out[] (optional, may be NULL) and the
//         half-step averages (F + prev) / 2 into avg[].
struct SolveOutputs {
    int mode;
    double* out[6];                       // Ex Ey Ez Bx By Bz
    const double* prev[6];
    double* avg[6];
};

int solve_fields(lc3d_ctx* ctx, int which, const SolveInputs& in,
                 const SolveOutputs& o, cudaStream_t s);

// FFT row transforms (fields_fft.cu): rows of `in` (length N for DCT-I,
// N - 2 for DST-I) are transformed and written transposed, out[k][r],
// optionally multiplied element-wise by lam[k][r] as they are written.
// Element types of a pass: the rows read, the arithmetic (and Lambda), the
// rows written.
enum FftTypes {
    FFT_F64 = 0,       // double -> double arithmetic -> double
    FFT_F64_F32 = 1,   // double -> float -> float
    FFT_F32 = 2,       // float -> float -> float
    FFT_F32_F64 = 3,   // float -> float -> double
};
struct FftRowsDesc {
    const void* in;
    int ld_in, rows, type;                // type: 0 DCT-I, 1 DST-I
    void* out;
    int ld_out;
    const void* lam;                      // in the arithmetic's type
    int ld_lam;
    double* partial;                      // optional: per-CTA sums of the written values
};
int fft_init(lc3d_ctx* ctx);
// Row pitch (elements) of the FFT passes' intermediate planes: float64 rows
// padded to whole 32-byte sectors (N rounded up to a multiple of 4), so a
// CTA's transposed 4-row stores fill whole sectors (transforms 0.319 ->
// 0.317 ms per step at 641^2); float32 intermediates at N (padding them
// measured slower: 0.235 -> 0.242).
inline int fft_pitch(int N, bool f32 = false) { return f32 ? N : (N + 3) / 4 * 4; }
int fft_cta_rows();                       // rows per CTA: partial sums per field = ceil(rows / this)
int fft_rows(lc3d_ctx* ctx, const FftRowsDesc* desc, int count, int types, cudaStream_t s);
int fft_plan(int P, int* rad);

// Mixed-precision transform stages (fields_mixed.cu): C = A B^T with one
// operand a sliced fixed transform matrix (0 = S2, 1 = C) and the other the
// float64 data operand `data` (data_rows x K, row-major, ld_data), sliced
// into the field's bf16 buffer before the GEMM.
struct MixedStageDesc {
    int field, fixed, data_is_a;
    const double* data;
    int ld_data, data_rows;
    int M, N, K;
    double* out;
    int ldo, transposed;                  // out[m][n] or out[n][m]
    const double* lam;                    // optional Lambda[m][n]
    int ldl;
};
int mixed_init(lc3d_ctx* ctx, int slices, int tf32);   // split-bf16 or split-tf32 transforms
void mixed_free(lc3d_ctx* ctx);
int mixed_stage(lc3d_ctx* ctx, const MixedStageDesc* d, int count, cudaStream_t s);
// one-time per-device kernel attributes (shared-memory opt-ins)
int particles_prepare();
int fft_prepare(int P);
int fields_init(lc3d_ctx* ctx);           // transform matrices, workspaces
int diag_init(lc3d_ctx* ctx);             // diagnostics.cu
void diag_free(lc3d_ctx* ctx);
void fields_free(lc3d_ctx* ctx);

// ---------------------------------------------------------------------------
// Context
// ---------------------------------------------------------------------------

struct lc3d_ctx {
    lc3d_params p;
    int device;
    int N, M, Nc, Nf;                     // M = N - 2
    double rb, sf;                        // reflect_boundary, 1/(c f)^2
    // owned constants
    double *m, *q, *x_init, *y_init, *ro_initial;
    double *inf_prev, *inf_next, *fine_grid;
    int32_t *idx_prev, *idx_next;
    int const_set;
    // owned state, double-buffered
    lc3d_state_ptrs st[2];
    int cur, state_set;
    // step workspaces
    double* pw[2][5];                     // predictor / corrector particles
    double* dens[4];                      // ro jx jy jz of predictor / corrector
    double* avg[6];                       // half-step averaged fields
    unsigned long long* acc;              // deposit fixed-point accumulators, 8 planes
    size_t acc_plane;                     // plane stride in words
    unsigned* err;                        // device error flag
    unsigned* err_host;                   // pinned host word lc3d_check_error reads it into
    double* zeros;                        // N x N zeros (absent beam)
    unsigned long long* resid;            // predicted-step residual maxima (2 words, double bits)
    double* diag_w;                       // zn diagnostic: Gaussian weights, then partial sums
    double* diag_buf;                     // zn diagnostic: two N x N blur planes
    int diag_r;                           // Gaussian radius
    double* beam_dev;                     // device copy of a host beam (lc3d_step_arrays_host_beam)
    double* packed;                       // coarse particles of the last move, [Nc*Nc][8] (x y m q px py pz -)
    cudaStream_t copy_stream;             // its host-to-device copies
    cudaEvent_t ev_main, ev_copy;         // ordering of those copies with the step's stream
    cudaStream_t fft_stream[2];           // further streams of the FFT passes (groups of fields)
    cudaEvent_t ev_fork, ev_join[2];      // their fork from and joins to the solve's stream
    // field-solver workspaces (fields.cu)
    double *S2, *C, *CT;                  // 2*DST-I (M x M), DCT-I (N x N), its transpose
    double *lam_dir, *lam_mix, *lam_mixT, *lam_neu;
    float *lam32_dir, *lam32_mix, *lam32_mixT, *lam32_neu;   // float32-transform precision only
    double* rhs[6];                       // right-hand sides, N x N planes
    double* t1[6];                        // transform scratch
    double* t2[6];
    double* raw[6];                       // raw solver output, zero border
    double* red;                          // Bz mean partial sums
    int red_blocks;
    int fft_ok, use_fft;                  // FFT transforms available / selected
    double* fft_tw;                       // FFT twiddles, P complex
    int fft_grid[4];                      // persistent FFT grid per FftTypes instantiation
    int fft_sms;                          // SMs of the device (the grid cap of lc3d_set_tiles)
    void* mixed;                          // mixed-precision solver state (fields_mixed.cu)
    // launch accounting / profiling
    long long launches[LC3D_NSTAGES];
    int prof_on, prof_used, prof_cap, prof_overflow;
    cudaEvent_t* prof_ev;                 // 2 per recorded launch
    int* prof_cat;
    double prof_ms[LC3D_NSTAGES];
    long long prof_count[LC3D_NSTAGES];
    // device-side beam and graph-replayed runs (run.cu)
    int capturing;                        // a step is being captured into a graph
    int one_stream;                       // solves on the caller's stream alone: a batch graph's
                                          // branches already overlap the simulations
    double* beam_buf;                     // N x N beam evaluated on the device
    void* run_ctl;                        // device RunCtl: xi counter, history
    double beam_A, beam_sr, beam_lf;      // amplitude, sigma_r, length factor
    cudaGraphExec_t graph[2];             // one xi step from state parity 0 / 1
    long long graph_launches[2][LC3D_NSTAGES];
    // bounded tensor-core pipeline waits (lc3d_test_wait_limit): limit in SM
    // clock cycles (0: the default) and the timeout test's load skipping
    long long wait_limit;
    int skip_loads;
    // tile shapes (lc3d_set_tiles): deposition fine rows per CTA (0: default)
    // and resident FFT CTAs per SM (0: as many as fit)
    int dep_rows;
    int fft_per_sm;
};

// The xi-step schedule (lc3d_api.cu), and the run machinery (run.cu).
int step_schedule(lc3d_ctx* c, const lc3d_state_ptrs& prev, const lc3d_state_ptrs& out, const double* beam,
                  cudaStream_t s);
int step_schedule_segment(lc3d_ctx* c, const lc3d_state_ptrs& prev, const lc3d_state_ptrs& out,
                          const double* beam, cudaStream_t s, int seg, DepositArgs* dep);
int run_init(lc3d_ctx* c);
void run_drop_graphs(lc3d_ctx* c);       // graphs of lc3d_run (re-captured on the next run)
void run_free(lc3d_ctx* c);
