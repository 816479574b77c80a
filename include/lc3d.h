/*
 * lc3d.h -- C ABI of the B200-native LCODE 3D xi-step solver (liblc3d.so).
 *
 * The reference (lotov/lcode3d) is one Python module, lcode.py; its public
 * boundary is the module contract that its CLI loop (lcode.py:1032-1051) and
 * embedding code use:
 *     init(config)                                   lcode.py:936-975
 *     step(config, const, virt_params, prev, beam_ro) lcode.py:828-931
 * plus the per-stage functions that step() calls. Each entry point below
 * replaces one of those functions (cited beside it); the Python package
 * lcode3d_b200 binds them with ctypes and keeps the reference's names,
 * argument meaning and attribute names on top.
 *
 * Conventions
 *  - All array pointers are DEVICE pointers to float64 (int32 where noted),
 *    C-contiguous, row-major with x as axis 0 (lcode.py:197, 951-953):
 *    grids are N x N (N = grid_steps), coarse particle arrays Nc x Nc,
 *    fine-lattice arrays have length Nf.
 *  - Every call is stream-ordered on `stream` (a cudaStream_t; NULL = the
 *    legacy default stream) and performs no implicit host synchronisation,
 *    except lc3d_check_error / lc3d_ez_history which read device memory.
 *  - A context owns all its device workspaces and its own copies of the
 *    constant arrays (const, virt_params). One context per host thread.
 *  - Return value: LC3D_OK (0) or one of the error codes below; the text of
 *    a code is lc3d_strerror(code). A particle whose 3x3 stencil would leave
 *    the grid is never written out of bounds: it is skipped, and the device
 *    error flag is raised (read it with lc3d_check_error), where the
 *    reference would corrupt memory (docs/overview/window_and_grids.rst:60).
 */
#ifndef LC3D_H
#define LC3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LC3D_OK 0
#define LC3D_ERR_PARAM 1        /* invalid parameter / config (the reference asserts) */
#define LC3D_ERR_CUDA 2         /* a CUDA runtime call failed */
#define LC3D_ERR_WINDOW 3       /* device flag: a particle stencil left the grid */
#define LC3D_ERR_NONFINITE 4    /* device flag: non-finite or out-of-range deposit */
#define LC3D_ERR_STATE 5        /* call order: state / const not set */
#define LC3D_ERR_SIZE 6         /* size beyond a documented maximum */
#define LC3D_ERR_TIMEOUT 7      /* device flag: a bounded wait in a kernel ran out */

/* Precision of the field solvers. */
#define LC3D_PREC_FP64 0        /* float64 solvers (transform form: fp64_transform) */
#define LC3D_PREC_MIXED 1       /* split-BF16 tcgen05 transforms, fp32 accumulate,
                                   float64 combination; grid_steps <= 1000 */
#define LC3D_PREC_TF32 3        /* split-TF32 tcgen05 transforms (kind::tf32, 10-bit
                                   digits, fp32 accumulate, float64 combination);
                                   mixed_slices digits per operand (default 3) */
#define LC3D_PREC_FFT32 2       /* float32 FFT transforms (float32 intermediates and
                                   eigenvalues); right-hand sides, field outputs,
                                   averaging and particles stay float64; needs
                                   2(N-1) to factor into 2, 3 and 5 */

/* Float64 transform method (lc3d_params.fp64_transform). */
#define LC3D_FP64_AUTO 0        /* FFT when 2(N-1) factors into 2, 3, 5; else dense */
#define LC3D_FP64_FFT 1         /* shared-memory FFT DST-I / DCT-I */
#define LC3D_FP64_DENSE 2       /* dense transform matrices (DGEMM form) */

/* Mirrors the reference config module attributes (config_example.py:1-30). */
typedef struct lc3d_params {
    int grid_steps;                       /* odd (lcode.py:941) */
    double grid_step_size;
    double xi_step_size;
    int plasma_coarseness;
    int plasma_fineness;
    int reflect_padding_steps;            /* > plasma_coarseness + 1 (lcode.py:944) */
    int plasma_padding_steps;
    double field_solver_subtraction_trick; /* multiplies the *_avg terms (lcode.py:264-268) */
    int field_solver_variant_A;
    int precision;                        /* LC3D_PREC_* */
    int fp64_transform;                   /* LC3D_FP64_* */
    int mixed_slices;                     /* bf16 slices per operand, 1..6 (0: 4) */
} lc3d_params;

/* The xi-step state, attribute names of lcode.py:926-929. */
typedef struct lc3d_state_ptrs {
    double *x_offt, *y_offt, *px, *py, *pz;   /* Nc x Nc */
    double *Ex, *Ey, *Ez, *Bx, *By, *Bz;      /* N x N */
    double *ro, *jx, *jy, *jz;                /* N x N */
} lc3d_state_ptrs;

/* const of lcode.py:964-965. */
typedef struct lc3d_const_ptrs {
    const double *m, *q, *x_init, *y_init;    /* Nc x Nc */
    const double *ro_initial;                 /* N x N */
} lc3d_const_ptrs;

/* virt_params of lcode.py:566-570 (indices as int32). */
typedef struct lc3d_virt_ptrs {
    const double *influence_prev, *influence_next;   /* Nf */
    const int32_t *indices_prev, *indices_next;      /* Nf */
    const double *fine_grid;                         /* Nf */
} lc3d_virt_ptrs;

typedef struct lc3d_ctx lc3d_ctx;

/* Derived sizes of a configuration without creating a context:
 * Nc = coarse particles per side, Nf = fine particles per side,
 * reflect_boundary as init() computes it (lcode.py:947-949, 454-487). */
int lc3d_sizes(const lc3d_params* p, int* Nc, int* Nf, double* reflect_boundary);

/* Create a context on `device` (replaces the per-config state that the
 * reference keeps in cp.memoize caches, lcode.py:144, 215, 316). */
int lc3d_create(const lc3d_params* p, int device, lc3d_ctx** out);
int lc3d_destroy(lc3d_ctx* ctx);
const char* lc3d_strerror(int code);

/* Copy const and virt_params into the context (device to device). */
int lc3d_set_const(lc3d_ctx* ctx, const lc3d_const_ptrs* c,
                   const lc3d_virt_ptrs* v, void* stream);

/* init() on the device (lcode.py:936-975 with make_plasma, lcode.py:490-573,
 * and initial_deposition, lcode.py:692-699): builds the context's const and
 * virt_params and its state at xi = 0 (zero offsets, momenta and fields)
 * from the parameters alone, bit-identical to the host layout of init().
 * lc3d_get_const copies the context's const and virt_params out (device
 * arrays, any may be NULL); the state comes out with lc3d_get_state. */
int lc3d_init_plasma(lc3d_ctx* ctx, void* stream);
int lc3d_get_const(lc3d_ctx* ctx, double* m, double* q, double* x_init, double* y_init,
                   double* ro_initial, double* influence_prev, double* influence_next,
                   int32_t* indices_prev, int32_t* indices_next, double* fine_grid,
                   void* stream);

/* Context-owned state (double-buffered): copy in / copy out. */
int lc3d_set_state(lc3d_ctx* ctx, const lc3d_state_ptrs* s, void* stream);
int lc3d_get_state(lc3d_ctx* ctx, lc3d_state_ptrs* s, void* stream);

/* One xi step on the context-owned state (lcode.py:828-931); beam_ro is an
 * N x N device array. Graph-capturable. */
int lc3d_step(lc3d_ctx* ctx, const double* beam_ro, void* stream);

/* One xi step from caller-owned prev into caller-owned out arrays
 * (lcode.py:828-931, the reference's ownership: prev is kept, out is new).
 * `out` must not alias `prev`. */
int lc3d_step_arrays(lc3d_ctx* ctx, const lc3d_state_ptrs* prev,
                     const lc3d_state_ptrs* out, const double* beam_ro,
                     void* stream);

/* lc3d_step_arrays with the beam in HOST memory (N x N float64; NULL: no
 * beam), as the reference's loop produces it (lcode.py:1040, 839). The copy
 * to the device runs on a stream of the context while the step's first
 * push and deposition run, and the first field solve waits for it. At
 * entry the call waits (on the host) for the previous call's copy to have
 * read its buffer; the caller must keep beam_host unchanged until the next
 * call on this context returns or the stream is synchronised. For a pinned
 * buffer the copy is asynchronous; for pageable memory the CUDA runtime
 * stages it during the call. */
int lc3d_step_arrays_host_beam(lc3d_ctx* ctx, const lc3d_state_ptrs* prev,
                               const lc3d_state_ptrs* out, const double* beam_host,
                               void* stream);

/* ---- device-side beam and graph-replayed runs ----
 * The reference evaluates config.beam on the host and copies it to the
 * device every step (lcode.py:1040, 839), and copies the whole Ez array back
 * to read Ez(0,0) (lcode.py:1043-1046). For the axisymmetric driver of the
 * benchmark configurations,
 *   rho_b = A exp(-(x^2 + y^2) / (2 sigma_r^2)) * 0.5 (1 - cos(sqrt(pi/2) xi / L))
 * for 0 <= xi <= 2 sqrt(2 pi) L, else 0 (xi = xi_i * xi_step_size, L the
 * length factor), a run needs no host work: lc3d_set_beam stores the
 * parameters (NULL: no beam), lc3d_run advances the context-owned state by
 * nsteps steps starting at xi index xi0, each step a replay of a CUDA graph
 * captured on first use (beam kernel, the step, Ez(N/2, N/2) appended to
 * ez_history[k], a device array of nsteps doubles, or NULL). Not while
 * lc3d_profile timing is enabled. */
typedef struct lc3d_beam_params {
    double amplitude, sigma_r, length_factor;
} lc3d_beam_params;

int lc3d_set_beam(lc3d_ctx* ctx, const lc3d_beam_params* beam);
/* the beam set by lc3d_set_beam at xi index xi_i into beam_ro (N x N, device) */
int lc3d_beam_eval(lc3d_ctx* ctx, int xi_i, double* beam_ro, void* stream);
int lc3d_run(lc3d_ctx* ctx, int xi0, int nsteps, double* ez_history, void* stream);

/* Batches of independent simulations (a parameter scan; no reference
 * counterpart -- the reference runs one simulation per process). Each
 * simulation is a context of its own (grid size, precision, beam and state
 * may differ; all on one device, const and state set). lc3d_batch_run
 * advances every simulation by nsteps steps; each step is ONE launch of a
 * CUDA graph that holds every simulation's whole step (device beam, solver,
 * Ez(0,0) record) on its own parallel branch. xi0[i] is simulation i's first
 * xi index, ez_history[i] a device array of nsteps doubles (the array or
 * its entries may be NULL). The graphs are recaptured when a context was
 * stepped on its own or its beam changed in between. */
typedef struct lc3d_batch lc3d_batch;
int lc3d_batch_create(lc3d_ctx* const* ctxs, int count, lc3d_batch** out);
int lc3d_batch_run(lc3d_batch* b, const int* xi0, int nsteps, double* const* ez_history, void* stream);
int lc3d_batch_destroy(lc3d_batch* b);

/* How a batch's graphs are built (no reference counterpart). 0 (default):
 * every simulation's whole step on its own branch. 1: each simulation's
 * step is cut at its three depositions, and every deposition point is ONE
 * launch over all simulations (a work list of (simulation, tile) items,
 * tiles of 8 fine rows) between the branches. Results are bit-identical to
 * the simulations run alone with 8-row deposition tiles. The next
 * lc3d_batch_run captures the graphs again. */
int lc3d_batch_set_mode(lc3d_batch* b, int multi_deposit);

/* ---- per-stage entry points (the functions step() calls) ---- */

/* move_estimate_wo_fields, lcode.py:369-391. */
int lc3d_move_estimate_wo_fields(lc3d_ctx* ctx, const double* m,
        const double* x_init, const double* y_init,
        const double* prev_x_offt, const double* prev_y_offt,
        const double* px, const double* py, const double* pz,
        double* out_x_offt, double* out_y_offt, void* stream);

/* move_smart / move_smart_kernel, lcode.py:704-823. */
int lc3d_move_smart(lc3d_ctx* ctx, const double* m, const double* q,
        const double* x_init, const double* y_init,
        const double* x_prev_offt, const double* y_prev_offt,
        const double* estimated_x_offt, const double* estimated_y_offt,
        const double* px_prev, const double* py_prev, const double* pz_prev,
        const double* Ex_avg, const double* Ey_avg, const double* Ez_avg,
        const double* Bx_avg, const double* By_avg, const double* Bz_avg,
        double* new_x_offt, double* new_y_offt,
        double* new_px, double* new_py, double* new_pz, void* stream);

/* deposit / deposit_kernel, lcode.py:626-689 (virt_params from the context;
 * ro_initial may be NULL for the initial deposition, lcode.py:692-699).
 * Deterministic: bit-identical results for identical inputs. */
int lc3d_deposit(lc3d_ctx* ctx, const double* ro_initial,
        const double* x_offt, const double* y_offt,
        const double* m, const double* q,
        const double* px, const double* py, const double* pz,
        double* out_ro, double* out_jx, double* out_jy, double* out_jz,
        void* stream);

/* calculate_Ex_Ey_Bx_By, lcode.py:246-290. */
int lc3d_calculate_Ex_Ey_Bx_By(lc3d_ctx* ctx,
        const double* Ex_avg, const double* Ey_avg,
        const double* Bx_avg, const double* By_avg,
        const double* beam_ro, const double* ro, const double* jx,
        const double* jy, const double* jz,
        const double* jx_prev, const double* jy_prev,
        double* Ex, double* Ey, double* Bx, double* By, void* stream);

/* calculate_Ez, lcode.py:160-184. */
int lc3d_calculate_Ez(lc3d_ctx* ctx, const double* jx, const double* jy,
                      double* Ez, void* stream);

/* calculate_Bz, lcode.py:333-364. */
int lc3d_calculate_Bz(lc3d_ctx* ctx, const double* jx, const double* jy,
                      double* Bz, void* stream);

/* ---- diagnostics ---- */

/* The density-noise figure of diags_ro_zn (lcode.py:979-987) for one N x N
 * array ro: mean |ro - G(ro)| / 4.23045376e-04 with G the Gaussian blur of
 * scipy.ndimage.gaussian_filter (sigma = 0.25 / grid_step_size, truncated at
 * 4 sigma, 'reflect' edges), written to *zn (a device double). The running
 * maximum over calls that the reference keeps is the caller's (a host
 * variable in lcode3d_b200.lcode.diags_ro_zn). Deterministic. */
int lc3d_diag_zn(lc3d_ctx* ctx, const double* ro, double* zn, void* stream);

/* ---- launch accounting and kernel timing ---- */

/* Stage categories of the launch counters and timers. */
#define LC3D_STAGE_MOVE 0          /* move_smart_kernel / estimate */
#define LC3D_STAGE_DEPOSIT 1       /* deposit_kernel (fine particles -> accumulators) */
#define LC3D_STAGE_DEPOSIT_FIN 2   /* accumulators -> ro, jx, jy, jz */
#define LC3D_STAGE_RHS 3           /* field-solver right-hand sides */
#define LC3D_STAGE_TRANSFORM 4     /* DST/DCT transform GEMMs */
#define LC3D_STAGE_FIELD_FIN 5     /* Variant A, Bz mean, half-step averages */
#define LC3D_STAGE_SLICE 6          /* float64 -> bf16 operand slicing (mixed precision) */
#define LC3D_STAGE_OTHER 7
#define LC3D_NSTAGES 8

/* Enable (1) or disable (0) CUDA-event timing of every kernel launch of
 * this context, and reset the counters. Not for use under stream capture.
 * No reference counterpart (the reference has no instrumentation). */
int lc3d_profile(lc3d_ctx* ctx, int enable);

/* Synchronise the device and report, per stage, the kernel launches issued
 * since the last reset (launches[]) and, with timing enabled, the summed
 * kernel time in ms (ms[]) and the number of timed launches (timed[]).
 * Arrays hold LC3D_NSTAGES entries; any may be NULL. Resets the counters. */
int lc3d_profile_read(lc3d_ctx* ctx, long long* launches, double* ms, long long* timed);

/* Read and clear the device error flag (synchronises `stream`); returns
 * LC3D_OK, LC3D_ERR_WINDOW, LC3D_ERR_NONFINITE or LC3D_ERR_TIMEOUT. */
int lc3d_check_error(lc3d_ctx* ctx, void* stream);

/* Tile shapes of this context (no reference counterpart; the autotuner of
 * lcode3d_b200.batch picks them per grid size). deposit_rows: fine-lattice
 * rows per CTA of the deposition, 4, 8 or 16 (0: the default, 8); the CTA
 * covers that many rows x 32 columns, and 8, 4 or 2 CTAs share an SM.
 * fft_ctas_per_sm: resident CTAs per SM of the persistent FFT row passes
 * (0: as many as fit). Results agree to rounding (the deposition's window
 * sums are grouped by tile). Graphs of lc3d_run are re-captured with the
 * new shapes; batches keep the shapes their contexts had when the batch
 * was made. Returns LC3D_ERR_PARAM for other values. */
int lc3d_set_tiles(lc3d_ctx* ctx, int deposit_rows, int fft_ctas_per_sm);

/* Test hook of the failure detection; no reference counterpart (the
 * reference has no bounded waits). Every wait in the tensor-core pipeline of
 * the mixed-precision transforms is bounded: once `cycles` SM clock cycles
 * have passed (cycles <= 0: the default, 2e9, one to two seconds) the kernel
 * stops waiting, frees its tensor memory, raises the timeout flag
 * (LC3D_ERR_TIMEOUT from lc3d_check_error) and returns, and the context
 * stays usable. With skip_loads != 0 the pipeline's producer issues no
 * loads, so the consumer's first wait runs out with no copy in flight; the
 * fields such a call writes are undefined. Only tests of that path set it. */
int lc3d_test_wait_limit(lc3d_ctx* ctx, long long cycles, int skip_loads);

/* ---- deposition that allocates nothing ----
 *
 * No counterpart in the reference. For callers that cannot allocate device
 * memory at the point where they deposit: a host program that reserved the
 * GPU's memory for its own pool up front and forbids further cudaMalloc,
 * or code that must not call cudaMalloc because it synchronises the device
 * or because a CUDA graph is being captured. It computes what lc3d_deposit
 * computes (same kernels, bit-identical results) without a context: every
 * input comes from the caller (virt_params as in lc3d_virt_ptrs, indices as
 * int32), and the scratch -- fixed-point accumulators and an error word --
 * lives in a file-scope device array sized for grids up to
 * LC3D_NOALLOC_MAX_GRID x LC3D_NOALLOC_MAX_GRID (6.6 MB, held by every GPU
 * that loads the library until the process exits). Larger grids return
 * LC3D_ERR_SIZE. ro_initial may be NULL.
 *
 * The first call on a device looks up the array's device address and sets
 * the kernel's shared-memory limit; make that first call before any stream
 * capture. Each call clears the scratch it uses first; calls that overlap
 * on the GPU (no ordering between their streams) race on the shared array.
 * Particles whose stencil leaves the grid, and particles with non-finite or
 * out-of-range deposit values, are skipped as in lc3d_deposit, but this
 * entry point does not report them. */
#define LC3D_NOALLOC_MAX_GRID 321
int lc3d_deposit_noalloc(const lc3d_params* p, const double* ro_initial,
        const double* x_offt, const double* y_offt,
        const double* m, const double* q,
        const double* px, const double* py, const double* pz,
        const double* influence_prev, const double* influence_next,
        const int32_t* indices_prev, const int32_t* indices_next,
        const double* fine_grid,
        double* out_ro, double* out_jx, double* out_jy, double* out_jz,
        void* stream);

/* ---- learned predictor stage ----
 *
 * No counterpart in the reference. The reference's step (lcode.py:828-931)
 * makes three particle passes: a predictor pass that moves the particles
 * with the PREVIOUS step's fields ("no halfstep-averaged fields yet",
 * lcode.py:846-871) and solves for first-pass fields F1, a corrector pass
 * with (F1 + prev) / 2 that solves for the step's fields F2 (lcode.py:
 * 876-901), and a final pass with (F2 + prev) / 2 (lcode.py:906-918).
 *
 * lc3d_step_arrays_first_pass is lc3d_step_arrays that also writes F1
 * (Ex, Ey, Ez, Bx, By, Bz after the Variant A extrapolation) to first[6]
 * (device arrays, N x N): the training targets of a predictor.
 *
 * lc3d_step_arrays_predicted runs the step with F1 replaced by pred[6]
 * (Ex, Ey, Ez, Bx, By, Bz; device arrays): the predictor pass only moves
 * the particles (its deposit and field solve are skipped), the corrector
 * and final passes are the reference's; with pred = F1 it reproduces
 * lc3d_step_arrays bit for bit. residual (a device double, or NULL)
 * receives max_f max|F2_f - pred_f| / max_f max|F2_f| over Ex, Ey, Bx, By,
 * Bz, the corrector's change of the prediction (a diagnostic: the plain
 * method's own F2 - F1 is of the same order).
 *
 * lc3d_fields_rel_diff writes max_f max|a_f - b_f| / max_f max|b_f| over
 * Ex, Ey, Bx, By, Bz of two sets of 6 fields to *out (a device double): a
 * caller that checks a prediction against a step's true F1 (recorded by
 * lc3d_step_arrays_first_pass) decides with it whether to keep predicting
 * (see lcode3d_b200.predictor.run_learned). */
int lc3d_step_arrays_first_pass(lc3d_ctx* ctx, const lc3d_state_ptrs* prev,
        const lc3d_state_ptrs* out, const double* beam_ro,
        double* const* first, void* stream);
int lc3d_step_arrays_predicted(lc3d_ctx* ctx, const lc3d_state_ptrs* prev,
        const lc3d_state_ptrs* out, const double* beam_ro,
        const double* const* pred, double* residual, void* stream);
int lc3d_fields_rel_diff(lc3d_ctx* ctx, const double* const* a, const double* const* b,
        double* out, void* stream);

/* A learned field predictor (no counterpart in the reference): a 3-level
 * convolutional U-Net (3x3 convolutions, 32 / 64 / 128 channels, bf16
 * weights and activations, fp32 accumulation; inference on the tcgen05
 * tensor cores) mapping the fields ro, jx, jy, jz, Ex, Ey, Bx, By, Bz of
 * steps t-1 and t-2 (pack: arrays of 9 in that order) to the first-pass
 * fields Ex, Ey, Bx, By, Bz of step t:
 *     pred_f = 2 F_f(t-1) - F_f(t-2) + o_f * net_f(F(t-1) / s, (F(t-1) - F(t-2)) / d, log10(s) / 4)
 * The scales are per sample: s_c and d_c are the root mean squares of field
 * c and of its difference over the grid, o is the root mean square of the
 * differences of Ex, Ey, Bx, By, Bz (each times a multiplier set by
 * lc3d_predictor_set_scales, default 1), computed on the device by
 * lc3d_predictor_pack, which also feeds log10(s_c) / 4 as 9 constant input
 * channels (27 of the 32 input channels are used). Parameters are one float32
 * array of lc3d_predictor_num_params() entries (per layer: weights
 * [9][Cout][Cin], then biases [Cout]). Arrays are device arrays; the
 * float64 fields are N x N as elsewhere. */
typedef struct lc3d_predictor lc3d_predictor;
#define LC3D_PRED_INPUT 0       /* bf16 [N][N + 1][32] network input */
#define LC3D_PRED_OUTPUT 1      /* f32 [N][N + 1][16] network output */
#define LC3D_PRED_TARGET 2      /* f32 [N][N + 1][16] training target */
long long lc3d_predictor_num_params(void);
int lc3d_predictor_create(int grid_steps, int device, lc3d_predictor** out);
int lc3d_predictor_destroy(lc3d_predictor* p);
int lc3d_predictor_set_params(lc3d_predictor* p, const float* params, void* stream);
int lc3d_predictor_get_params(lc3d_predictor* p, float* params, void* stream);
int lc3d_predictor_get_grad(lc3d_predictor* p, float* grad, void* stream);
/* multipliers (host arrays) of the 18 input and 5 output scales */
int lc3d_predictor_set_scales(lc3d_predictor* p, const double* in_mult, const double* out_mult);
/* scales and network input from f1[9] (step t-1) and f2[9] (step t-2) */
int lc3d_predictor_pack(lc3d_predictor* p, const double* const* f1, const double* const* f2, void* stream);
/* the network on the packed input */
int lc3d_predictor_forward(lc3d_predictor* p, void* stream);
/* after pack and forward: pred_f = 2 f1_f - f2_f + o_f output_f for Ex, Ey,
 * Bx, By, Bz, and 2 f1 - f2 for Ez (arrays of 6: Ex, Ey, Ez, Bx, By, Bz) */
int lc3d_predictor_predict(lc3d_predictor* p, const double* const* f1, const double* const* f2,
        double* const* pred, void* stream);
/* training target (first - (2 f1 - f2)) / o from the first-pass fields
 * (arrays of 6 as above; the Ez entries are not used and may be NULL),
 * after pack */
int lc3d_predictor_set_target(lc3d_predictor* p, const double* const* first, const double* const* f1,
        const double* const* f2, void* stream);
/* after lc3d_predictor_forward: mean squared error of the output against the
 * target added to *loss (device float), gradients of all parameters */
int lc3d_predictor_backward(lc3d_predictor* p, float* loss, void* stream);
/* one Adam step (beta 0.9 / 0.999) on the last gradients */
int lc3d_predictor_adam(lc3d_predictor* p, float lr, void* stream);
/* a device buffer of the predictor (LC3D_PRED_*): its address and size */
int lc3d_predictor_tensor(lc3d_predictor* p, int which, void** ptr, long long* bytes);
/* read and clear the predictor's device error flag (LC3D_ERR_TIMEOUT) */
int lc3d_predictor_check_error(lc3d_predictor* p, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LC3D_H */
