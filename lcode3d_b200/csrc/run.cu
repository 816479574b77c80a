// Device-side beam, on-device Ez(0,0) history and graph-replayed xi steps.
//
// The reference evaluates the beam on the host every step, copies it to the
// device (lcode.py:1040, 839) and copies the whole Ez array back to read one
// element (lcode.py:1043-1046). Here a run of many steps needs no host work:
// the benchmark driver
//     rho_b = A exp(-(x^2 + y^2) / (2 sigma_r^2)) 0.5 (1 - cos(sqrt(pi/2) xi / L))
// for 0 <= xi <= 2 sqrt(2 pi) L (else 0), xi = xi_i xi_step_size, is evaluated
// by a kernel from a device xi counter, and Ez at the grid centre is appended
// to a device array after every step. One whole xi step (beam, the 23 solver
// launches, the record) is captured once per state parity into a CUDA graph
// and replayed.

#include <cmath>
#include <cstring>

#include "lc3d_internal.cuh"

namespace {

struct RunCtl {
    int xi;        // xi index of the next step
    int xi0;       // xi index of the first step of the current run
    double* ez;    // history of the current run (may be NULL)
};

__device__ __forceinline__ double beam_value(int k, int N, double h, double xi, double A, double sr, double lf) {
    const int i = k / N, j = k - i * N;
    double v = 0;
    if (xi >= 0 && xi <= 2 * sqrt(2 * M_PI) * lf) {
        const double x = (i - N / 2) * h, y = (j - N / 2) * h;
        v = A * exp(-(x * x + y * y) / (2 * sr * sr)) * 0.5 * (1 - cos(sqrt(M_PI / 2) * xi / lf));
    }
    return v;
}

__global__ void __launch_bounds__(256) beam_kernel(double* out, int N, double h, double dxi, double A, double sr,
                                                   double lf, const RunCtl* ctl) {
    pdl_wait();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N * N) return;
    out[k] = beam_value(k, N, h, ctl->xi * dxi, A, sr, lf);
}

__global__ void __launch_bounds__(256) beam_at_kernel(double* out, int N, double h, double xi, double A, double sr,
                                                      double lf) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= N * N) return;
    out[k] = beam_value(k, N, h, xi, A, sr, lf);
}

__global__ void record_kernel(const double* Ez, int center, RunCtl* ctl) {
    pdl_wait();
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        if (ctl->ez) ctl->ez[ctl->xi - ctl->xi0] = Ez[center];
        ctl->xi += 1;
    }
}

__global__ void set_ctl_kernel(RunCtl* ctl, int xi0, double* ez) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        ctl->xi = xi0;
        ctl->xi0 = xi0;
        ctl->ez = ez;
    }
}

void drop_graphs(lc3d_ctx* c) {
    for (int p = 0; p < 2; ++p)
        if (c->graph[p]) {
            cudaGraphExecDestroy(c->graph[p]);
            c->graph[p] = nullptr;
        }
}

// Enqueue one whole xi step from state parity `par` on `s`: device beam,
// the step, the Ez(0,0) record. Counts its launches into c->launches.
int enqueue_step(lc3d_ctx* c, int par, cudaStream_t s) {
    const int N = c->N;
    {
        ProfScope ps(c, LC3D_STAGE_OTHER, s);
        LC3D_CUDA_TRY(launch_pdl(beam_kernel, dim3((N * N + 255) / 256), dim3(256), 0, s, c->beam_buf, N,
                                 c->p.grid_step_size, c->p.xi_step_size, c->beam_A, c->beam_sr, c->beam_lf,
                                 static_cast<const RunCtl*>(c->run_ctl)));
        LC3D_CUDA_TRY(cudaGetLastError());
    }
    LC3D_TRY(step_schedule(c, c->st[par], c->st[par ^ 1], c->beam_buf, s));
    ProfScope ps(c, LC3D_STAGE_OTHER, s);
    LC3D_CUDA_TRY(launch_pdl(record_kernel, dim3(1), dim3(32), 0, s, static_cast<const double*>(c->st[par ^ 1].Ez),
                             (N / 2) * N + N / 2, static_cast<RunCtl*>(c->run_ctl)));
    LC3D_CUDA_TRY(cudaGetLastError());
    return LC3D_OK;
}

// Segment `seg` of one whole xi step (step_schedule_segment): the device
// beam opens segment 0 and the Ez(0,0) record closes segment 3.
int enqueue_step_segment(lc3d_ctx* c, int par, cudaStream_t s, int seg, DepositArgs* dep) {
    const int N = c->N;
    if (seg == 0) {
        ProfScope ps(c, LC3D_STAGE_OTHER, s);
        LC3D_CUDA_TRY(launch_pdl(beam_kernel, dim3((N * N + 255) / 256), dim3(256), 0, s, c->beam_buf, N,
                                 c->p.grid_step_size, c->p.xi_step_size, c->beam_A, c->beam_sr, c->beam_lf,
                                 static_cast<const RunCtl*>(c->run_ctl)));
        LC3D_CUDA_TRY(cudaGetLastError());
    }
    LC3D_TRY(step_schedule_segment(c, c->st[par], c->st[par ^ 1], c->beam_buf, s, seg, dep));
    if (seg == 3) {
        ProfScope ps(c, LC3D_STAGE_OTHER, s);
        LC3D_CUDA_TRY(launch_pdl(record_kernel, dim3(1), dim3(32), 0, s,
                                 static_cast<const double*>(c->st[par ^ 1].Ez), (N / 2) * N + N / 2,
                                 static_cast<RunCtl*>(c->run_ctl)));
        LC3D_CUDA_TRY(cudaGetLastError());
    }
    return LC3D_OK;
}

// Capture one xi step from state parity `par` into c->graph[par].
int capture(lc3d_ctx* c, int par) {
    cudaStream_t cs;
    LC3D_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    long long saved[LC3D_NSTAGES];
    memcpy(saved, c->launches, sizeof(saved));
    memset(c->launches, 0, sizeof(c->launches));
    int rc = LC3D_OK;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = LC3D_ERR_CUDA;
    } else {
        c->capturing = 1;
        rc = enqueue_step(c, par, cs);
        c->capturing = 0;
        const cudaError_t e = cudaStreamEndCapture(cs, &g);   // always end the capture
        if (rc == LC3D_OK && e != cudaSuccess) {
            lc3d_set_last_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
            rc = LC3D_ERR_CUDA;
        }
    }
    if (rc == LC3D_OK) {
        const cudaError_t e = cudaGraphInstantiate(&c->graph[par], g, 0);
        if (e != cudaSuccess) {
            lc3d_set_last_cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
            rc = LC3D_ERR_CUDA;
            c->graph[par] = nullptr;
        }
    }
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    memcpy(c->graph_launches[par], c->launches, sizeof(c->launches));
    memcpy(c->launches, saved, sizeof(saved));
    return rc;
}

}  // namespace

void run_drop_graphs(lc3d_ctx* c) { drop_graphs(c); }

int run_init(lc3d_ctx* c) {
    LC3D_CUDA_TRY(cudaMalloc(&c->beam_buf, (size_t)c->N * c->N * sizeof(double)));
    LC3D_CUDA_TRY(cudaMemset(c->beam_buf, 0, (size_t)c->N * c->N * sizeof(double)));
    LC3D_CUDA_TRY(cudaMalloc(&c->run_ctl, sizeof(RunCtl)));
    LC3D_CUDA_TRY(cudaMemset(c->run_ctl, 0, sizeof(RunCtl)));
    c->beam_A = 0;
    c->beam_sr = 1;
    c->beam_lf = 1;
    return LC3D_OK;
}

void run_free(lc3d_ctx* c) {
    drop_graphs(c);
    if (c->beam_buf) cudaFree(c->beam_buf);
    if (c->run_ctl) cudaFree(c->run_ctl);
    c->beam_buf = nullptr;
    c->run_ctl = nullptr;
}

extern "C" int lc3d_set_beam(lc3d_ctx* c, const lc3d_beam_params* b) {
    if (!c) return LC3D_ERR_PARAM;
    const double A = b ? b->amplitude : 0.0, sr = b ? b->sigma_r : 1.0, lf = b ? b->length_factor : 1.0;
    if (!(sr > 0) || !(lf > 0) || !std::isfinite(A)) return LC3D_ERR_PARAM;
    if (A != c->beam_A || sr != c->beam_sr || lf != c->beam_lf) {
        int dev = -1;
        cudaGetDevice(&dev);
        if (dev != c->device) cudaSetDevice(c->device);
        cudaDeviceSynchronize();   // no replay of the old graphs may be in flight
        drop_graphs(c);            // the parameters are baked into the graphs
        if (dev >= 0 && dev != c->device) cudaSetDevice(dev);
    }
    c->beam_A = A;
    c->beam_sr = sr;
    c->beam_lf = lf;
    return LC3D_OK;
}

extern "C" int lc3d_beam_eval(lc3d_ctx* c, int xi_i, double* beam_ro, void* stream) {
    if (!c || !beam_ro) return LC3D_ERR_PARAM;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != c->device) cudaSetDevice(c->device);
    const int N = c->N;
    beam_at_kernel<<<(N * N + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        beam_ro, N, c->p.grid_step_size, xi_i * c->p.xi_step_size, c->beam_A, c->beam_sr, c->beam_lf);
    const cudaError_t e = cudaGetLastError();
    if (dev >= 0 && dev != c->device) cudaSetDevice(dev);
    if (e != cudaSuccess) {
        lc3d_set_last_cuda_error(e, "beam_at_kernel", __FILE__, __LINE__);
        return LC3D_ERR_CUDA;
    }
    return LC3D_OK;
}

extern "C" int lc3d_run(lc3d_ctx* c, int xi0, int nsteps, double* ez_history, void* stream) {
    if (!c || nsteps < 0) return LC3D_ERR_PARAM;
    if (c->const_set != 3 || !c->state_set) return LC3D_ERR_STATE;
    if (c->prof_on) return LC3D_ERR_STATE;   // per-launch timing does not see inside graphs
    int prev_dev = -1;
    LC3D_CUDA_TRY(cudaGetDevice(&prev_dev));
    if (prev_dev != c->device) LC3D_CUDA_TRY(cudaSetDevice(c->device));
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int rc = LC3D_OK;
    for (int p = 0; p < 2 && rc == LC3D_OK; ++p)
        if (!c->graph[p]) rc = capture(c, p);
    if (rc == LC3D_OK) {
        set_ctl_kernel<<<1, 32, 0, s>>>(static_cast<RunCtl*>(c->run_ctl), xi0, ez_history);
        if (cudaGetLastError() != cudaSuccess) rc = LC3D_ERR_CUDA;
    }
    for (int k = 0; k < nsteps && rc == LC3D_OK; ++k) {
        const cudaError_t e = cudaGraphLaunch(c->graph[c->cur], s);
        if (e != cudaSuccess) {
            lc3d_set_last_cuda_error(e, "cudaGraphLaunch", __FILE__, __LINE__);
            rc = LC3D_ERR_CUDA;
            break;
        }
        for (int q = 0; q < LC3D_NSTAGES; ++q) c->launches[q] += c->graph_launches[c->cur][q];
        c->cur ^= 1;
    }
    if (prev_dev != c->device) cudaSetDevice(prev_dev);
    return rc;
}

// ---------------------------------------------------------------------------
// Batches of independent simulations (the parameter-scan use case): every
// simulation keeps its own context (own grid size, beam, state); one CUDA
// graph per xi step holds every simulation's whole step on its own parallel
// branch, so one graph launch advances the batch by a step and the branches
// fill the GPU together. Two graphs alternate with the state parity.
// ---------------------------------------------------------------------------

struct lc3d_batch {
    int n, device;
    lc3d_ctx** c;
    int* par0;                 // each context's state parity at capture
    int phase;                 // 0: contexts at par0, 1: at par0 ^ 1
    cudaStream_t cap;          // capture stream
    cudaStream_t* br;          // one branch stream per simulation
    cudaEvent_t fork;
    cudaEvent_t* join;
    cudaGraphExec_t g[2];
    long long launches;        // kernel launches per batch step
    // multi-deposit mode: every deposition point of a step is one launch
    // over all simulations (deposit_multi_kernel) between segments of the
    // simulations' steps
    int multi;
    DepositArgs* dargs;        // device [2 phases][3 depositions][n]
    int* dcta;                 // device [n + 1]: prefix sums of the simulations' tile counts
    int dctas;
};

namespace {

void batch_drop(lc3d_batch* b) {
    for (int p = 0; p < 2; ++p)
        if (b->g[p]) {
            cudaGraphExecDestroy(b->g[p]);
            b->g[p] = nullptr;
        }
}

int batch_capture(lc3d_batch* b, int ph) {
    int rc = LC3D_OK;
    cudaGraph_t g = nullptr;
    long long count = 0;
    if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return LC3D_ERR_CUDA;
    if (cudaEventRecord(b->fork, b->cap) != cudaSuccess) rc = LC3D_ERR_CUDA;
    for (int i = 0; i < b->n && rc == LC3D_OK; ++i) {
        lc3d_ctx* c = b->c[i];
        if (cudaStreamWaitEvent(b->br[i], b->fork, 0) != cudaSuccess) {
            rc = LC3D_ERR_CUDA;
            break;
        }
        long long saved[LC3D_NSTAGES];
        memcpy(saved, c->launches, sizeof(saved));
        memset(c->launches, 0, sizeof(c->launches));
        c->capturing = 1;
        c->one_stream = 1;
        rc = enqueue_step(c, b->par0[i] ^ ph, b->br[i]);
        c->capturing = 0;
        c->one_stream = 0;
        for (int q = 0; q < LC3D_NSTAGES; ++q) count += c->launches[q];
        memcpy(c->graph_launches[b->par0[i] ^ ph], c->launches, sizeof(c->launches));
        memcpy(c->launches, saved, sizeof(saved));
        if (rc == LC3D_OK && (cudaEventRecord(b->join[i], b->br[i]) != cudaSuccess ||
                              cudaStreamWaitEvent(b->cap, b->join[i], 0) != cudaSuccess))
            rc = LC3D_ERR_CUDA;
    }
    const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (rc == LC3D_OK && e != cudaSuccess) {
        lc3d_set_last_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        rc = LC3D_ERR_CUDA;
    }
    if (rc == LC3D_OK) {
        const cudaError_t ei = cudaGraphInstantiate(&b->g[ph], g, 0);
        if (ei != cudaSuccess) {
            lc3d_set_last_cuda_error(ei, "cudaGraphInstantiate", __FILE__, __LINE__);
            b->g[ph] = nullptr;
            rc = LC3D_ERR_CUDA;
        }
    }
    if (g) cudaGraphDestroy(g);
    b->launches = count;
    return rc;
}

// Multi-deposit capture: the step of every simulation in four segments on
// its branch; after segments 0-2 the branches join, one deposit_multi_kernel
// launch does all simulations' depositions, and the branches fork again.
// The depositions' arguments are gathered on the host during the capture and
// copied to b->dargs after it (the graph holds only their device address).
int batch_capture_multi(lc3d_batch* b, int ph) {
    int rc = LC3D_OK;
    cudaGraph_t g = nullptr;
    long long count = 0;
    const int n = b->n;
    DepositArgs* host = new DepositArgs[3 * n]();
    // the launch's work list: tile offsets of the simulations (they depend on
    // the fine lattice only), known before the capture fixes the grid size
    int* start = new int[n + 1];
    start[0] = 0;
    for (int i = 0; i < n; ++i) {
        lc3d_ctx* c = b->c[i];
        DepositArgs t{};
        t.Nf = c->Nf;
        t.fine_off = deposit_fine_offset(c->p.plasma_fineness);
        start[i + 1] = start[i] + deposit_multi_tiles(t);
        memset(c->graph_launches[b->par0[i] ^ ph], 0, sizeof(c->graph_launches[0]));   // gathered over segments
    }
    b->dctas = start[n];
    if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        delete[] host;
        delete[] start;
        return LC3D_ERR_CUDA;
    }
    for (int seg = 0; seg < 4 && rc == LC3D_OK; ++seg) {
        if (cudaEventRecord(b->fork, b->cap) != cudaSuccess) rc = LC3D_ERR_CUDA;
        for (int i = 0; i < n && rc == LC3D_OK; ++i) {
            lc3d_ctx* c = b->c[i];
            const int par = b->par0[i] ^ ph;
            if (cudaStreamWaitEvent(b->br[i], b->fork, 0) != cudaSuccess) {
                rc = LC3D_ERR_CUDA;
                break;
            }
            long long saved[LC3D_NSTAGES];
            memcpy(saved, c->launches, sizeof(saved));
            memset(c->launches, 0, sizeof(c->launches));
            c->capturing = 1;
            c->one_stream = 1;
            DepositArgs dummy{};
            rc = enqueue_step_segment(c, par, b->br[i], seg, seg < 3 ? &host[seg * n + i] : &dummy);
            c->capturing = 0;
            c->one_stream = 0;
            for (int q = 0; q < LC3D_NSTAGES; ++q) {
                count += c->launches[q];
                c->graph_launches[par][q] += c->launches[q];
            }
            memcpy(c->launches, saved, sizeof(saved));
            if (rc == LC3D_OK && (cudaEventRecord(b->join[i], b->br[i]) != cudaSuccess ||
                                  cudaStreamWaitEvent(b->cap, b->join[i], 0) != cudaSuccess))
                rc = LC3D_ERR_CUDA;
        }
        if (seg < 3 && rc == LC3D_OK) {
            rc = launch_deposit_multi(b->dargs + ((size_t)ph * 3 + seg) * n, b->dcta, n, b->dctas, b->cap);
            // the batch's deposition launch is counted on the first simulation's context
            b->c[0]->graph_launches[b->par0[0] ^ ph][LC3D_STAGE_DEPOSIT] += 1;
            count += 1;
        }
    }
    const cudaError_t e = cudaStreamEndCapture(b->cap, &g);
    if (rc == LC3D_OK && e != cudaSuccess) {
        lc3d_set_last_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
        rc = LC3D_ERR_CUDA;
    }
    if (rc == LC3D_OK) {
        const cudaError_t ei = cudaGraphInstantiate(&b->g[ph], g, 0);
        if (ei != cudaSuccess) {
            lc3d_set_last_cuda_error(ei, "cudaGraphInstantiate", __FILE__, __LINE__);
            b->g[ph] = nullptr;
            rc = LC3D_ERR_CUDA;
        }
    }
    if (g) cudaGraphDestroy(g);
    if (rc == LC3D_OK) {
        // the work list and this phase's deposition arguments, before any replay
        cudaError_t ec = cudaMemcpy(b->dcta, start, (size_t)(n + 1) * sizeof(int), cudaMemcpyHostToDevice);
        if (ec == cudaSuccess)
            ec = cudaMemcpy(b->dargs + (size_t)ph * 3 * n, host, (size_t)3 * n * sizeof(DepositArgs),
                            cudaMemcpyHostToDevice);
        if (ec != cudaSuccess) {
            lc3d_set_last_cuda_error(ec, "cudaMemcpy", __FILE__, __LINE__);
            rc = LC3D_ERR_CUDA;
        }
    }
    delete[] start;
    delete[] host;
    b->launches = count;
    return rc;
}

void batch_free(lc3d_batch* b) {
    if (!b) return;
    batch_drop(b);
    if (b->dargs) cudaFree(b->dargs);
    if (b->dcta) cudaFree(b->dcta);
    if (b->br)
        for (int i = 0; i < b->n; ++i)
            if (b->br[i]) cudaStreamDestroy(b->br[i]);
    if (b->join)
        for (int i = 0; i < b->n; ++i)
            if (b->join[i]) cudaEventDestroy(b->join[i]);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete[] b->c;
    delete[] b->par0;
    delete[] b->br;
    delete[] b->join;
    delete b;
}

}  // namespace

extern "C" int lc3d_batch_create(lc3d_ctx* const* ctxs, int count, lc3d_batch** out) {
    if (!ctxs || count < 1 || !out) return LC3D_ERR_PARAM;
    *out = nullptr;
    const int dev = ctxs[0] ? ctxs[0]->device : -1;
    for (int i = 0; i < count; ++i)
        if (!ctxs[i] || ctxs[i]->device != dev) return LC3D_ERR_PARAM;
    int prev = -1;
    LC3D_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != dev) LC3D_CUDA_TRY(cudaSetDevice(dev));
    lc3d_batch* b = new lc3d_batch;
    memset(b, 0, sizeof(*b));
    b->n = count;
    b->device = dev;
    b->c = new lc3d_ctx*[count];
    b->par0 = new int[count];
    b->br = new cudaStream_t[count]();
    b->join = new cudaEvent_t[count]();
    int rc = LC3D_OK;
    for (int i = 0; i < count; ++i) b->c[i] = ctxs[i];
    if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        rc = LC3D_ERR_CUDA;
    for (int i = 0; i < count && rc == LC3D_OK; ++i)
        if (cudaStreamCreateWithFlags(&b->br[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) != cudaSuccess)
            rc = LC3D_ERR_CUDA;
    if (prev != dev) cudaSetDevice(prev);
    if (rc != LC3D_OK) {
        batch_free(b);
        return rc;
    }
    *out = b;
    return LC3D_OK;
}

extern "C" int lc3d_batch_set_mode(lc3d_batch* b, int multi_deposit) {
    if (!b || (multi_deposit != 0 && multi_deposit != 1)) return LC3D_ERR_PARAM;
    int prev = -1;
    LC3D_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != b->device) LC3D_CUDA_TRY(cudaSetDevice(b->device));
    int rc = LC3D_OK;
    if (cudaDeviceSynchronize() != cudaSuccess) rc = LC3D_ERR_CUDA;   // no replay of the old graphs in flight
    if (rc == LC3D_OK) {
        batch_drop(b);   // captured again, in the new form, by the next run
        b->multi = multi_deposit;
        if (multi_deposit && !b->dargs) {
            if (cudaMalloc(&b->dargs, (size_t)6 * b->n * sizeof(DepositArgs)) != cudaSuccess ||
                cudaMalloc(&b->dcta, (size_t)(b->n + 1) * sizeof(int)) != cudaSuccess)
                rc = LC3D_ERR_CUDA;
        }
    }
    if (prev != b->device) cudaSetDevice(prev);
    return rc;
}

extern "C" int lc3d_batch_destroy(lc3d_batch* b) {
    if (!b) return LC3D_OK;
    cudaDeviceSynchronize();
    batch_free(b);
    return LC3D_OK;
}

extern "C" int lc3d_batch_run(lc3d_batch* b, const int* xi0, int nsteps, double* const* ez_history,
                              void* stream) {
    if (!b || !xi0 || nsteps < 0) return LC3D_ERR_PARAM;
    for (int i = 0; i < b->n; ++i) {
        lc3d_ctx* c = b->c[i];
        if (c->const_set != 3 || !c->state_set) return LC3D_ERR_STATE;
        if (c->prof_on) return LC3D_ERR_STATE;
    }
    int prev = -1;
    LC3D_CUDA_TRY(cudaGetDevice(&prev));
    if (prev != b->device) LC3D_CUDA_TRY(cudaSetDevice(b->device));
    const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int rc = LC3D_OK;
    // (re)capture when a context was stepped on its own or its beam changed
    bool fresh = b->g[0] && b->g[1];
    for (int i = 0; i < b->n && fresh; ++i)
        if (b->c[i]->cur != (b->par0[i] ^ b->phase) || !b->c[i]->graph[0]) fresh = false;
    if (!fresh) {
        batch_drop(b);
        b->phase = 0;
        for (int i = 0; i < b->n; ++i) {
            b->par0[i] = b->c[i]->cur;
            // mark the single-context graphs valid so lc3d_set_beam can drop
            // them (and with them this batch's graphs) on a beam change
            if (!b->c[i]->graph[0] && rc == LC3D_OK) rc = capture(b->c[i], 0);
            if (!b->c[i]->graph[1] && rc == LC3D_OK) rc = capture(b->c[i], 1);
        }
        for (int ph = 0; ph < 2 && rc == LC3D_OK; ++ph) rc = b->multi ? batch_capture_multi(b, ph) : batch_capture(b, ph);
    }
    for (int i = 0; i < b->n && rc == LC3D_OK; ++i) {
        set_ctl_kernel<<<1, 32, 0, s>>>(static_cast<RunCtl*>(b->c[i]->run_ctl), xi0[i],
                                        ez_history ? ez_history[i] : nullptr);
        if (cudaGetLastError() != cudaSuccess) rc = LC3D_ERR_CUDA;
    }
    for (int k = 0; k < nsteps && rc == LC3D_OK; ++k) {
        const cudaError_t e = cudaGraphLaunch(b->g[b->phase], s);
        if (e != cudaSuccess) {
            lc3d_set_last_cuda_error(e, "cudaGraphLaunch", __FILE__, __LINE__);
            rc = LC3D_ERR_CUDA;
            break;
        }
        for (int i = 0; i < b->n; ++i) {
            lc3d_ctx* c = b->c[i];
            for (int q = 0; q < LC3D_NSTAGES; ++q) c->launches[q] += c->graph_launches[c->cur][q];
            c->cur ^= 1;
        }
        b->phase ^= 1;
    }
    if (prev != b->device) cudaSetDevice(prev);
    return rc;
}
